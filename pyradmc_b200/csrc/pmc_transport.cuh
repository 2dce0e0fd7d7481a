// pmc_transport.cuh — the persistent photon and electron transport kernels.
//
// Behavioural spec: photon_kernel / electron_kernel of
// pyradmc/backends/warp/kernels.py:1171-1885, which mirror the reference loops
// transport/photon.py:100-282 and transport/electron.py:207-482 statement for
// statement.  The structure is B200-first rather than a translation:
//   * persistent grids (a multiple of the SM count) with per-lane refill: a
//     lane whose particle ends takes the next one at once, from the input
//     queue first and then from the batch's primary cursor, so no lane idles
//     behind the longest particle of its warp;
//   * photon primaries are generated inside the photon kernel and never touch
//     a queue;
//   * queue rotation, the primary admission window and the "work left" flag
//     are advanced on the device by the last block of each kernel, so a whole
//     batch drains without one host round trip (and inside one CUDA graph);
//   * energy books and event counters accumulate in shared memory and reach
//     global memory once per block.
#pragma once

#include <cooperative_groups.h>

#include "pmc_common.cuh"
#include "pmc_physics.cuh"

namespace pmc {

namespace cg = cooperative_groups;

// Flags raised on the device and reported by the host after a batch.
constexpr int kFlagOverflow = 1;
constexpr int kFlagStepCap = 2;
constexpr int kFlagRoundCap = 4;

// Device-resident scheduling state of one drain (one statistical batch).
struct Sched {
    int p_in, e_in;                 // input photon / electron queue (0/1)
    unsigned int count[4];          // push counters: P0, P1, E0, E1
    unsigned int head[4];           // fetch heads
    unsigned long long cursor;      // next primary of the batch block
    unsigned long long limit;       // admission limit of the current round
    unsigned long long block_end;   // primaries in the batch block
    unsigned long long budget;      // primaries admitted per round
    unsigned int blocks_done;
    int flags;
    int remaining;                  // 1 while work is left
    int batch;
    long long rounds;               // rounds of the current batch
    long long total_rounds;         // rounds of the whole call (not reset per batch)
    long long max_rounds;
    unsigned long long cond_handle; // CUDA graph conditional handle (0: host loop)
};

// Primary generator of the current group (device-resident).
struct GenDesc {
    int type;           // 0 pencil, 1 parallel/lattice, 2 spectral fan, 3 upload
    int kind;           // particle kind of analytic primaries
    int forward;        // 1: open-field run (history = batch * per_batch + t)
    int correlated;
    int group;          // columns in this group
    int n_bins;
    float energy;
    float px, py, pz, dx, dy, dz;       // pencil
    float z0;                            // parallel / lattice
    float fx, fy, fz;                    // spectral focal point
    float uax, uay, uaz, vax, vay, vaz;  // aperture axes
    float width_u, width_v;
    long long per_batch_fwd;             // forward: histories per batch
    const long long* pb_prefix;          // [group+1] exclusive prefix of per-batch counts
    const long long* per_batch;          // [group]
    const long long* hist_offset;        // [group] first global history of each beamlet
    const float* x_lo;                   // [group] lattice bounds
    const float* x_ext;
    const float* y_lo;
    const float* y_ext;
    const float* cx;                     // [group] spectral centres
    const float* cy;
    const float* cz;
    const float* edges;                  // [n_bins+1]
    const float* cdf;                    // [n_bins]
    const int* up_kind;                  // upload route, [n_histories]
    const float* up_energy;
    const float* up_pos;
    const float* up_dir;
    const float* up_weight;
    int book_emitted;                    // spectral/upload: book emitted energy per primary
};

struct Counters {
    unsigned long long flights, interactions, substeps, deposits, pushes, primaries;
    long long escaped, unscored, deposited, emitted, violations;
};

struct TransportParams {
    GridInfo gi;          // transport grid
    GridInfo si;          // scoring grid
    const float2* vox;    // (density, material bits) per transport voxel
    Tables tab;
    Slot* q[4];           // P0, P1, E0, E1
    unsigned int capacity;
    Sched* sched;
    const GenDesc* gen;
    unsigned long long* edep;  // [group][n_scoring_voxels] int64 quanta
    Counters* counters;
    uint32_t seed_lo, seed_hi;
    float pcut, ecut;
    float step_fraction;
    float deposit_resolution;
    int transport_electrons;
    int msc_gs;
    int dose_to_water;
    int split_n;
    long long max_steps;
};

// ---- per-block books ------------------------------------------------------------
struct BlockBooks {
    unsigned long long flights, interactions, substeps, deposits, pushes, primaries;
    long long escaped, unscored, deposited, emitted, violations;
};

__device__ __forceinline__ long long quantize_signed(float amount) {
    return (long long)floor((double)amount * kInvQuantum + 0.5);
}

__device__ __forceinline__ void book_add(long long* slot, long long v) {
    if (v != 0) atomicAdd((unsigned long long*)slot, (unsigned long long)v);
}

// kernels.py:459 _spr_factor: restricted-stopping ratio water/medium, exactly 1
// under dose-to-medium and for water deposits.
__device__ __forceinline__ float spr_factor(const TransportParams& P, float e, int mat) {
    if (P.dose_to_water == 0 || mat == kWater) return 1.0f;
    const LogIdx li = log_index(fmaxf(e, P.ecut), P.tab.e_log_min, P.tab.e_inv_dlog, P.tab.n_points);
    const float sw = lerp1(P.tab.ec + (long long)kWater * P.tab.n_points, li);
    const float sm = lerp1(P.tab.ec + (long long)mat * P.tab.n_points, li);
    return sw / sm;
}

// Where a deposit's quanta go.  DirectSink issues one atomic per deposit;
// HeldSink keeps one pending (entry, quanta) pair in registers and merges the
// next deposit into it when it lands in the same entry — an electron's two
// half-substep deposits and its next substep's usually do — so a run of
// deposits into one voxel costs one atomic.  Integer sums: merging is exact.
struct DirectSink {
    unsigned long long n = 0;  // atomics issued
    __device__ __forceinline__ void add(const TransportParams& P, long long flat,
                                        unsigned long long q) {
        atomicAdd(P.edep + flat, q);
        ++n;
    }
};

struct HeldSink {
    long long idx = -1;
    unsigned long long q = 0;
    unsigned long long n = 0;
    __device__ __forceinline__ void add(const TransportParams& P, long long flat,
                                        unsigned long long quanta) {
        if (flat == idx) {
            q += quanta;
            return;
        }
        release(P);
        idx = flat;
        q = quanta;
    }
    __device__ __forceinline__ void release(const TransportParams& P) {
        if (q != 0ull) {
            atomicAdd(P.edep + idx, q);
            ++n;
        }
        idx = -1;
        q = 0ull;
    }
};

// kernels.py:536 _deposit: quantize once, route by position into the scoring
// grid of this particle's column, or into the unscored book.
template <class Sink>
__device__ __forceinline__ void deposit(const TransportParams& P, BlockBooks& B, long long base,
                                       float x, float y, float z, float amount, float factor,
                                       Sink& sink) {
    if (point_inside(x, y, z, P.si)) {
        const long long idx = flat_index(x, y, z, P.si);
        const long long q =
            (long long)((double)amount * (double)factor * kInvQuantum + 0.5);
        if (q != 0) sink.add(P, base + idx, (unsigned long long)q);
        if (P.dose_to_water) {
            book_add(&B.deposited, (long long)((double)amount * kInvQuantum + 0.5));
        }
    } else {
        book_add(&B.unscored, (long long)((double)amount * kInvQuantum + 0.5));
    }
}

__device__ __forceinline__ void escape(BlockBooks& B, float amount) {
    book_add(&B.escaped, quantize_signed(amount));
}

// kernels.py:600 _deposit_or_escape: escape is decided on the transport grid.
template <class Sink>
__device__ __forceinline__ void deposit_or_escape(const TransportParams& P, BlockBooks& B,
                                                  long long base, float x, float y, float z,
                                                  float amount, float factor, Sink& sink) {
    if (amount <= 0.0f) return;
    if (point_inside(x, y, z, P.gi)) deposit(P, B, base, x, y, z, amount, factor, sink);
    else escape(B, amount);
}

// kernels.py:631 _deposit_spread: equal pieces at piece midpoints.
template <class Sink>
__device__ inline void deposit_spread(const TransportParams& P, BlockBooks& B, long long base,
                                      float x, float y, float z, float ux, float uy, float uz,
                                      float length, float amount, float factor, Sink& sink) {
    const int n = substep_pieces(length, P.deposit_resolution);
    const float share = amount / (float)n;
    const float piece = length / (float)n;
    for (int k = 0; k < n; ++k) {
        const float t = ((float)k + 0.5f) * piece;
        deposit_or_escape(P, B, base, x + ux * t, y + uy * t, z + uz * t, share, factor, sink);
    }
}

// Warp-aggregated queue push (one atomic per converged group of pushing lanes).
__device__ __forceinline__ void queue_push(const TransportParams& P, int qi, int kind, int beamlet,
                                           float e, float w, float x, float y, float z, float ux,
                                           float uy, float uz, const StreamId& sid,
                                           unsigned long long& n_push) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(&P.sched->count[qi], (unsigned int)g.size());
    base = g.shfl(base, 0);
    const unsigned int idx = base + g.thread_rank();
    ++n_push;
    if (idx >= P.capacity) {
        atomicOr(&P.sched->flags, kFlagOverflow);
        return;
    }
    Slot* s = P.q[qi] + idx;
    s->a = make_float4(e, w, x, y);
    s->b = make_float4(z, ux, uy, uz);
    s->c = make_uint4(sid.id_lo, sid.id_hi, sid.tag, sid.ctr);
    s->d = make_uint4(pack_meta(kind, 0, beamlet), 0u, 0u, 0u);
}

__device__ __forceinline__ unsigned long long fetch_one(unsigned long long* ctr) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned long long base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, (unsigned long long)g.size());
    base = g.shfl(base, 0);
    return base + g.thread_rank();
}
__device__ __forceinline__ unsigned int fetch_one(unsigned int* ctr) {
    cg::coalesced_group g = cg::coalesced_threads();
    unsigned int base = 0;
    if (g.thread_rank() == 0) base = atomicAdd(ctr, (unsigned int)g.size());
    base = g.shfl(base, 0);
    return base + g.thread_rank();
}

// ---- particle state ----------------------------------------------------------------
struct Particle {
    float e, w, x, y, z, ux, uy, uz;
    int kind, primary, beamlet;
    long long steps;
    Rng rng;
};

__device__ __forceinline__ void load_slot(const TransportParams& P, const Slot* q, unsigned int i,
                                          Particle& p) {
    const Slot* s = q + i;
    const float4 a = s->a, b = s->b;
    const uint4 c = s->c, d = s->d;
    p.e = a.x; p.w = a.y; p.x = a.z; p.y = a.w;
    p.z = b.x; p.ux = b.y; p.uy = b.z; p.uz = b.w;
    p.kind = (int)(d.x & 3u);
    p.primary = (int)((d.x >> 2) & 1u);
    p.beamlet = (int)(d.x >> 3);
    p.steps = 0;
    p.rng.load(P.seed_lo, P.seed_hi, StreamId{c.x, c.y, c.z, c.w});
}

// Vacuum flight to the grid for a particle born outside (photon.py:137-148);
// returns false (energy escaped) when the flight misses the grid.
__device__ __forceinline__ bool enter_grid(const TransportParams& P, BlockBooks& B, Particle& p,
                                           float latent) {
    if (point_inside(p.x, p.y, p.z, P.gi)) return true;
    float t = slab_entry_distance(p.x, p.y, p.z, p.ux, p.uy, p.uz, P.gi);
    if (t >= kInfinityCm) {
        escape(B, p.w * (p.e + latent));
        return false;
    }
    t += kEntryNudge;
    p.x += t * p.ux;
    p.y += t * p.uy;
    p.z += t * p.uz;
    if (!point_inside(p.x, p.y, p.z, P.gi)) {
        escape(B, p.w * (p.e + latent));
        return false;
    }
    return true;
}

// ---- primary generation (kernels.py:1888-2401) -------------------------------------
// Maps primary t of the current batch block to its beamlet and history, seeds
// the history's stream, and samples the primary exactly as the host sources do
// (same uniforms, same order).  Returns the particle kind.
__device__ inline int generate_primary(const TransportParams& P, const GenDesc& G, int batch,
                                       unsigned long long t, Particle& p, BlockBooks& B) {
    // G is the device-resident descriptor, read field by field as needed.
    int local = 0;
    long long key;
    long long record;
    if (G.forward) {
        key = (long long)batch * G.per_batch_fwd + (long long)t;
        record = key;
    } else {
        int lo = 0, hi = G.group;  // largest local with pb_prefix[local] <= t
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if ((unsigned long long)__ldg(G.pb_prefix + mid) <= t) lo = mid;
            else hi = mid;
        }
        local = lo;
        const long long i = (long long)t - __ldg(G.pb_prefix + local);
        const long long r = (long long)batch * __ldg(G.per_batch + local) + i;
        const long long h = __ldg(G.hist_offset + local) + r;
        key = G.correlated ? r : h;
        record = h;
    }
    p.rng.k0 = P.seed_lo;
    p.rng.k1 = P.seed_hi;
    p.rng.id_lo = (uint32_t)((unsigned long long)key & 0xffffffffull);
    p.rng.id_hi = (uint32_t)((unsigned long long)key >> 32);
    p.rng.tag = 0u;
    p.rng.ctr = 0u;
    p.beamlet = local;
    p.primary = 1;
    p.steps = 0;
    p.w = 1.0f;
    p.kind = G.kind;
    if (G.type == 0) {  // pencil: no draws
        p.e = G.energy;
        p.x = G.px; p.y = G.py; p.z = G.pz;
        p.ux = G.dx; p.uy = G.dy; p.uz = G.dz;
    } else if (G.type == 1) {  // parallel field / beamlet lattice: two uniforms
        p.e = G.energy;
        p.x = __ldg(G.x_lo + local) + __ldg(G.x_ext + local) * p.rng.uniform();
        p.y = __ldg(G.y_lo + local) + __ldg(G.y_ext + local) * p.rng.uniform();
        p.z = G.z0;
        p.ux = 0.0f; p.uy = 0.0f; p.uz = 1.0f;
    } else if (G.type == 2) {  // divergent spectral fan: four uniforms
        const float u_bin = p.rng.uniform();
        const float u_within = p.rng.uniform();
        const float du = (p.rng.uniform() - 0.5f) * G.width_u;
        const float dv = (p.rng.uniform() - 0.5f) * G.width_v;
        int lo = 0, hi = G.n_bins;  // lower_bound: first k with cdf[k] >= u_bin
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(G.cdf + mid) < u_bin) lo = mid + 1;
            else hi = mid;
        }
        const int k = min(lo, G.n_bins - 1);
        const float e_lo = __ldg(G.edges + k);
        p.e = e_lo + (__ldg(G.edges + k + 1) - e_lo) * u_within;
        const float dx = __ldg(G.cx + local) + du * G.uax + dv * G.vax - G.fx;
        const float dy = __ldg(G.cy + local) + du * G.uay + dv * G.vay - G.fy;
        const float dz = __ldg(G.cz + local) + du * G.uaz + dv * G.vaz - G.fz;
        const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
        p.x = G.fx; p.y = G.fy; p.z = G.fz;
        p.ux = dx * inv; p.uy = dy * inv; p.uz = dz * inv;
    } else {  // host-sampled record
        p.kind = __ldg(G.up_kind + record);
        p.e = __ldg(G.up_energy + record);
        p.w = __ldg(G.up_weight + record);
        p.x = __ldg(G.up_pos + 3 * record);
        p.y = __ldg(G.up_pos + 3 * record + 1);
        p.z = __ldg(G.up_pos + 3 * record + 2);
        p.ux = __ldg(G.up_dir + 3 * record);
        p.uy = __ldg(G.up_dir + 3 * record + 1);
        p.uz = __ldg(G.up_dir + 3 * record + 2);
    }
    if (G.book_emitted) {
        const float latent = p.kind == kPositron ? 2.0f * kElectronMass : 0.0f;
        book_add(&B.emitted, quantize_signed(p.w * (p.e + latent)));
    }
    return p.kind;
}

// ---- annihilation at rest (transport/particles.py:75, kernels.py:675) ------------
template <class Sink>
__device__ inline void annihilate_at_rest(const TransportParams& P, BlockBooks& B, Particle& p,
                                          long long base, int q_photon, float factor, Sink& sink,
                                          unsigned long long& n_push) {
    if (P.pcut >= kElectronMass) {
        deposit(P, B, base, p.x, p.y, p.z, p.w * 2.0f * kElectronMass, factor, sink);
        return;
    }
    float ax, ay, az;
    sample_isotropic_direction(p.rng, ax, ay, az);
    const StreamId s1 = p.rng.spawn();
    queue_push(P, q_photon, kPhoton, p.beamlet, kElectronMass, p.w, p.x, p.y, p.z, ax, ay, az, s1,
               n_push);
    const StreamId s2 = p.rng.spawn();
    queue_push(P, q_photon, kPhoton, p.beamlet, kElectronMass, p.w, p.x, p.y, p.z, -ax, -ay, -az,
               s2, n_push);
}

// ---- last-block scheduler steps ------------------------------------------------------
__device__ inline bool last_block_arrives(Sched* S) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned int done = atomicAdd(&S->blocks_done, 1u);
        last = (done == gridDim.x - 1);
    }
    __syncthreads();
    return last;
}

__device__ inline void flush_books(const TransportParams& P, BlockBooks& B) {
    __syncthreads();
    if (threadIdx.x == 0) {
        Counters* C = P.counters;
        if (B.flights) atomicAdd(&C->flights, B.flights);
        if (B.interactions) atomicAdd(&C->interactions, B.interactions);
        if (B.substeps) atomicAdd(&C->substeps, B.substeps);
        if (B.deposits) atomicAdd(&C->deposits, B.deposits);
        if (B.pushes) atomicAdd(&C->pushes, B.pushes);
        if (B.primaries) atomicAdd(&C->primaries, B.primaries);
        book_add(&C->escaped, B.escaped);
        book_add(&C->unscored, B.unscored);
        book_add(&C->deposited, B.deposited);
        book_add(&C->emitted, B.emitted);
        book_add(&C->violations, B.violations);
    }
}

__device__ __forceinline__ void init_books(BlockBooks& B) {
    if (threadIdx.x == 0) {
        B.flights = B.interactions = B.substeps = B.deposits = B.pushes = B.primaries = 0ull;
        B.escaped = B.unscored = B.deposited = B.emitted = B.violations = 0ll;
    }
    __syncthreads();
}

__device__ __forceinline__ void block_sum_add(unsigned long long* dst, unsigned long long v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// ---- the photon kernel ---------------------------------------------------------------
// One lane transports one photon to termination (Woodcock tracking), then takes
// the next: queued photons first, then fresh primaries of the batch block.
__global__ void __launch_bounds__(256, 3) photon_kernel(TransportParams P) {
    __shared__ BlockBooks B;
    init_books(B);
    Sched* S = P.sched;
    const int pin = S->p_in, ein = S->e_in;
    const int q_in = pin, q_out = pin ^ 1, q_el = 2 + ein;
    const unsigned int n_in = min(S->count[q_in], P.capacity);
    const unsigned long long limit = S->limit;
    const int batch = S->batch;
    const GenDesc& G = *P.gen;
    const Tables& T = P.tab;
    const float pcut = P.pcut, ecut = P.ecut;

    unsigned long long n_flight = 0, n_inter = 0, n_push = 0, n_prim = 0;
    DirectSink dep;
    Particle p;
    bool active = false, exhausted = false;
    float e_tab = -1.0f, maj = 0.0f;
    LogIdx li{0, 0.0f};
    int mat_tab = -1;
    float4 ch = make_float4(0.f, 0.f, 0.f, 0.f);
    long long base = 0;

    for (unsigned int it = 0;; ++it) {
        if ((it & 255u) == 0u) {
            if (__any_sync(0xffffffffu, (*(volatile int*)&S->flags) & (kFlagOverflow | kFlagStepCap)))
                break;
        }
        if (!active && !exhausted) {
            const unsigned int i = fetch_one(&S->head[q_in]);
            bool got = false;
            if (i < n_in) {
                load_slot(P, P.q[q_in], i, p);
                got = true;
            } else {
                const unsigned long long t = fetch_one(&S->cursor);
                if (t < limit) {
                    ++n_prim;
                    const int kind = generate_primary(P, G, batch, t, p, B);
                    if (kind == kPhoton) {
                        got = true;
                    } else {  // charged primary: hand to the electron queue unchanged
                        queue_push(P, q_el, kind, p.beamlet, p.e, p.w, p.x, p.y, p.z, p.ux, p.uy,
                                   p.uz, p.rng.state(), n_push);
                    }
                } else {
                    exhausted = true;
                }
            }
            if (got) {
                active = enter_grid(P, B, p, 0.0f);
                base = (long long)p.beamlet * P.si.n_voxels;
                e_tab = -1.0f;
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted)) break;
        if (!active) continue;

        // ---- one Woodcock flight (photon.py:150-181) ----
        if (++p.steps > P.max_steps) {
            atomicOr(&S->flags, kFlagStepCap);
            escape(B, p.w * p.e);
            active = false;
            continue;
        }
        if (p.e != e_tab) {
            li = log_index(p.e, T.p_log_min, T.p_inv_dlog, T.n_points);
            maj = lerp1(T.maj, li);
            e_tab = p.e;
            mat_tab = -1;
        }
        ++n_flight;
        const float step = sample_path_length(maj, p.rng);
        p.x += step * p.ux;
        p.y += step * p.uy;
        p.z += step * p.uz;
        if (!point_inside(p.x, p.y, p.z, P.gi)) {
            escape(B, p.w * p.e);
            active = false;
            continue;
        }
        const float2 vx = __ldg(P.vox + flat_index(p.x, p.y, p.z, P.gi));
        const float rho = vx.x;
        const int mat = __float_as_int(vx.y);
        if (mat != mat_tab) {
            ch = lerp4(T.ch + (long long)mat * T.n_points, li);
            mat_tab = mat;
        }
        const float mc = rho * ch.x, mp = rho * ch.y, mpa = rho * ch.z, mr = rho * ch.w;
        const float mu_real = mc + mp + mpa + mr;
        if (mu_real > maj * (1.0f + 1.0e-9f)) {
            book_add(&B.violations, 1);
            escape(B, p.w * p.e);
            active = false;
            continue;
        }
        if (p.rng.uniform() * maj >= mu_real) continue;  // delta scattering
        ++n_inter;
        const int process = select_photon_process(mc, mp, mpa, mr, p.rng);

        if (process == 3) {  // coherent
            const float c = sample_coherent_cos_theta(T, mat, p.e, p.rng);
            const float phi = kTwoPi * p.rng.uniform();
            rotate_direction(p.ux, p.uy, p.uz, c, phi);
        } else if (process == 0) {  // Compton
            if (P.split_n > 1 && p.primary) {
                // Compton splitting of a source photon (photon.py:190-224): N
                // copies of weight w/N, each pushed as a non-primary photon.
                const float split_w = p.w / (float)P.split_n;
                for (int k = 0; k < P.split_n; ++k) {
                    const float ratio = sample_compton_energy_ratio(p.e, p.rng);
                    const float recoil = p.e * (1.0f - ratio);
                    const float phi = kTwoPi * p.rng.uniform();
                    if (P.transport_electrons && recoil > ecut) {
                        float ex = p.ux, ey = p.uy, ez = p.uz;
                        rotate_direction(ex, ey, ez, compton_electron_cos_theta(p.e, ratio),
                                         phi + kPi);
                        const StreamId sid = p.rng.spawn();
                        queue_push(P, q_el, kElectron, p.beamlet, recoil, split_w, p.x, p.y, p.z,
                                   ex, ey, ez, sid, n_push);
                    } else {
                        deposit(P, B, base, p.x, p.y, p.z, split_w * recoil,
                                spr_factor(P, recoil, mat), dep);
                    }
                    float gx = p.ux, gy = p.uy, gz = p.uz;
                    rotate_direction(gx, gy, gz, compton_cos_theta(p.e, ratio), phi);
                    const float es = p.e * ratio;
                    if (es <= pcut) {
                        deposit(P, B, base, p.x, p.y, p.z, split_w * es, spr_factor(P, es, mat),
                                dep);
                        continue;
                    }
                    float cw = split_w;
                    bool keep = true;
                    if (es < kRouletteMeV && cw < kRouletteWeightCap) {
                        const float nw = roulette_weight(cw, kRouletteSurvival, p.rng);
                        escape(B, (cw - nw) * es);
                        if (nw == 0.0f) keep = false;
                        else cw = nw;
                    }
                    if (keep) {
                        const StreamId sid = p.rng.spawn();
                        queue_push(P, q_out, kPhoton, p.beamlet, es, cw, p.x, p.y, p.z, gx, gy, gz,
                                   sid, n_push);
                    }
                }
                active = false;
                continue;
            }
            const float ratio = sample_compton_energy_ratio(p.e, p.rng);
            const float recoil = p.e * (1.0f - ratio);
            const float phi = kTwoPi * p.rng.uniform();
            if (P.transport_electrons && recoil > ecut) {
                float ex = p.ux, ey = p.uy, ez = p.uz;
                rotate_direction(ex, ey, ez, compton_electron_cos_theta(p.e, ratio), phi + kPi);
                const StreamId sid = p.rng.spawn();
                queue_push(P, q_el, kElectron, p.beamlet, recoil, p.w, p.x, p.y, p.z, ex, ey, ez,
                           sid, n_push);
            } else {
                deposit(P, B, base, p.x, p.y, p.z, p.w * recoil, spr_factor(P, recoil, mat), dep);
            }
            rotate_direction(p.ux, p.uy, p.uz, compton_cos_theta(p.e, ratio), phi);
            p.e *= ratio;
            if (p.e <= pcut) {
                deposit(P, B, base, p.x, p.y, p.z, p.w * p.e, spr_factor(P, p.e, mat), dep);
                active = false;
                continue;
            }
            if (p.e < kRouletteMeV && p.w < kRouletteWeightCap) {
                const float nw = roulette_weight(p.w, kRouletteSurvival, p.rng);
                escape(B, (p.w - nw) * p.e);
                if (nw == 0.0f) {
                    active = false;
                    continue;
                }
                p.w = nw;
            }
        } else if (process == 1) {  // photoelectric: forward, no fluorescence
            if (P.transport_electrons && p.e > ecut) {
                const StreamId sid = p.rng.spawn();
                queue_push(P, q_el, kElectron, p.beamlet, p.e, p.w, p.x, p.y, p.z, p.ux, p.uy,
                           p.uz, sid, n_push);
            } else {
                deposit(P, B, base, p.x, p.y, p.z, p.w * p.e, spr_factor(P, p.e, mat), dep);
            }
            active = false;
        } else {  // pair production
            const float kinetic = p.e - 2.0f * kElectronMass;
            if (P.transport_electrons) {
                const float fraction = p.rng.uniform();
                const float share_e = fraction * kinetic;
                const float share_p = (1.0f - fraction) * kinetic;
                if (share_e > ecut) {
                    const StreamId sid = p.rng.spawn();
                    queue_push(P, q_el, kElectron, p.beamlet, share_e, p.w, p.x, p.y, p.z, p.ux,
                               p.uy, p.uz, sid, n_push);
                } else {
                    deposit(P, B, base, p.x, p.y, p.z, p.w * share_e, spr_factor(P, share_e, mat),
                            dep);
                }
                if (share_p > ecut) {
                    const StreamId sid = p.rng.spawn();
                    queue_push(P, q_el, kPositron, p.beamlet, share_p, p.w, p.x, p.y, p.z, p.ux,
                               p.uy, p.uz, sid, n_push);
                } else {
                    deposit(P, B, base, p.x, p.y, p.z, p.w * share_p, spr_factor(P, share_p, mat),
                            dep);
                    annihilate_at_rest(P, B, p, base, q_out, spr_factor(P, kElectronMass, mat),
                                       dep, n_push);
                }
            } else {
                deposit(P, B, base, p.x, p.y, p.z, p.w * kinetic, spr_factor(P, kinetic, mat),
                        dep);
                annihilate_at_rest(P, B, p, base, q_out, spr_factor(P, kElectronMass, mat), dep,
                                   n_push);
            }
            active = false;
        }
    }

    block_sum_add(&B.flights, n_flight);
    block_sum_add(&B.interactions, n_inter);
    block_sum_add(&B.deposits, dep.n);
    block_sum_add(&B.pushes, n_push);
    block_sum_add(&B.primaries, n_prim);
    flush_books(P, B);

    // The last block retires the consumed photon queue and clamps the cursor.
    if (last_block_arrives(S) && threadIdx.x == 0) {
        S->count[q_in] = 0u;
        S->head[q_in] = 0u;
        S->p_in = q_out;
        if (S->cursor > S->limit) S->cursor = S->limit;
        S->blocks_done = 0u;
        __threadfence();
    }
}

// ---- the electron kernel -------------------------------------------------------------
// One lane runs one electron or positron to ECUT (Class II condensed history,
// electron.py:345-481); delta rays go to the next round's electron queue,
// bremsstrahlung and annihilation photons to the next photon round.
__global__ void __launch_bounds__(256, 4) electron_kernel(TransportParams P) {
    __shared__ BlockBooks B;
    init_books(B);
    Sched* S = P.sched;
    const int pin = S->p_in, ein = S->e_in;
    const int q_in = 2 + ein, q_out = 2 + (ein ^ 1), q_ph = pin;
    const unsigned int n_in = min(S->count[q_in], P.capacity);
    const Tables& T = P.tab;
    const float pcut = P.pcut, ecut = P.ecut;

    unsigned long long n_sub = 0, n_push = 0;
    HeldSink dep;
    Particle p;
    bool active = false, exhausted = false;
    float latent = 0.0f;
    long long base = 0;

    for (unsigned int it = 0;; ++it) {
        if ((it & 255u) == 0u) {
            if (__any_sync(0xffffffffu, (*(volatile int*)&S->flags) & (kFlagOverflow | kFlagStepCap)))
                break;
        }
        if (!active) dep.release(P);  // the finished particle's last held deposit
        if (!active && !exhausted) {
            const unsigned int i = fetch_one(&S->head[q_in]);
            if (i < n_in) {
                load_slot(P, P.q[q_in], i, p);
                latent = p.kind == kPositron ? 2.0f * kElectronMass : 0.0f;
                base = (long long)p.beamlet * P.si.n_voxels;
                active = enter_grid(P, B, p, latent);
            } else {
                exhausted = true;
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted)) break;
        if (!active) continue;

        if (++p.steps > P.max_steps) {
            atomicOr(&S->flags, kFlagStepCap);
            escape(B, p.w * (p.e + latent));
            active = false;
            continue;
        }
        if (p.e <= ecut) {  // terminal: local deposit (electron.py:347-365)
            const int tm = __float_as_int(__ldg(P.vox + flat_index(p.x, p.y, p.z, P.gi)).y);
            deposit(P, B, base, p.x, p.y, p.z, p.w * p.e, spr_factor(P, p.e, tm), dep);
            if (p.kind == kPositron)
                annihilate_at_rest(P, B, p, base, q_ph, spr_factor(P, kElectronMass, tm), dep,
                                   n_push);
            active = false;
            continue;
        }
        ++n_sub;
        const float2 vx = __ldg(P.vox + flat_index(p.x, p.y, p.z, P.gi));
        const float rho = vx.x;
        const int mat = __float_as_int(vx.y);
        const long long row = (long long)mat * T.n_points;

        // --- substep length ---
        const LogIdx le = log_index(p.e, T.e_log_min, T.e_inv_dlog, T.n_points);
        const float4 A = lerp4(T.ea + row, le);  // csda, moller, restricted range, radiative
        const float range_cm = A.x / rho;
        float s_max = P.step_fraction * range_cm;
        if (!P.msc_gs) {
            const float tp = lerp2(T.eb + row, le).x;
            s_max = fminf(s_max, kHingeTheta2Max / (tp * rho));
        }
        const float s_boundary =
            distance_to_voxel_boundary(p.x, p.y, p.z, p.ux, p.uy, p.uz, P.gi) + kBoundaryNudge;
        const float s_geometry = fminf(s_max, s_boundary);
        const float sigma_moller = rho * A.y;
        float s = s_geometry;
        bool moller_pending = false;
        if (sigma_moller > 0.0f) {
            const float s_int = sample_path_length(sigma_moller, p.rng);
            if (s_int <= s_geometry) {
                s = s_int;
                moller_pending = true;
            }
        }
        // --- continuous loss, exact DPM range map ---
        const float available = A.z;
        float de;
        if (rho * s >= available) {
            s = available / rho;
            de = p.e - ecut;
            moller_pending = false;
        } else {
            const LogIdx lr = log_index(available - rho * s, T.r_log_min, T.r_inv_dlog, T.n_points);
            float e_end = lerp1(T.er + row, lr);
            e_end = fminf(fmaxf(e_end, ecut), p.e);
            de = p.e - e_end;
        }
        float emit_p, local_brems;
        brems_step_parameters(p.e, A.w, rho, s, pcut, emit_p, local_brems);
        const float continuous = de + local_brems;
        const bool emit_brems = p.rng.uniform() < emit_p;
        const float factor = spr_factor(P, p.e, mat);

        // --- random hinge: move, deflect, move ---
        const float s1 = p.rng.uniform() * s;
        const float s2 = s - s1;
        float d1 = 0.0f;
        if (s > 0.0f) d1 = continuous * (s1 / s);
        const float d2 = continuous - d1;

        deposit_spread(P, B, base, p.x, p.y, p.z, p.ux, p.uy, p.uz, s1, p.w * d1, factor, dep);
        p.e -= d1;
        p.x += p.ux * s1;
        p.y += p.uy * s1;
        p.z += p.uz * s1;
        if (!point_inside(p.x, p.y, p.z, P.gi)) {
            escape(B, p.w * (p.e + latent));
            active = false;
            continue;
        }
        const LogIdx lh = log_index(p.e, T.e_log_min, T.e_inv_dlog, T.n_points);
        const float2 Bh = lerp2(T.eb + row, lh);  // scattering power, log eta
        const float ms = Bh.x * rho * s;
        float cos_hinge;
        if (P.msc_gs) {
            const float fx = Bh.y * T.gs_bins_per_log;
            const float fy = logf(fmaxf(ms, kGsThetaMin2)) * T.gs_bins_per_log;
            cos_hinge = sample_gs_cos_theta(T, fx, fy, ms, p.rng);
        } else {
            cos_hinge = sample_hinge_cos_theta(ms, p.rng);
        }
        const float phi = kTwoPi * p.rng.uniform();
        rotate_direction(p.ux, p.uy, p.uz, cos_hinge, phi);

        if (emit_brems && p.e > pcut) {
            float k = sample_brems_energy(p.e, pcut, p.rng);
            k = fminf(k, p.e - d2);
            if (k > pcut) {
                float pw = p.w;
                if (k < kRouletteMeV && p.w < kRouletteWeightCap) {
                    pw = roulette_weight(p.w, kRouletteSurvival, p.rng);
                    escape(B, (p.w - pw) * k);
                }
                if (pw > 0.0f) {
                    const StreamId sid = p.rng.spawn();
                    queue_push(P, q_ph, kPhoton, p.beamlet, k, pw, p.x, p.y, p.z, p.ux, p.uy, p.uz,
                               sid, n_push);
                }
            } else {
                deposit_or_escape(P, B, base, p.x, p.y, p.z, p.w * k, spr_factor(P, k, mat), dep);
            }
            p.e -= k;
        }

        deposit_spread(P, B, base, p.x, p.y, p.z, p.ux, p.uy, p.uz, s2, p.w * d2, factor, dep);
        p.e -= d2;
        p.x += p.ux * s2;
        p.y += p.uy * s2;
        p.z += p.uz * s2;
        if (!point_inside(p.x, p.y, p.z, P.gi)) {
            escape(B, p.w * (p.e + latent));
            active = false;
            continue;
        }

        // --- discrete Moller event at the end of the substep ---
        if (moller_pending && p.e > 2.0f * ecut) {
            const float w = sample_moller_delta_energy(p.e, ecut, p.rng);
            float cd, cp;
            moller_direction_cosines(p.e, w, cd, cp);
            const float mphi = kTwoPi * p.rng.uniform();
            float dx = p.ux, dy = p.uy, dz = p.uz;
            rotate_direction(dx, dy, dz, cd, mphi);
            const StreamId sid = p.rng.spawn();
            queue_push(P, q_out, kElectron, p.beamlet, w, p.w, p.x, p.y, p.z, dx, dy, dz, sid,
                       n_push);
            rotate_direction(p.ux, p.uy, p.uz, cp, mphi + kPi);
            p.e -= w;
        }
    }

    dep.release(P);
    block_sum_add(&B.substeps, n_sub);
    block_sum_add(&B.deposits, dep.n);
    block_sum_add(&B.pushes, n_push);
    flush_books(P, B);

    // The last block retires the consumed electron queue, opens the next
    // admission window and publishes whether any work is left.
    if (last_block_arrives(S) && threadIdx.x == 0) {
        S->count[q_in] = 0u;
        S->head[q_in] = 0u;
        S->e_in = ein ^ 1;
        S->rounds += 1;
        S->total_rounds += 1;
        const unsigned long long next_limit = S->cursor + S->budget;
        S->limit = next_limit < S->block_end ? next_limit : S->block_end;
        const bool work = S->cursor < S->block_end || S->count[S->p_in] > 0u ||
                          S->count[2 + (ein ^ 1)] > 0u;
        int remaining = work ? 1 : 0;
        if (S->flags & (kFlagOverflow | kFlagStepCap)) remaining = 0;
        if (remaining && S->rounds >= S->max_rounds) {
            S->flags |= kFlagRoundCap;
            remaining = 0;
        }
        S->remaining = remaining;
        S->blocks_done = 0u;
        __threadfence();
        if (S->cond_handle != 0ull)
            cudaGraphSetConditional((cudaGraphConditionalHandle)S->cond_handle,
                                    (unsigned int)remaining);
    }
}

}  // namespace pmc
