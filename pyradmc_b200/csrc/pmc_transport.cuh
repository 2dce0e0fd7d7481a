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
#include "pmc_reduce.cuh"
#include "pmc_stack.cuh"

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

// One beamlet (or one mixture component of a beamlet) of the record
// generator, 64 bytes:
//   lattice: a = (x_lo, x_extent, y_lo, y_extent), b = (z0, energy, -, -)
//   fan:     a = (focal, width_u), b = (aperture centre, width_v),
//            c = (u axis, first spectrum entry), d = (v axis, -)
// d.w holds the kind (0 lattice, 1 fan) in bit 0 and the fan's spectrum bin
// count above it, as integer bits.  Spectra are concatenated in segments of
// n_bins + 1 entries that start at the same index in the edge and the
// cumulative arrays (the cumulative segment's last entry is unused).
struct __align__(16) BeamletRec {
    float4 a, b, c, d;
};

// Primary generator of the current group (device-resident).
struct GenDesc {
    int type;           // 0 pencil, 1 parallel/lattice, 2 spectral fan, 3 upload, 4 records,
                        // 5 resident phase space
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
    long long n_records;                 // resident phase space: records in up_*
    const BeamletRec* recs;              // records: [group][n_comp]
    const float* comp_cdf;               // records: [n_comp] mixture selection
    int n_comp;
    int masked;                          // spectral fan through a transmission mask
    int mask_n_u, mask_n_v;
    const float* mask;                   // [mask_n_u * mask_n_v]
    float mcx, mcy, mcz;                 // mask plane centre
    float mux, muy, muz, mvx, mvy, mvz;  // mask pixel axes
    float mask_wu, mask_wv;
    int stacked;                         // collimated: weight by the stack transmission
    pmc_head::Stack stack;
    pmc_head::Mu stack_mu;               // macroscopic attenuation, one row per device
};

struct Counters {
    unsigned long long flights, interactions, substeps, deposits, pushes, primaries;
    long long escaped, unscored, deposited, emitted, violations;
};

// Cylindrical scoring bins (geometry/cylinder.py): depth along z by radial
// shell about an axis parallel to z, edges in float32 as the Warp kernels hold
// them, radial edges squared.
struct CylInfo {
    float ax, ay;             // axis
    float z_lo, z_hi;         // first and last depth edge
    float r_in_sq, r_out_sq;  // first and last squared radial edge
    int n_depth, n_shells;
    const float* z_edges;     // [n_depth + 1]
    const float* r_edges_sq;  // [n_shells + 1]
};

struct TransportParams {
    GridInfo gi;          // transport grid
    GridInfo si;          // scoring grid (score_mode 0)
    int score_mode;       // 0 rectilinear, 1 cylindrical
    CylInfo cyl;          // scoring bins (score_mode 1)
    const float2* vox;    // (density, material bits) per transport voxel
    Tables tab;
    Slot* q[4];           // P0, P1, E0, E1
    unsigned int capacity;
    Sched* sched;
    const GenDesc* gen;
    unsigned long long* edep;  // [group][col_stride] int64 quanta
    unsigned int* dirty;       // sector bitmap of edep (pmc_reduce.cuh)
    long long col_stride;      // entries per column: scoring voxels rounded up to a tile
    Counters* counters;
    uint32_t seed_lo, seed_hi;
    float pcut, ecut;
    float step_fraction;
    float deposit_resolution;
    int transport_electrons;
    int msc_gs;
    int dose_to_water;
    int split_n;
    int max_steps;
    int tail_steps;       // steps a lane may still take once its round's input ran dry
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
// Every atomic also marks its entry's sector in the dirty bitmap, the only
// sectors the batch fold visits.
struct DirectSink {
    unsigned int n = 0;  // atomics issued
    __device__ __forceinline__ void add(const TransportParams& P, long long flat,
                                        unsigned long long q) {
        atomicAdd(P.edep + flat, q);
        mark_dirty(P.dirty, flat);
        ++n;
    }
};

struct HeldSink {
    long long idx = -1;
    unsigned long long q = 0;
    unsigned int n = 0;
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
            mark_dirty(P.dirty, idx);
            ++n;
        }
        idx = -1;
        q = 0ull;
    }
};

// edge_bin_index (geometry/cylinder.py): the bin k with edges[k] <= v <
// edges[k + 1], clamped into [0, n - 1]; the caller has checked containment.
__device__ __forceinline__ int edge_bin_index(float v, const float* edges, int n) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (v >= __ldg(edges + mid)) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// kernels.py:492 _scoring_index: the flat scoring bin of a position, or -1
// when the scoring geometry excludes it (half-open on every axis and shell).
__device__ __forceinline__ long long scoring_index(const TransportParams& P, float x, float y,
                                                   float z) {
    if (P.score_mode == 0) return point_inside(x, y, z, P.si) ? flat_index(x, y, z, P.si) : -1;
    const CylInfo& c = P.cyl;
    if (z < c.z_lo || z >= c.z_hi) return -1;
    const float dx = x - c.ax, dy = y - c.ay;
    const float r2 = dx * dx + dy * dy;
    if (r2 < c.r_in_sq || r2 >= c.r_out_sq) return -1;
    const int depth = edge_bin_index(z, c.z_edges, c.n_depth);
    const int shell = edge_bin_index(r2, c.r_edges_sq, c.n_shells);
    return (long long)depth * c.n_shells + shell;
}

// kernels.py:536 _deposit: quantize once, route by position into the scoring
// grid of this particle's column, or into the unscored book.
template <class Sink>
__device__ __forceinline__ void deposit(const TransportParams& P, BlockBooks& B, long long base,
                                       float x, float y, float z, float amount, float factor,
                                       Sink& sink) {
    const long long idx = scoring_index(P, x, y, z);
    if (idx >= 0) {
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
                                           unsigned int& n_push) {
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

// Park an unfinished particle in queue qi for the next round: its whole state
// (phase space, kind, primary flag, beamlet, stream position, steps taken)
// goes into the slot, so the next round continues it exactly where it stopped.
struct Particle;
__device__ __forceinline__ void queue_suspend(const TransportParams& P, int qi, const Particle& p,
                                              unsigned int& n_push);

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
    int steps;  // the host caps max_steps below 2^31
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
    p.steps = (int)d.y;
    p.rng.load(P.seed_lo, P.seed_hi, StreamId{c.x, c.y, c.z, c.w});
}

__device__ __forceinline__ void queue_suspend(const TransportParams& P, int qi, const Particle& p,
                                              unsigned int& n_push) {
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
    const StreamId sid = p.rng.state();
    s->a = make_float4(p.e, p.w, p.x, p.y);
    s->b = make_float4(p.z, p.ux, p.uy, p.uz);
    s->c = make_uint4(sid.id_lo, sid.id_hi, sid.tag, sid.ctr);
    s->d = make_uint4(pack_meta(p.kind, p.primary, p.beamlet), (uint32_t)p.steps, 0u, 0u);
}

// Copy `n` table entries into the block's shared memory (strided over the block).
template <typename T>
__device__ __forceinline__ void stage(T* dst, const T* src, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = __ldg(src + i);
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

// The transmission of a user mask plane along the primary's full line
// (_MaskTransmission.factors, geometry/collimation.py:1041-1080; device twin
// kernels.py:2190-2244): zero for a ray parallel to the plane or crossing it
// outside the rectangle, else the bilinear value between pixel centres,
// clamped in the half-pixel border, in the incremental form that leaves a
// plateau of equal pixels exactly at their value.
__device__ inline float mask_transmission(const GenDesc& G, const Particle& p) {
    const float nx = G.muy * G.mvz - G.muz * G.mvy;
    const float ny = G.muz * G.mvx - G.mux * G.mvz;
    const float nz = G.mux * G.mvy - G.muy * G.mvx;
    const float den = p.ux * nx + p.uy * ny + p.uz * nz;
    if (den == 0.0f) return 0.0f;
    const float t = ((G.mcx - p.x) * nx + (G.mcy - p.y) * ny + (G.mcz - p.z) * nz) / den;
    const float ox = p.x + t * p.ux - G.mcx;
    const float oy = p.y + t * p.uy - G.mcy;
    const float oz = p.z + t * p.uz - G.mcz;
    const float u = ox * G.mux + oy * G.muy + oz * G.muz;
    const float v = ox * G.mvx + oy * G.mvy + oz * G.mvz;
    if (!(fabsf(u) <= 0.5f * G.mask_wu && fabsf(v) <= 0.5f * G.mask_wv)) return 0.0f;
    const int nu = G.mask_n_u, nv = G.mask_n_v;
    float pu = (u + 0.5f * G.mask_wu) / (G.mask_wu / (float)nu) - 0.5f;
    float pv = (v + 0.5f * G.mask_wv) / (G.mask_wv / (float)nv) - 0.5f;
    pu = fmaxf(0.0f, fminf(pu, (float)(nu - 1)));
    pv = fmaxf(0.0f, fminf(pv, (float)(nv - 1)));
    const int i0 = min((int)pu, max(nu - 2, 0));
    const int j0 = min((int)pv, max(nv - 2, 0));
    const int i1 = min(i0 + 1, nu - 1);
    const int j1 = min(j0 + 1, nv - 1);
    const float fu = pu - (float)i0, fv = pv - (float)j0;
    const float v00 = __ldg(G.mask + i0 * nv + j0), v10 = __ldg(G.mask + i1 * nv + j0);
    const float v01 = __ldg(G.mask + i0 * nv + j1), v11 = __ldg(G.mask + i1 * nv + j1);
    return v00 + fu * (v10 - v00) + fv * (v01 - v00) + fu * fv * (v11 - v10 - v01 + v00);
}

// Narrow-beam transmission of a collimated source (_StackTransmission.factors,
// geometry/collimation.py:927-985): exp(-sum_j mu_j(E) t_j), t_j the chord of
// the primary's full line through device j and mu_j that device's macroscopic
// total attenuation on its log-log table.  A ray trapped in a slab has an
// infinite chord and a zero transmission.
__device__ inline float stack_transmission(const GenDesc& G, const Particle& p) {
    const float x[3] = {p.x, p.y, p.z}, u[3] = {p.ux, p.uy, p.uz};
    float lp[3], ld[3];
    pmc_head::to_local(G.stack, x, u, lp, ld);
    float tau = 0.0f;
    for (int j = 0; j < G.stack.n; ++j) {
        const float t = pmc_head::device_len(G.stack, j, lp, ld, 0);
        if (t > 0.0f) tau += pmc_head::mu_at(G.stack_mu, G.stack_mu.log_total, j, p.e) * t;
    }
    return expf(-tau);
}

// ---- primary generation (kernels.py:1888-2401) -------------------------------------
// Maps primary t of the current batch block to its beamlet and history, seeds
// the history's stream, and samples the primary exactly as the host sources do
// (same uniforms, same order).  Returns the particle kind, or -1 when the
// source emits nothing for this history (a masked fan's zero transmission).
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
    } else if (G.type == 4) {  // per-beamlet record (CompositeBeamletSource.emit for mixtures)
        const BeamletRec* r = G.recs + (long long)local * G.n_comp;
        if (G.n_comp > 1) {  // one uniform: the first component whose cdf reaches it
            const float u = p.rng.uniform();
            int lo = 0, hi = G.n_comp;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(G.comp_cdf + mid) < u) lo = mid + 1;
                else hi = mid;
            }
            r += min(lo, G.n_comp - 1);
        }
        const float4 a = __ldg(&r->a), b = __ldg(&r->b);
        const float4 d = __ldg(&r->d);
        const int bits = __float_as_int(d.w);
        p.kind = kPhoton;
        if ((bits & 1) == 0) {  // lattice rectangle: two uniforms
            p.e = b.y;
            p.x = a.x + a.y * p.rng.uniform();
            p.y = a.z + a.w * p.rng.uniform();
            p.z = b.x;
            p.ux = 0.0f; p.uy = 0.0f; p.uz = 1.0f;
        } else {  // divergent fan through the aperture: four uniforms
            const float4 c = __ldg(&r->c);
            const int first = __float_as_int(c.w);
            const int n_bins = bits >> 1;
            const float u_bin = p.rng.uniform();
            const float u_within = p.rng.uniform();
            const float du = (p.rng.uniform() - 0.5f) * a.w;
            const float dv = (p.rng.uniform() - 0.5f) * b.w;
            int lo = 0, hi = n_bins;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(G.cdf + first + mid) < u_bin) lo = mid + 1;
                else hi = mid;
            }
            const int k = first + min(lo, n_bins - 1);
            const float e_lo = __ldg(G.edges + k);
            p.e = e_lo + (__ldg(G.edges + k + 1) - e_lo) * u_within;
            const float dx = b.x + du * c.x + dv * d.x - a.x;
            const float dy = b.y + du * c.y + dv * d.y - a.y;
            const float dz = b.z + du * c.z + dv * d.z - a.z;
            const float inv = 1.0f / sqrtf(dx * dx + dy * dy + dz * dz);
            p.x = a.x; p.y = a.y; p.z = a.z;
            p.ux = dx * inv; p.uy = dy * inv; p.uz = dz * inv;
        }
    } else {  // host-sampled record: the run's history, or the batch block's slot t (Dij);
              // resident phase space: a record drawn by the history's own stream
        long long ri = G.forward ? record : (long long)t;
        if (G.type == 5) {
            const unsigned long long r =
                ((unsigned long long)p.rng.next_u32() << 32) | (unsigned long long)p.rng.next_u32();
            ri = (long long)__umul64hi(r, (unsigned long long)G.n_records);
        }
        p.kind = G.up_kind ? __ldg(G.up_kind + ri) : kPhoton;
        p.e = __ldg(G.up_energy + ri);
        p.w = __ldg(G.up_weight + ri);
        p.x = __ldg(G.up_pos + 3 * ri);
        p.y = __ldg(G.up_pos + 3 * ri + 1);
        p.z = __ldg(G.up_pos + 3 * ri + 2);
        p.ux = __ldg(G.up_dir + 3 * ri);
        p.uy = __ldg(G.up_dir + 3 * ri + 1);
        p.uz = __ldg(G.up_dir + 3 * ri + 2);
    }
    if (G.type != 3 && G.type != 5) {  // host records carry their own weights
        // a zero weight emits nothing; the history still counts in the batch mean
        if (G.masked) p.w *= mask_transmission(G, p);
        if (G.stacked && p.w != 0.0f) p.w *= stack_transmission(G, p);
        if (p.w == 0.0f) return -1;
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
                                          unsigned int& n_push) {
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
// kSmem: the channel rows of every material and the majorant row are staged in
// the block's shared memory (dynamic, n_materials * n_points * 16 + n_points * 4
// bytes) instead of being read through L1.
// kMinBlocks: resident blocks of 256 per SM the register allocation targets
// (3: 80 registers, no spill; 4: 64 registers, a few bytes spilled).
template <bool kSmem, int kMinBlocks = 3>
__global__ void __launch_bounds__(256, kMinBlocks) photon_kernel(TransportParams P) {
    __shared__ BlockBooks B;
    extern __shared__ __align__(16) unsigned char pmc_smem[];
    const float4* tab_ch = P.tab.ch;
    const float* tab_maj = P.tab.maj;
    if constexpr (kSmem) {
        const int n = P.tab.n_materials * P.tab.n_points;
        float4* sch = reinterpret_cast<float4*>(pmc_smem);
        float* smaj = reinterpret_cast<float*>(sch + n);
        stage(sch, P.tab.ch, n);
        stage(smaj, P.tab.maj, P.tab.n_points);
        tab_ch = sch;
        tab_maj = smaj;
    }
    init_books(B);  // its barrier also publishes the staged tables
    Sched* S = P.sched;
    const int pin = S->p_in, ein = S->e_in;
    const int q_in = pin, q_out = pin ^ 1, q_el = 2 + ein;
    const unsigned int n_in = min(S->count[q_in], P.capacity);
    const Tables& T = P.tab;
    const float pcut = P.pcut, ecut = P.ecut;

    unsigned int n_flight = 0, n_inter = 0, n_push = 0;  // per lane and launch
    DirectSink dep;
    Particle p;
    bool active = false, exhausted = false, dry = false;
    int tail = 0;  // steps of the current photon since its warp found the round dry
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
        if (!active && !exhausted) {  // the round's photons: secondaries, parked, then primaries
            const unsigned int i = fetch_one(&S->head[q_in]);
            if (i < n_in) {
                load_slot(P, P.q[q_in], i, p);
                active = enter_grid(P, B, p, 0.0f);
                base = (long long)p.beamlet * P.col_stride;
                e_tab = -1.0f;
                tail = 0;
            } else {
                exhausted = true;
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted)) break;
        if (!dry) dry = __any_sync(0xffffffffu, exhausted);
        if (!active) continue;
        // Once the round's input has run dry, a photon that still needs more than
        // tail_steps flights is parked for the next round instead of holding its
        // warp (and its block's barrier) while every other lane idles.
        if (dry && ++tail > P.tail_steps) {
            queue_suspend(P, q_out, p, n_push);
            active = false;
            continue;
        }

        // ---- one Woodcock flight (photon.py:150-181) ----
        if (++p.steps > P.max_steps) {
            atomicOr(&S->flags, kFlagStepCap);
            escape(B, p.w * p.e);
            active = false;
            continue;
        }
        if (p.e != e_tab) {
            li = log_index(p.e, T.p_log_min, T.p_inv_dlog, T.n_points);
            maj = lerp1<kSmem>(tab_maj, li);
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
            ch = lerp4<kSmem>(tab_ch + (long long)mat * T.n_points, li);
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
    flush_books(P, B);

    // The last block retires the consumed photon queue; the round's admission
    // window has been generated.
    if (last_block_arrives(S) && threadIdx.x == 0) {
        S->count[q_in] = 0u;
        S->head[q_in] = 0u;
        S->p_in = q_out;
        S->cursor = S->limit;
        S->blocks_done = 0u;
        __threadfence();
    }
}

// ---- the primary generator ---------------------------------------------------------
// The round's admission window [cursor, limit) of the batch block, one thread
// per primary (kernels.py:1888-2401): sampled at full warp width, flown
// through vacuum to the grid, then queued with its stream position — photons
// into the round's photon input queue behind the secondaries already there,
// charged primaries into its electron queue.  The photon kernel then loads
// every particle the same way, and no lane of it idles behind another's
// primary sampling.
__global__ void __launch_bounds__(256) generate_kernel(TransportParams P) {
    __shared__ BlockBooks B;
    init_books(B);
    Sched* S = P.sched;
    const unsigned long long cursor = S->cursor, limit = S->limit;
    const int q_ph = S->p_in, q_el = 2 + S->e_in;
    const int batch = S->batch;
    const GenDesc& G = *P.gen;
    unsigned int n_push = 0, n_prim = 0;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long t = cursor + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
         t < limit; t += stride) {
        Particle p;
        ++n_prim;
        const int kind = generate_primary(P, G, batch, t, p, B);
        if (kind < 0) continue;
        if (kind == kPhoton) {
            if (enter_grid(P, B, p, 0.0f)) queue_suspend(P, q_ph, p, n_push);
        } else {  // charged primary: to the electron queue unchanged (it enters there)
            queue_push(P, q_el, kind, p.beamlet, p.e, p.w, p.x, p.y, p.z, p.ux, p.uy, p.uz,
                       p.rng.state(), n_push);
        }
    }
    block_sum_add(&B.pushes, n_push);
    block_sum_add(&B.primaries, n_prim);
    flush_books(P, B);
}

__device__ __forceinline__ long long col_base(const TransportParams& P, const Particle& p) {
    return (long long)p.beamlet * P.col_stride;
}

// Annihilation energy a positron still carries (2 m c^2), booked with it on escape.
__device__ __forceinline__ float rest_energy(const Particle& p) {
    return p.kind == kPositron ? 2.0f * kElectronMass : 0.0f;
}

// ---- the electron kernel -------------------------------------------------------------
// One lane runs one electron or positron to ECUT (Class II condensed history,
// electron.py:345-481); delta rays go to the next round's electron queue,
// bremsstrahlung and annihilation photons to the next photon round.
// kSmem: the (csda range, moller, restricted range, radiative stopping) and
// (scattering power, log eta) rows of every material are staged in the block's
// shared memory (n_materials * n_points * 24 bytes); the inverse-range row
// (one read per substep) stays on the L1 path.
// kMinBlocks: as for the photon kernel (4: 64 registers, a few bytes spilled;
// 3: 85 registers, none).
template <bool kSmem, int kMinBlocks = 4>
__global__ void __launch_bounds__(256, kMinBlocks) electron_kernel(TransportParams P) {
    __shared__ BlockBooks B;
    extern __shared__ __align__(16) unsigned char pmc_smem[];
    const float4* tab_ea = P.tab.ea;
    const float2* tab_eb = P.tab.eb;
    if constexpr (kSmem) {
        const int n = P.tab.n_materials * P.tab.n_points;
        float4* sea = reinterpret_cast<float4*>(pmc_smem);
        float2* seb = reinterpret_cast<float2*>(sea + n);
        stage(sea, P.tab.ea, n);
        stage(seb, P.tab.eb, n);
        tab_ea = sea;
        tab_eb = seb;
    }
    init_books(B);  // its barrier also publishes the staged tables
    Sched* S = P.sched;
    const int pin = S->p_in, ein = S->e_in;
    const int q_in = 2 + ein, q_out = 2 + (ein ^ 1), q_ph = pin;
    const unsigned int n_in = min(S->count[q_in], P.capacity);
    const Tables& T = P.tab;
    const float pcut = P.pcut, ecut = P.ecut;

    unsigned int n_sub = 0, n_push = 0;  // per lane and launch
    HeldSink dep;
    // The particle's column offset (col_base) is recomputed at each deposit
    // instead of being held in two registers for the particle's whole life.
    Particle p;
    bool active = false, exhausted = false, dry = false;
    int tail = 0;  // substeps of the current particle since its warp found the round dry

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
                active = enter_grid(P, B, p, rest_energy(p));
                tail = 0;
            } else {
                exhausted = true;
            }
        }
        if (!__any_sync(0xffffffffu, active || !exhausted)) break;
        if (!dry) dry = __any_sync(0xffffffffu, exhausted);
        if (!active) continue;
        // Park a particle that outlives the round's input by tail_steps substeps
        // (its held deposit is released at the top of the next iteration).
        if (dry && ++tail > P.tail_steps) {
            queue_suspend(P, q_out, p, n_push);
            active = false;
            continue;
        }

        if (++p.steps > P.max_steps) {
            atomicOr(&S->flags, kFlagStepCap);
            escape(B, p.w * (p.e + rest_energy(p)));
            active = false;
            continue;
        }
        if (p.e <= ecut) {  // terminal: local deposit (electron.py:347-365)
            const int tm = __float_as_int(__ldg(P.vox + flat_index(p.x, p.y, p.z, P.gi)).y);
            deposit(P, B, col_base(P, p), p.x, p.y, p.z, p.w * p.e, spr_factor(P, p.e, tm), dep);
            if (p.kind == kPositron)
                annihilate_at_rest(P, B, p, col_base(P, p), q_ph, spr_factor(P, kElectronMass, tm), dep,
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
        const float4 A = lerp4<kSmem>(tab_ea + row, le);  // csda, moller, restricted range, radiative
        const float range_cm = A.x / rho;
        float s_max = P.step_fraction * range_cm;
        if (!P.msc_gs) {
            const float tp = lerp2<kSmem>(tab_eb + row, le).x;
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

        deposit_spread(P, B, col_base(P, p), p.x, p.y, p.z, p.ux, p.uy, p.uz, s1, p.w * d1, factor, dep);
        p.e -= d1;
        p.x += p.ux * s1;
        p.y += p.uy * s1;
        p.z += p.uz * s1;
        if (!point_inside(p.x, p.y, p.z, P.gi)) {
            escape(B, p.w * (p.e + rest_energy(p)));
            active = false;
            continue;
        }
        const LogIdx lh = log_index(p.e, T.e_log_min, T.e_inv_dlog, T.n_points);
        const float2 Bh = lerp2<kSmem>(tab_eb + row, lh);  // scattering power, log eta
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
                deposit_or_escape(P, B, col_base(P, p), p.x, p.y, p.z, p.w * k, spr_factor(P, k, mat), dep);
            }
            p.e -= k;
        }

        deposit_spread(P, B, col_base(P, p), p.x, p.y, p.z, p.ux, p.uy, p.uz, s2, p.w * d2, factor, dep);
        p.e -= d2;
        p.x += p.ux * s2;
        p.y += p.uy * s2;
        p.z += p.uz * s2;
        if (!point_inside(p.x, p.y, p.z, P.gi)) {
            escape(B, p.w * (p.e + rest_energy(p)));
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
