// pmc_presolve.cu — the treatment-head pre-solve on the GPU (C-ABI in
// include/pyradmc_b200_presolve.h).
//
// One thread per primary traces it through the beam-limiting stack and the
// air column (geometry/head.py:373-575 is the algorithm; the chord lengths
// restate the scalar twins of geometry/collimation.py:253-490) and writes its
// exit-plane particles into fixed slots (transmitted, stack scatter, air
// photon, air electron), so the output order is the primaries' order whatever
// the scheduling; a block count, a host prefix sum and a block-local rank then
// compact the kept slots.  Random numbers: the Philox stream of (seed,
// primary index) under a tag of its own.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/pyradmc_b200.h"
#include "../../include/pyradmc_b200_presolve.h"
#include "pmc_common.cuh"
#include "pmc_physics.cuh"
#include "pmc_stack.cuh"

namespace pmc_head {

using pmc::Rng;

constexpr int kThreads = 256;
constexpr uint32_t kHeadTag = 0x48454144u;  // stream tag of the pre-solve ("HEAD")

struct Params {
    int first_compton, has_air, air_row;
    float air_z0, air_z1, exit_z, pcut, ecut, floor;
    uint32_t seed_lo, seed_hi;
};

// One exit-plane slot; kind 0 = empty.
struct Out {
    int* kind;
    float* energy;
    float* pos;
    float* dir;
    float* weight;
};

// head.py:319-337: a secondary below the floor survives with probability
// w / floor at weight floor.
__device__ __forceinline__ float roulette(float w, float floor, Rng& rng) {
    if (floor <= 0.0f || w <= 0.0f || w >= floor) return w;
    return rng.uniform() < w / floor ? floor : 0.0f;
}

// A kept particle slides straight to the exit plane into its slot; a dropped
// one adds its weight x energy to `dropped` (head.py:576-599).
__device__ __forceinline__ void emit(const Stack& S, const Params& P, const Out& o, long long slot, int kind,
                                     float e, const float* x, const float* u, float w, float cutoff,
                                     double& dropped) {
    bool kept = false;
    if (w > 0.0f && e >= cutoff) {
        const float d_w = S.rot[6] * u[0] + S.rot[7] * u[1] + S.rot[8] * u[2];
        if (d_w > 0.0f) {
            const float p_w = S.rot[6] * (x[0] - S.origin[0]) + S.rot[7] * (x[1] - S.origin[1]) +
                              S.rot[8] * (x[2] - S.origin[2]);
            const float t = (P.exit_z - p_w) / d_w;
            if (t >= 0.0f) {
                kept = true;
                o.kind[slot] = kind;
                o.energy[slot] = e;
                o.weight[slot] = w;
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    o.pos[3 * slot + k] = x[k] + t * u[k];
                    o.dir[3 * slot + k] = u[k];
                }
            }
        }
    }
    if (!kept) dropped += (double)w * (double)e;
}

__global__ void __launch_bounds__(kThreads) presolve_kernel(Stack S, Mu M, Params P, long long n,
                                                          const float* __restrict__ energy,
                                                          const float* __restrict__ pos,
                                                          const float* __restrict__ dir,
                                                          const float* __restrict__ weight, Out o,
                                                          int per_primary, double* __restrict__ block_dropped) {
    __shared__ double red[kThreads / 32];
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double dropped = 0.0;
    if (i < n) {
        const float e = energy[i], w = weight[i];
        const float x[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
        const float u[3] = {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]};
        float pl[3], dl[3];
        to_local(S, x, u, pl, dl);
        Rng rng;
        rng.load(P.seed_lo, P.seed_hi, pmc::StreamId{(uint32_t)i, (uint32_t)(i >> 32), kHeadTag, 0u});
        long long slot = i * per_primary;
        const long long s_trans = slot++;

        // ---- the stack (head.py:424-484) ----
        float tau[kMaxDevices];
        float tau_total = 0.0f;
        for (int j = 0; j < S.n; ++j) {
            tau[j] = mu_at(M, M.log_total, j, e) * device_len(S, j, pl, dl, 0);
            tau_total += tau[j];
        }
        float trans_w = w * expf(-tau_total);
        if (P.first_compton) {
            const long long s_scat = slot++;
            if (tau_total > 0.0f) {
                // the device by its share of the optical depth; the site at its
                // mid-plane crossing (the stated approximation of head.py:37-41)
                const float pick = rng.uniform() * tau_total;
                int jd = S.n - 1;
                float acc = 0.0f;
                for (int j = 0; j < S.n; ++j) {
                    acc += tau[j];
                    if (pick <= acc) {
                        jd = j;
                        break;
                    }
                }
                const float z_mid = 0.5f * (S.z_top[jd] + S.z_bottom[jd]);
                const float t_mid = (z_mid - pl[2]) / dl[2];
                const float site[3] = {x[0] + t_mid * u[0], x[1] + t_mid * u[1], x[2] + t_mid * u[2]};
                const float cf = mu_at(M, M.log_compton, jd, e) / mu_at(M, M.log_total, jd, e);
                const float iw = w * (1.0f - expf(-tau_total));
                const float ratio = pmc::sample_compton_energy_ratio(e, rng);
                const float e_out = ratio * e;
                const float phi = pmc::kTwoPi * rng.uniform();
                float d_out[3] = {u[0], u[1], u[2]};
                pmc::rotate_direction(d_out[0], d_out[1], d_out[2], pmc::compton_cos_theta(e, ratio), phi);
                float sl[3], sd[3];
                to_local(S, site, d_out, sl, sd);
                float tau_out = 0.0f;
                for (int j = 0; j < S.n; ++j)
                    tau_out += mu_at(M, M.log_total, j, e_out) * device_len(S, j, sl, sd, 1);
                const float sw = roulette(iw * cf * expf(-tau_out), P.floor, rng);
                emit(S, P, o, s_scat, 1, e_out, site, d_out, sw, P.pcut, dropped);
            }
        }

        // ---- the air column, primaries only (head.py:487-553) ----
        if (P.has_air) {
            const bool forward = dl[2] > 0.0f;
            const float length = forward ? (P.air_z1 - P.air_z0) / dl[2] : 0.0f;
            const float mu_air = mu_at(M, M.log_total, P.air_row, e);
            const float tau_air = mu_air * length;
            const float pre = trans_w;
            trans_w *= expf(-tau_air);
            if (P.first_compton) {
                const long long s_ph = slot++, s_el = slot++;
                if (forward && tau_air > 0.0f) {
                    const float iw = pre * (1.0f - expf(-tau_air));
                    const float pw = iw * (mu_at(M, M.log_compton, P.air_row, e) / mu_air);
                    const float ud = rng.uniform();
                    const float depth = -logf(1.0f - ud * (1.0f - expf(-tau_air))) / mu_air;
                    const float t0 = (P.air_z0 - pl[2]) / dl[2] + depth;
                    const float site[3] = {x[0] + t0 * u[0], x[1] + t0 * u[1], x[2] + t0 * u[2]};
                    const float ratio = pmc::sample_compton_energy_ratio(e, rng);
                    const float e_ph = ratio * e, e_el = e - e_ph;
                    const float phi = pmc::kTwoPi * rng.uniform();
                    float d_ph[3] = {u[0], u[1], u[2]}, d_el[3] = {u[0], u[1], u[2]};
                    pmc::rotate_direction(d_ph[0], d_ph[1], d_ph[2], pmc::compton_cos_theta(e, ratio), phi);
                    pmc::rotate_direction(d_el[0], d_el[1], d_el[2], pmc::compton_electron_cos_theta(e, ratio),
                                          phi + pmc::kPi);
                    // the two arms are rouletted independently (head.py:528-531)
                    const float w_ph = roulette(pw, P.floor, rng);
                    const float w_el = roulette(pw, P.floor, rng);
                    emit(S, P, o, s_ph, 1, e_ph, site, d_ph, w_ph, P.pcut, dropped);
                    emit(S, P, o, s_el, 2, e_el, site, d_el, w_el, P.ecut, dropped);
                }
            }
        }
        emit(S, P, o, s_trans, 1, e, x, u, trans_w, P.pcut, dropped);
    }
    // per-block dropped weight-energy (summed on the host in block order)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dropped += __shfl_xor_sync(0xffffffffu, dropped, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = dropped;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) s += red[k];
        block_dropped[blockIdx.x] = s;
    }
}

// Kept slots per block of kThreads consecutive slots.
__global__ void __launch_bounds__(kThreads) count_slots(const int* __restrict__ kind, long long n_slots,
                                                       int* __restrict__ block_counts) {
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int keep = s < n_slots && kind[s] != 0;
    const int c = __syncthreads_count(keep);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = c;
}

// Kept slot s goes to block_offsets[block] + its rank in the block.
__global__ void __launch_bounds__(kThreads) compact_slots(Out in, long long n_slots,
                                                         const long long* __restrict__ block_offsets,
                                                         Out out) {
    __shared__ int warp_base[kThreads / 32];
    const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int keep = s < n_slots && in.kind[s] != 0;
    const unsigned int ballot = __ballot_sync(0xffffffffu, keep);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) warp_base[warp] = __popc(ballot);
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < kThreads / 32; ++k) {
            const int c = warp_base[k];
            warp_base[k] = acc;
            acc += c;
        }
    }
    __syncthreads();
    if (keep) {
        const long long dst = block_offsets[blockIdx.x] + warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
        out.kind[dst] = in.kind[s];
        out.energy[dst] = in.energy[s];
        out.weight[dst] = in.weight[s];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            out.pos[3 * dst + k] = in.pos[3 * s + k];
            out.dir[3 * dst + k] = in.dir[3 * s + k];
        }
    }
}

__global__ void __launch_bounds__(kThreads) path_lengths_kernel(Stack S, long long n, const float* __restrict__ pos,
                                                               const float* __restrict__ dir, int from_origin,
                                                               float* __restrict__ out) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float pl[3], dl[3];
    to_local(S, pos + 3 * i, dir + 3 * i, pl, dl);
    for (int j = 0; j < S.n; ++j) out[i * S.n + j] = device_len(S, j, pl, dl, from_origin);
}

}  // namespace pmc_head

// ---- host side -------------------------------------------------------------------
namespace {

using namespace pmc_head;

// Device buffers of one call, freed on every exit path.
struct Arena {
    std::vector<void*> ptrs;
    ~Arena() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        if (cudaMalloc(&p, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
    template <typename T>
    T* upload(const T* src, size_t n) {
        T* d = alloc<T>(n);
        if (d && n && cudaMemcpy(d, src, sizeof(T) * n, cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
        return d;
    }
    float* upload_f32(const double* src, size_t n) {  // float64 host array -> float32 device array
        std::vector<float> f(n);
        for (size_t i = 0; i < n; ++i) f[i] = (float)src[i];
        return upload(f.data(), n);
    }
};

bool stack_ok(const pmc_head_stack* s) {
    if (!s || s->n_devices < 1 || s->n_devices > kMaxDevices || !s->kind || !s->z_top || !s->z_bottom ||
        !s->jaw_axis || !s->jaw_edge_neg || !s->jaw_edge_pos || !s->jaw_focused || !s->mlc_tip_radius ||
        !s->mlc_focused_sides || !s->mlc_n_pairs || !s->mlc_edges_off || !s->mlc_tips_off)
        return false;
    for (int j = 0; j < s->n_devices; ++j) {
        if (s->kind[j] != 0 && s->kind[j] != 1) return false;
        if (!(s->z_bottom[j] > s->z_top[j])) return false;
        if (s->kind[j] == 0 && s->jaw_axis[j] != 0 && s->jaw_axis[j] != 1) return false;
        if (s->kind[j] == 1) {
            const long long n = s->mlc_n_pairs[j];
            if (n < 0 || s->mlc_edges_off[j] < 0 || s->mlc_tips_off[j] < 0 ||
                s->mlc_edges_off[j] + n + (n > 0 ? 1 : 0) > s->n_leaf_edges ||
                s->mlc_tips_off[j] + n > s->n_tips)
                return false;
            if (n > 0 && (!s->leaf_edges_v || !s->tips_neg || !s->tips_pos)) return false;
        }
    }
    return true;
}

int upload_stack(Arena& a, const pmc_head_stack* s, Stack& S) {
    S.n = s->n_devices;
    for (int k = 0; k < 3; ++k) S.origin[k] = (float)s->origin[k];
    for (int k = 0; k < 9; ++k) S.rot[k] = (float)s->rotation[k];
    const size_t n = (size_t)s->n_devices;
    S.kind = a.upload(s->kind, n);
    S.z_top = a.upload_f32(s->z_top, n);
    S.z_bottom = a.upload_f32(s->z_bottom, n);
    S.jaw_axis = a.upload(s->jaw_axis, n);
    S.jaw_neg = a.upload_f32(s->jaw_edge_neg, n);
    S.jaw_pos = a.upload_f32(s->jaw_edge_pos, n);
    S.jaw_focused = a.upload(s->jaw_focused, n);
    S.tip_radius = a.upload_f32(s->mlc_tip_radius, n);
    S.focused_sides = a.upload(s->mlc_focused_sides, n);
    S.n_pairs = a.upload(s->mlc_n_pairs, n);
    S.edges_off = a.upload(s->mlc_edges_off, n);
    S.tips_off = a.upload(s->mlc_tips_off, n);
    const size_t ne = (size_t)(s->n_leaf_edges > 0 ? s->n_leaf_edges : 0);
    const size_t nt = (size_t)(s->n_tips > 0 ? s->n_tips : 0);
    S.leaf_edges = ne ? a.upload_f32(s->leaf_edges_v, ne) : a.alloc<float>(1);
    S.tips_neg = nt ? a.upload_f32(s->tips_neg, nt) : a.alloc<float>(1);
    S.tips_pos = nt ? a.upload_f32(s->tips_pos, nt) : a.alloc<float>(1);
    const bool ok = S.kind && S.z_top && S.z_bottom && S.jaw_axis && S.jaw_neg && S.jaw_pos && S.jaw_focused &&
                    S.tip_radius && S.focused_sides && S.n_pairs && S.edges_off && S.tips_off && S.leaf_edges &&
                    S.tips_neg && S.tips_pos;
    return ok ? PMC_OK : PMC_ERR_CUDA;
}

int blocks_for(long long n) { return (int)((n + kThreads - 1) / kThreads); }

}  // namespace

extern "C" int pmc_head_path_lengths(const pmc_head_stack* stack, int64_t n, const float* pos, const float* dir,
                                     int32_t from_origin, float* out) {
    if (!stack_ok(stack) || n < 0 || (n > 0 && (!pos || !dir || !out))) return PMC_ERR_INVALID;
    if (n == 0) return PMC_OK;
    Arena a;
    Stack S{};
    if (upload_stack(a, stack, S) != PMC_OK) return PMC_ERR_CUDA;
    const float* dp = a.upload(pos, (size_t)n * 3);
    const float* dd = a.upload(dir, (size_t)n * 3);
    float* dout = a.alloc<float>((size_t)n * stack->n_devices);
    if (!dp || !dd || !dout) return PMC_ERR_CUDA;
    path_lengths_kernel<<<blocks_for(n), kThreads>>>(S, n, dp, dd, from_origin ? 1 : 0, dout);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return PMC_ERR_CUDA;
    if (cudaMemcpy(out, dout, sizeof(float) * (size_t)n * stack->n_devices, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PMC_ERR_CUDA;
    return PMC_OK;
}

extern "C" int pmc_presolve_head(const pmc_head_stack* stack, const pmc_head_mu* mu, const pmc_head_params* params,
                                 int64_t n, const float* energy, const float* pos, const float* dir,
                                 const float* weight, int64_t capacity, int32_t* out_kind, float* out_energy,
                                 float* out_pos, float* out_dir, float* out_weight, int64_t* count,
                                 double* dropped) {
    if (!stack_ok(stack) || !mu || !params || !count || n < 1 || !energy || !pos || !dir || !weight ||
        capacity < 0)
        return PMC_ERR_INVALID;
    const int rows = stack->n_devices + (params->has_air ? 1 : 0);
    if (mu->n_table < 2 || mu->n_rows < rows || !mu->log_energy || !mu->log_total || !mu->log_compton)
        return PMC_ERR_INVALID;
    if (params->has_air && (params->air_row < 0 || params->air_row >= mu->n_rows)) return PMC_ERR_INVALID;
    const double span = mu->log_energy[mu->n_table - 1] - mu->log_energy[0];
    if (!(span > 0.0)) return PMC_ERR_INVALID;
    const int fc = params->first_compton ? 1 : 0, air = params->has_air ? 1 : 0;
    const int per_primary = 1 + fc * (1 + 2 * air);
    const long long n_slots = (long long)n * per_primary;

    Arena a;
    Stack S{};
    if (upload_stack(a, stack, S) != PMC_OK) return PMC_ERR_CUDA;
    Mu M{};
    M.n_rows = mu->n_rows;
    M.n_table = mu->n_table;
    M.log_e0 = (float)mu->log_energy[0];
    M.inv_dlog = (float)((mu->n_table - 1) / span);
    M.log_total = a.upload_f32(mu->log_total, (size_t)mu->n_rows * mu->n_table);
    M.log_compton = a.upload_f32(mu->log_compton, (size_t)mu->n_rows * mu->n_table);
    Params P{};
    P.first_compton = fc;
    P.has_air = air;
    P.air_row = params->air_row;
    P.air_z0 = (float)params->air_z_start;
    P.air_z1 = (float)params->air_z_end;
    P.exit_z = (float)params->exit_z;
    P.pcut = (float)params->pcut;
    P.ecut = (float)params->ecut;
    P.floor = (float)params->weight_floor;
    P.seed_lo = (uint32_t)(params->seed & 0xffffffffull);
    P.seed_hi = (uint32_t)(params->seed >> 32);
    const float* d_e = a.upload(energy, (size_t)n);
    const float* d_p = a.upload(pos, (size_t)n * 3);
    const float* d_d = a.upload(dir, (size_t)n * 3);
    const float* d_w = a.upload(weight, (size_t)n);
    Out slots{a.alloc<int>(n_slots), a.alloc<float>(n_slots), a.alloc<float>(3 * n_slots),
              a.alloc<float>(3 * n_slots), a.alloc<float>(n_slots)};
    const int nb = blocks_for(n), sb = blocks_for(n_slots);
    double* d_drop = a.alloc<double>(nb);
    int* d_counts = a.alloc<int>(sb);
    long long* d_offsets = a.alloc<long long>(sb);
    if (!M.log_total || !M.log_compton || !d_e || !d_p || !d_d || !d_w || !slots.kind || !slots.energy ||
        !slots.pos || !slots.dir || !slots.weight || !d_drop || !d_counts || !d_offsets)
        return PMC_ERR_CUDA;
    if (cudaMemset(slots.kind, 0, sizeof(int) * (size_t)n_slots) != cudaSuccess) return PMC_ERR_CUDA;
    presolve_kernel<<<nb, kThreads>>>(S, M, P, n, d_e, d_p, d_d, d_w, slots, per_primary, d_drop);
    count_slots<<<sb, kThreads>>>(slots.kind, n_slots, d_counts);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return PMC_ERR_CUDA;

    // dropped weight-energy and the kept count, summed in block order
    std::vector<double> drop(nb);
    std::vector<int> counts(sb);
    std::vector<long long> offsets(sb);
    if (cudaMemcpy(drop.data(), d_drop, sizeof(double) * nb, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(counts.data(), d_counts, sizeof(int) * sb, cudaMemcpyDeviceToHost) != cudaSuccess)
        return PMC_ERR_CUDA;
    double dsum = 0.0;
    for (double v : drop) dsum += v;
    if (dropped) *dropped = dsum;
    long long total = 0;
    for (int b = 0; b < sb; ++b) {
        offsets[b] = total;
        total += counts[b];
    }
    *count = total;
    if (total > capacity) return PMC_ERR_CAPACITY;
    if (total == 0) return PMC_OK;
    if (!out_kind || !out_energy || !out_pos || !out_dir || !out_weight) return PMC_ERR_INVALID;
    if (cudaMemcpy(d_offsets, offsets.data(), sizeof(long long) * sb, cudaMemcpyHostToDevice) != cudaSuccess)
        return PMC_ERR_CUDA;
    if (params->outputs_on_device) {  // straight into the caller's device arrays
        Out dst{out_kind, out_energy, out_pos, out_dir, out_weight};
        compact_slots<<<sb, kThreads>>>(slots, n_slots, d_offsets, dst);
        return cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess ? PMC_OK : PMC_ERR_CUDA;
    }
    Out packed{a.alloc<int>(total), a.alloc<float>(total), a.alloc<float>(3 * total), a.alloc<float>(3 * total),
               a.alloc<float>(total)};
    if (!packed.kind || !packed.energy || !packed.pos || !packed.dir || !packed.weight) return PMC_ERR_CUDA;
    compact_slots<<<sb, kThreads>>>(slots, n_slots, d_offsets, packed);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return PMC_ERR_CUDA;
    const bool ok = cudaMemcpy(out_kind, packed.kind, sizeof(int) * total, cudaMemcpyDeviceToHost) == cudaSuccess &&
                    cudaMemcpy(out_energy, packed.energy, sizeof(float) * total, cudaMemcpyDeviceToHost) == cudaSuccess &&
                    cudaMemcpy(out_pos, packed.pos, sizeof(float) * 3 * total, cudaMemcpyDeviceToHost) == cudaSuccess &&
                    cudaMemcpy(out_dir, packed.dir, sizeof(float) * 3 * total, cudaMemcpyDeviceToHost) == cudaSuccess &&
                    cudaMemcpy(out_weight, packed.weight, sizeof(float) * total, cudaMemcpyDeviceToHost) == cudaSuccess;
    return ok ? PMC_OK : PMC_ERR_CUDA;
}
