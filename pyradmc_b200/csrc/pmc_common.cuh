// pmc_common.cuh — shared device types, constants, the Philox RNG and the
// scalar geometry/table helpers of the B200 transport.
//
// The physics is float32, like the Warp kernels it replaces
// (pyradmc/backends/warp/kernels.py module docstring); scoring is int64
// fixed-point and every reduction is float64 with an explicit operation order.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pmc {

// ---- constants (pyradmc/__init__.py:22-112, kernels.py:96-116) -------------
constexpr float kElectronMass = 0.51099895069f;       // ELECTRON_MASS_MEV
constexpr float kRouletteMeV = 0.5f;                   // PHOTON_ROULETTE_MEV
constexpr float kRouletteSurvival = 0.5f;              // PHOTON_ROULETTE_SURVIVAL
constexpr float kRouletteWeightCap = 4.0f;             // PHOTON_ROULETTE_WEIGHT_CAP
constexpr double kQuantum = 1.0e-9;                    // ENERGY_QUANTUM_MEV
constexpr double kInvQuantum = 1.0e9;
constexpr float kEntryNudge = 1.0e-4f;                 // float32 entry nudge (kernels.py:101)
constexpr float kBoundaryNudge = 1.0e-4f;              // BOUNDARY_NUDGE_CM (transport/electron.py:151)
constexpr float kInfinityCm = 1.0e30f;                 // _INFINITY_CM (kernels.py:106)
constexpr float kHingeTheta2Max = 0.10f;               // STEP_HINGE_THETA2_MAX
constexpr float kGsThetaMin2 = 1.0e-12f;               // _GS_THETA2_MIN (data/interface.py:62)
constexpr float kPoleFloor = 1.0e-20f;                 // physics/direction.py:20
constexpr float kTwoPi = 6.283185307179586f;
constexpr float kPi = 3.141592653589793f;
constexpr float kRayleighPerMeV = 80.65543f;           // RAYLEIGH_MOMENTUM_TRANSFER_PER_MEV
constexpr int kWater = 0;                              // data/materials.py:148

constexpr int kPhoton = 0;
constexpr int kElectron = 1;
constexpr int kPositron = 2;

// ---- Philox4x32-10 counter-based generator ----------------------------------
// Salmon, Moraes, Dror & Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11, doi:10.1145/2063384.2063405.  The multipliers and Weyl increments are
// the published Philox4x32 constants.  A particle's stream is the Philox key
// (the run seed) applied to the counter (block, id_lo, id_hi, tag): primaries
// use tag 0 and id = their history key, so a stream is a pure function of
// (seed, history key) — the reproducibility contract of rng/interface.py.
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

__host__ __device__ inline void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += kPhiloxW0;
            k1 += kPhiloxW1;
        }
#ifdef __CUDA_ARCH__
        const uint32_t lo0 = kPhiloxM0 * c[0];
        const uint32_t hi0 = __umulhi(kPhiloxM0, c[0]);
        const uint32_t lo1 = kPhiloxM1 * c[2];
        const uint32_t hi1 = __umulhi(kPhiloxM1, c[2]);
#else
        const uint64_t p0 = (uint64_t)kPhiloxM0 * c[0];
        const uint64_t p1 = (uint64_t)kPhiloxM1 * c[2];
        const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
        const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        const uint32_t n0 = hi1 ^ c[1] ^ k0;
        const uint32_t n2 = hi0 ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = lo1;
        c[2] = n2;
        c[3] = lo0;
    }
}

// Stream identity carried by a queued particle (16 bytes).
struct StreamId {
    uint32_t id_lo, id_hi, tag, ctr;
};

struct Rng {
    uint32_t k0, k1;          // run seed
    uint32_t id_lo, id_hi, tag;
    uint32_t ctr;             // uniforms consumed
    uint32_t b0, b1, b2, b3;  // current Philox block (valid when ctr % 4 != 0)

    __device__ inline void load(uint32_t seed_lo, uint32_t seed_hi, const StreamId& s) {
        k0 = seed_lo;
        k1 = seed_hi;
        id_lo = s.id_lo;
        id_hi = s.id_hi;
        tag = s.tag;
        ctr = s.ctr;
        if ((ctr & 3u) != 0u) refill();
    }
    __device__ inline void refill() {
        uint32_t c[4] = {ctr >> 2, id_lo, id_hi, tag};
        philox4x32_10(c, k0, k1);
        b0 = c[0];
        b1 = c[1];
        b2 = c[2];
        b3 = c[3];
    }
    // Registers only: the word is selected, never indexed (an indexed array
    // would live in local memory).
    __device__ inline uint32_t next_u32() {
        const uint32_t slot = ctr & 3u;
        if (slot == 0u) refill();
        const uint32_t r = slot == 0u ? b0 : slot == 1u ? b1 : slot == 2u ? b2 : b3;
        ++ctr;
        return r;
    }
    // U[0, 1) with 24-bit resolution: cannot return 1.0 (rng/interface.py:55-61).
    __device__ inline float uniform() { return (float)(next_u32() >> 8) * (1.0f / 16777216.0f); }
    // Child stream for a queued secondary: three parent draws name it, so it is a
    // deterministic function of the parent's stream and draw position, whatever
    // thread or queue slot carries either particle (rng/warp_shim.py:67-78).
    __device__ inline StreamId spawn() {
        StreamId c;
        c.id_lo = next_u32();
        c.id_hi = next_u32();
        c.tag = next_u32() | 1u;
        c.ctr = 0u;
        return c;
    }
    __device__ inline StreamId state() const { return StreamId{id_lo, id_hi, tag, ctr}; }
};

// ---- queue slot: one particle, 64 bytes (four 16-byte vectors) --------------
// meta = kind (bits 0-1) | primary (bit 2) | beamlet << 3; d.y carries the
// steps a suspended particle has already taken (0 for a new one).
struct __align__(16) Slot {
    float4 a;  // energy, weight, x, y
    float4 b;  // z, ux, uy, uz
    uint4 c;   // stream id_lo, id_hi, tag, ctr
    uint4 d;   // meta, steps taken, spare
};

__device__ inline uint32_t pack_meta(int kind, int primary, int beamlet) {
    return (uint32_t)kind | ((uint32_t)primary << 2) | ((uint32_t)beamlet << 3);
}

// ---- grids (geometry/grid.py) -------------------------------------------------
struct GridInfo {
    float x_lo, y_lo, z_lo;
    float x_hi, y_hi, z_hi;
    float sx, sy, sz;
    int nx, ny, nz;
    long long n_voxels;
};

// point_inside (geometry/grid.py:35): half-open box containment.
__device__ __forceinline__ bool point_inside(float x, float y, float z, const GridInfo& g) {
    if (x < g.x_lo || x >= g.x_hi) return false;
    if (y < g.y_lo || y >= g.y_hi) return false;
    return !(z < g.z_lo || z >= g.z_hi);
}

// point_axis_index (geometry/grid.py:58): floor, clamped into [0, n-1].
__device__ __forceinline__ int axis_index(float p, float o, float s, int n) {
    int i = (int)floorf((p - o) / s);
    if (i < 0) return 0;
    if (i >= n) return n - 1;
    return i;
}

__device__ __forceinline__ long long flat_index(float x, float y, float z, const GridInfo& g) {
    const int ix = axis_index(x, g.x_lo, g.sx, g.nx);
    const int iy = axis_index(y, g.y_lo, g.sy, g.ny);
    const int iz = axis_index(z, g.z_lo, g.sz, g.nz);
    return ((long long)ix * g.ny + iy) * g.nz + iz;
}

// slab_entry_distance (geometry/grid.py:83): distance from an outside point to
// the box along u; a miss is >= kInfinityCm.
__device__ inline float slab_entry_distance(float x, float y, float z, float ux, float uy, float uz,
                                            const GridInfo& g) {
    float t_near = 0.0f;
    float t_far = INFINITY;
    if (ux == 0.0f) {
        if (x < g.x_lo || x >= g.x_hi) return INFINITY;
    } else {
        float t1 = (g.x_lo - x) / ux, t2 = (g.x_hi - x) / ux;
        if (t1 > t2) { float t = t1; t1 = t2; t2 = t; }
        t_near = fmaxf(t_near, t1);
        t_far = fminf(t_far, t2);
    }
    if (uy == 0.0f) {
        if (y < g.y_lo || y >= g.y_hi) return INFINITY;
    } else {
        float t1 = (g.y_lo - y) / uy, t2 = (g.y_hi - y) / uy;
        if (t1 > t2) { float t = t1; t1 = t2; t2 = t; }
        t_near = fmaxf(t_near, t1);
        t_far = fminf(t_far, t2);
    }
    if (uz == 0.0f) {
        if (z < g.z_lo || z >= g.z_hi) return INFINITY;
    } else {
        float t1 = (g.z_lo - z) / uz, t2 = (g.z_hi - z) / uz;
        if (t1 > t2) { float t = t1; t1 = t2; t2 = t; }
        t_near = fmaxf(t_near, t1);
        t_far = fminf(t_far, t2);
    }
    if (t_near > t_far || t_far <= 0.0f) return INFINITY;
    return t_near;
}

// distance_to_voxel_boundary (geometry/grid.py:151), clamped non-negative so a
// sub-ulp face position cannot produce a negative (trapping) substep.
__device__ inline float distance_to_voxel_boundary(float x, float y, float z, float ux, float uy,
                                                   float uz, const GridInfo& g) {
    float r = INFINITY;
    const int ix = axis_index(x, g.x_lo, g.sx, g.nx);
    if (ux > 0.0f) r = fminf(r, (g.x_lo + (float)(ix + 1) * g.sx - x) / ux);
    else if (ux < 0.0f) r = fminf(r, (g.x_lo + (float)ix * g.sx - x) / ux);
    const int iy = axis_index(y, g.y_lo, g.sy, g.ny);
    if (uy > 0.0f) r = fminf(r, (g.y_lo + (float)(iy + 1) * g.sy - y) / uy);
    else if (uy < 0.0f) r = fminf(r, (g.y_lo + (float)iy * g.sy - y) / uy);
    const int iz = axis_index(z, g.z_lo, g.sz, g.nz);
    if (uz > 0.0f) r = fminf(r, (g.z_lo + (float)(iz + 1) * g.sz - z) / uz);
    else if (uz < 0.0f) r = fminf(r, (g.z_lo + (float)iz * g.sz - z) / uz);
    return fmaxf(r, 0.0f);
}

// ---- tables (data/tables.py) --------------------------------------------------
// Device layout: the quantities one lookup needs together share a vector.
//   photon grid, per material:  ch[m][i]  = (compton, photo, pair, rayleigh)
//   photon grid:                maj[i]
//   electron grid, per material: ea[m][i] = (csda_range, moller, restricted_range,
//                                            stopping_radiative)
//                                eb[m][i] = (scattering_power, log_eta)
//                                ec[m][i] = stopping_restricted (dose-to-water)
//   range grid, per material:    er[m][i] = energy_of_restricted_range
// Interpolation is linear in value on the log grid, clamped flat outside
// (lookup_loglinear_1d/2d, data/tables.py:83-133).
struct Tables {
    const float4* ch;
    const float* maj;
    const float4* ea;
    const float2* eb;
    const float* ec;
    const float* er;
    const float* coh_x;    // [n_coherent]
    const float* coh_cum;  // [n_mat][n_coherent]
    int n_points;
    int n_materials;
    int n_coherent;
    float p_log_min, p_inv_dlog;
    float e_log_min, e_inv_dlog;
    float r_log_min, r_inv_dlog;
    // Goudsmit-Saunderson grid, corner-packed: gs4[(ix * (n_theta2-1) + iy) * n_u + u]
    // = (g[ix][iy][u], g[ix+1][iy][u], g[ix][iy+1][u], g[ix+1][iy+1][u]).
    const float4* gs4;
    int gs_ix0, gs_iy0, gs_n_eta, gs_n_theta2, gs_n_u;
    float gs_bins_per_log;
};

struct LogIdx {
    int i;
    float w;
};

__device__ __forceinline__ LogIdx log_index(float q, float log_min, float inv_dlog, int n) {
    float t = (logf(q) - log_min) * inv_dlog;
    t = fminf(fmaxf(t, 0.0f), (float)(n - 1));
    LogIdx r;
    r.i = min((int)t, n - 2);
    r.w = t - (float)r.i;
    return r;
}

// Table reads: kShared selects a copy staged in the block's shared memory
// (plain loads) over the read-only global path (__ldg, which must never see a
// shared-memory address).  The values are the same either way.
template <bool kShared, typename T>
__device__ __forceinline__ T ld_tab(const T* p) {
    if constexpr (kShared) return *p;
    else return __ldg(p);
}

template <bool kShared = false>
__device__ __forceinline__ float lerp1(const float* v, LogIdx li) {
    return ld_tab<kShared>(v + li.i) * (1.0f - li.w) + ld_tab<kShared>(v + li.i + 1) * li.w;
}
template <bool kShared = false>
__device__ __forceinline__ float2 lerp2(const float2* v, LogIdx li) {
    const float2 a = ld_tab<kShared>(v + li.i), b = ld_tab<kShared>(v + li.i + 1);
    const float u = 1.0f - li.w;
    return make_float2(a.x * u + b.x * li.w, a.y * u + b.y * li.w);
}
template <bool kShared = false>
__device__ __forceinline__ float4 lerp4(const float4* v, LogIdx li) {
    const float4 a = ld_tab<kShared>(v + li.i), b = ld_tab<kShared>(v + li.i + 1);
    const float u = 1.0f - li.w;
    return make_float4(a.x * u + b.x * li.w, a.y * u + b.y * li.w, a.z * u + b.z * li.w,
                       a.w * u + b.w * li.w);
}

}  // namespace pmc
