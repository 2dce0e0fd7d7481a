// pmc_stack.cuh — a beam-limiting stack on the device: jaw pairs and
// multi-leaf collimators as flat float32 arrays, the chord length of a ray
// through each device, and log-log attenuation tables.  Shared by the
// treatment-head pre-solve (pmc_presolve.cu) and the transport's primary
// generator (stack transmission of a collimated source).
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace pmc_head {

constexpr int kMaxDevices = 16;

// The fields of pyRadMC's CompiledStack (geometry/collimation.py:871-903) in
// the beam frame: origin at the focal spot, rows u, v, w of rot.
struct Stack {
    int n;
    float origin[3];
    float rot[9];
    const int* kind;
    const float* z_top;
    const float* z_bottom;
    const int* jaw_axis;
    const float* jaw_neg;
    const float* jaw_pos;
    const int* jaw_focused;
    const float* tip_radius;
    const int* focused_sides;
    const int* n_pairs;
    const int* edges_off;
    const int* tips_off;
    const float* leaf_edges;
    const float* tips_neg;
    const float* tips_pos;
};

struct Mu {
    int n_rows, n_table;
    float log_e0, inv_dlog;  // the table's energies are log-uniform
    const float* log_total;
    const float* log_compton;
};

// ---- chord lengths (collimation.py:253-490) ------------------------------------
__device__ __forceinline__ float clip_len(float lo, float hi) { return hi <= lo ? 0.0f : hi - lo; }

// [s_lo, s_hi] within the half-space a + t b >= 0 (<= 0 when !above).
__device__ __forceinline__ float affine_len(float s_lo, float s_hi, float a, float b, bool above) {
    if (b == 0.0f) {
        const bool inside = above ? a >= 0.0f : a <= 0.0f;
        return inside ? clip_len(s_lo, s_hi) : 0.0f;
    }
    const float t_root = -a / b;
    const bool opens_up = above ? b > 0.0f : b < 0.0f;
    return opens_up ? clip_len(fmaxf(s_lo, t_root), s_hi) : clip_len(s_lo, fminf(s_hi, t_root));
}

// The slab z_top <= w <= z_bottom along the ray (false: the ray misses it).
__device__ __forceinline__ bool slab(float p_w, float d_w, float z_top, float z_bottom, int from_origin,
                                     float& s_lo, float& s_hi) {
    if (d_w == 0.0f) {
        if (p_w < z_top || p_w > z_bottom) return false;
        s_lo = -INFINITY;
        s_hi = INFINITY;
    } else {
        const float ta = (z_top - p_w) / d_w, tb = (z_bottom - p_w) / d_w;
        s_lo = fminf(ta, tb);
        s_hi = fmaxf(ta, tb);
    }
    if (from_origin) s_lo = fmaxf(s_lo, 0.0f);
    return true;
}

__device__ inline float jaw_len(const Stack& S, int j, const float* p, const float* d, int from_origin) {
    float s_lo, s_hi;
    if (!slab(p[2], d[2], S.z_top[j], S.z_bottom[j], from_origin, s_lo, s_hi)) return 0.0f;
    const int q = S.jaw_axis[j];
    const float e_pos = S.jaw_pos[j], e_neg = S.jaw_neg[j];
    float a_pos, b_pos, a_neg, b_neg;
    if (S.jaw_focused[j]) {  // the face pivots through the focal spot: z_mid q = edge w
        const float z_mid = 0.5f * (S.z_top[j] + S.z_bottom[j]);
        a_pos = z_mid * p[q] - e_pos * p[2];
        b_pos = z_mid * d[q] - e_pos * d[2];
        a_neg = z_mid * p[q] - e_neg * p[2];
        b_neg = z_mid * d[q] - e_neg * d[2];
    } else {
        a_pos = p[q] - e_pos;
        b_pos = d[q];
        a_neg = p[q] - e_neg;
        b_neg = d[q];
    }
    return affine_len(s_lo, s_hi, a_pos, b_pos, true) + affine_len(s_lo, s_hi, a_neg, b_neg, false);
}

// One rounded leaf end within [is_lo, is_hi]: the flat body (u >= c for the
// +u bank) united with the tip disc of radius r about (c, z_mid) in the (u, w)
// plane, by inclusion-exclusion.
__device__ inline float tip_len(float is_lo, float is_hi, const float* p, const float* d, float c, float z_mid,
                         float r, bool above) {
    float bo_lo, bo_hi;
    if (d[0] == 0.0f) {
        const bool inside = above ? p[0] >= c : p[0] <= c;
        bo_lo = inside ? -INFINITY : INFINITY;
        bo_hi = inside ? INFINITY : -INFINITY;
    } else {
        const float t_edge = (c - p[0]) / d[0];
        const bool opens_up = above ? d[0] > 0.0f : d[0] < 0.0f;
        bo_lo = opens_up ? t_edge : -INFINITY;
        bo_hi = opens_up ? INFINITY : t_edge;
    }
    const float ou = p[0] - c, ow = p[2] - z_mid;
    const float qa = d[0] * d[0] + d[2] * d[2];
    const float qb = 2.0f * (d[0] * ou + d[2] * ow);
    const float qc = ou * ou + ow * ow - r * r;
    float di_lo, di_hi;
    if (qa > 0.0f) {
        const float disc = qb * qb - 4.0f * qa * qc;
        if (disc > 0.0f) {
            const float hw = sqrtf(disc);
            di_lo = (-qb - hw) / (2.0f * qa);
            di_hi = (-qb + hw) / (2.0f * qa);
        } else {
            di_lo = INFINITY;
            di_hi = -INFINITY;
        }
    } else {  // parallel to the cylinder's axis: wholly inside or outside
        di_lo = qc <= 0.0f ? -INFINITY : INFINITY;
        di_hi = qc <= 0.0f ? INFINITY : -INFINITY;
    }
    const float body = clip_len(fmaxf(is_lo, bo_lo), fminf(is_hi, bo_hi));
    const float disc_l = clip_len(fmaxf(is_lo, di_lo), fminf(is_hi, di_hi));
    const float both = clip_len(fmaxf(is_lo, fmaxf(bo_lo, di_lo)), fminf(is_hi, fminf(bo_hi, di_hi)));
    return body + disc_l - both;
}

__device__ inline float mlc_len(const Stack& S, int j, const float* p, const float* d, int from_origin) {
    float s_lo, s_hi;
    if (!slab(p[2], d[2], S.z_top[j], S.z_bottom[j], from_origin, s_lo, s_hi)) return 0.0f;
    const float z_mid = 0.5f * (S.z_top[j] + S.z_bottom[j]);
    const float r = S.tip_radius[j];
    // the leaf side planes as affine functions of t: z_mid v = edge w when
    // focused, v = edge (k, w_p, w_d) = (1, 1, 0) otherwise
    const bool foc = S.focused_sides[j] != 0;
    const float k = foc ? z_mid : 1.0f, w_p = foc ? p[2] : 1.0f, w_d = foc ? d[2] : 0.0f;
    const float* edges = S.leaf_edges + S.edges_off[j];
    const float* t_neg = S.tips_neg + S.tips_off[j];
    const float* t_pos = S.tips_pos + S.tips_off[j];
    float total = 0.0f;
    for (int i = 0; i < S.n_pairs[j]; ++i) {
        const float a_lo = k * p[1] - edges[i] * w_p, b_lo = k * d[1] - edges[i] * w_d;
        const float a_hi = k * p[1] - edges[i + 1] * w_p, b_hi = k * d[1] - edges[i + 1] * w_d;
        float g_lo, g_hi, h_lo, h_hi;
        if (b_lo == 0.0f) {  // {a_lo + t b_lo >= 0}
            g_lo = a_lo >= 0.0f ? -INFINITY : INFINITY;
            g_hi = a_lo >= 0.0f ? INFINITY : -INFINITY;
        } else if (b_lo > 0.0f) {
            g_lo = -a_lo / b_lo;
            g_hi = INFINITY;
        } else {
            g_lo = -INFINITY;
            g_hi = -a_lo / b_lo;
        }
        if (b_hi == 0.0f) {  // {a_hi + t b_hi <= 0}
            h_lo = a_hi <= 0.0f ? -INFINITY : INFINITY;
            h_hi = a_hi <= 0.0f ? INFINITY : -INFINITY;
        } else if (b_hi < 0.0f) {
            h_lo = -a_hi / b_hi;
            h_hi = INFINITY;
        } else {
            h_lo = -INFINITY;
            h_hi = -a_hi / b_hi;
        }
        const float is_lo = fmaxf(s_lo, fmaxf(g_lo, h_lo));
        const float is_hi = fminf(s_hi, fminf(g_hi, h_hi));
        total += tip_len(is_lo, is_hi, p, d, t_pos[i] + r, z_mid, r, true);
        total += tip_len(is_lo, is_hi, p, d, t_neg[i] - r, z_mid, r, false);
    }
    return total;
}

__device__ __forceinline__ float device_len(const Stack& S, int j, const float* p, const float* d,
                                            int from_origin) {
    return S.kind[j] == 0 ? jaw_len(S, j, p, d, from_origin) : mlc_len(S, j, p, d, from_origin);
}

__device__ __forceinline__ void to_local(const Stack& S, const float* x, const float* u, float* p, float* d) {
    const float dx = x[0] - S.origin[0], dy = x[1] - S.origin[1], dz = x[2] - S.origin[2];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        p[r] = S.rot[3 * r] * dx + S.rot[3 * r + 1] * dy + S.rot[3 * r + 2] * dz;
        d[r] = S.rot[3 * r] * u[0] + S.rot[3 * r + 1] * u[1] + S.rot[3 * r + 2] * u[2];
    }
}

// Macroscopic mu of a row: linear in log energy on the log-log table, clamped.
__device__ __forceinline__ float mu_at(const Mu& M, const float* table, int row, float e) {
    float t = (logf(e) - M.log_e0) * M.inv_dlog;
    t = fminf(fmaxf(t, 0.0f), (float)(M.n_table - 1));
    const int i = min((int)t, M.n_table - 2);
    const float f = t - (float)i;
    const float* r = table + (long long)row * M.n_table;
    return expf(r[i] * (1.0f - f) + r[i + 1] * f);
}


}  // namespace pmc_head
