// pmc_physics.cuh — scalar physics samplers, float32, one per reference
// function in pyradmc/physics/*.py.  Each consumes exactly the uniforms its
// reference counterpart consumes, in the same order.
#pragma once

#include "pmc_common.cuh"

namespace pmc {

// physics/path.py:15 — s = -ln(1 - u) / mu.  1 - u is exact for a 24-bit u.
__device__ __forceinline__ float sample_path_length(float mu, Rng& rng) {
    return -logf(1.0f - rng.uniform()) / mu;
}

// physics/direction.py:34 — rotate (ux, uy, uz) by polar cos_theta, azimuth phi.
__device__ __forceinline__ void rotate_direction(float& ux, float& uy, float& uz, float cos_theta,
                                                 float phi) {
    const float sin_theta = sqrtf(fmaxf(0.0f, 1.0f - cos_theta * cos_theta));
    float sin_phi, cos_phi;
    sincosf(phi, &sin_phi, &cos_phi);
    const float t2 = ux * ux + uy * uy;
    if (t2 > kPoleFloor) {
        const float t = sqrtf(t2);
        const float inv = sin_theta / t;
        const float vx = ux * cos_theta + inv * (ux * uz * cos_phi - uy * sin_phi);
        const float vy = uy * cos_theta + inv * (uy * uz * cos_phi + ux * sin_phi);
        const float vz = uz * cos_theta - t * sin_theta * cos_phi;
        ux = vx;
        uy = vy;
        uz = vz;
        return;
    }
    const float sign = uz > 0.0f ? 1.0f : -1.0f;
    ux = sin_theta * cos_phi;
    uy = sign * sin_theta * sin_phi;
    uz = sign * cos_theta;
}

// physics/direction.py:23 — isotropic direction, two uniforms.
__device__ __forceinline__ void sample_isotropic_direction(Rng& rng, float& ax, float& ay,
                                                           float& az) {
    const float c = 1.0f - 2.0f * rng.uniform();
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    const float phi = kTwoPi * rng.uniform();
    float sp, cp;
    sincosf(phi, &sp, &cp);
    ax = s * cp;
    ay = s * sp;
    az = c;
}

// physics/compton.py:19 — Kahn's rejection for r = E'/E; three uniforms per round.
__device__ inline float sample_compton_energy_ratio(float energy, Rng& rng) {
    const float alpha = energy / kElectronMass;
    const float two_alpha = 2.0f * alpha;
    const float branch = (1.0f + two_alpha) / (9.0f + two_alpha);
    for (int round = 0; round < (1 << 20); ++round) {
        const float u1 = rng.uniform();
        const float u2 = rng.uniform();
        const float u3 = rng.uniform();
        if (u1 <= branch) {
            const float x = 1.0f + two_alpha * u2;
            if (u3 <= 4.0f * (x - 1.0f) / (x * x)) return 1.0f / x;
        } else {
            const float x = (1.0f + two_alpha) / (1.0f + two_alpha * u2);
            const float c = 1.0f - (x - 1.0f) / alpha;
            if (u3 <= 0.5f * (c * c + 1.0f / x)) return 1.0f / x;
        }
    }
    return 1.0f;  // unreachable for any physical energy; bounded so no lane can spin
}

// physics/compton.py:67
__device__ __forceinline__ float compton_cos_theta(float energy, float ratio) {
    const float alpha = energy / kElectronMass;
    const float c = 1.0f + 1.0f / alpha - 1.0f / (alpha * ratio);
    return fminf(1.0f, fmaxf(-1.0f, c));
}

// physics/compton.py:91
__device__ __forceinline__ float compton_electron_cos_theta(float energy, float ratio) {
    const float recoil = energy * (1.0f - ratio);
    const float p = sqrtf(recoil * (recoil + 2.0f * kElectronMass));
    const float cg = compton_cos_theta(energy, ratio);
    const float ce = (energy - ratio * energy * cg) / p;
    return fminf(1.0f, fmaxf(-1.0f, ce));
}

// physics/channel.py:17 — channel by cumulative inversion on one uniform.
__device__ __forceinline__ int select_photon_process(float c, float p, float pair, float r,
                                                     Rng& rng) {
    const float threshold = rng.uniform() * (c + p + pair + r);
    if (threshold < c) return 0;
    if (threshold < c + p) return 1;
    if (threshold < c + p + pair) return 2;
    return 3;
}

// physics/roulette.py:25 — one fair game; one uniform.
__device__ __forceinline__ float roulette_weight(float w, float survival, Rng& rng) {
    float survivor = 0.0f;
    if (rng.uniform() < survival) survivor = w / survival;
    return survivor;
}

// physics/brems.py:30 — (emission probability, local sub-PCUT deposit).
__device__ __forceinline__ void brems_step_parameters(float e, float s_rad, float rho, float step,
                                                      float pcut, float& prob, float& local) {
    const float loss = s_rad * rho * step;
    if (e <= pcut) {
        prob = 0.0f;
        local = loss;
        return;
    }
    const float emitted = 1.0f - pcut / e;
    const float mean_k = (e - pcut) / logf(e / pcut);
    prob = loss * emitted / mean_k;
    local = loss * (1.0f - emitted);
}

// physics/brems.py:69 — k = PCUT (E/PCUT)^u; one uniform.
__device__ __forceinline__ float sample_brems_energy(float e, float pcut, Rng& rng) {
    return pcut * expf(rng.uniform() * logf(e / pcut));
}

// physics/moller.py:18 — restricted Moller DCS by rejection; two uniforms per round.
__device__ inline float sample_moller_delta_energy(float e, float cut, Rng& rng) {
    const float tau = e / kElectronMass;
    const float tr = tau / (tau + 1.0f);
    const float tr2 = tr * tr;
    const float two_tau = (2.0f * tau + 1.0f) / ((tau + 1.0f) * (tau + 1.0f));
    const float w_min = cut / e;
    const float bound = 2.0f + 0.25f * tr2;
    for (int round = 0; round < (1 << 20); ++round) {
        const float u = rng.uniform();
        const float x = w_min / (1.0f - u * (1.0f - 2.0f * w_min));
        const float ratio = x / (1.0f - x);
        const float accept = 1.0f + ratio * ratio + x * x * tr2 - two_tau * ratio;
        if (rng.uniform() * bound <= accept) return x * e;
    }
    return cut;  // bounded; the acceptance is >= 1/2.25 per round
}

// physics/moller.py:60
__device__ __forceinline__ void moller_direction_cosines(float e, float w, float& cd, float& cp) {
    const float two_m = 2.0f * kElectronMass;
    cd = sqrtf(w * (e + two_m) / (e * (w + two_m)));
    const float rest = e - w;
    cp = sqrtf(rest * (e + two_m) / (e * (rest + two_m)));
    cd = fminf(1.0f, cd);
    cp = fminf(1.0f, cp);
}

// physics/msc.py:37 — Gaussian hinge; one uniform.
__device__ __forceinline__ float sample_hinge_cos_theta(float ms, Rng& rng) {
    const float theta = sqrtf(-ms * logf(1.0f - rng.uniform()));
    return cosf(fminf(theta, kPi));
}

// expm1 for the GS anchor 1 - exp(-theta2/2).  CUDA's expm1f keeps full float
// precision at the tiny arguments short substeps produce.
__device__ __forceinline__ float gs_one_minus_cos(float ms) { return -expm1f(-0.5f * ms); }

// physics/gs.py:102 + :39 — bilinear blend of the four bracketing tables at
// one equal-probability bin; one uniform (none when <theta^2> <= 0).
__device__ inline float sample_gs_cos_theta(const Tables& t, float fx, float fy, float ms,
                                            Rng& rng) {
    int ix = (int)floorf(fx) - t.gs_ix0;
    int iy = (int)floorf(fy) - t.gs_iy0;
    ix = min(max(ix, 0), t.gs_n_eta - 2);
    iy = min(max(iy, 0), t.gs_n_theta2 - 2);
    const float tx = fminf(fmaxf(fx - (float)(t.gs_ix0 + ix), 0.0f), 1.0f);
    const float ty = fminf(fmaxf(fy - (float)(t.gs_iy0 + iy), 0.0f), 1.0f);
    if (ms <= 0.0f) return 1.0f;
    const float u = rng.uniform() * (float)t.gs_n_u;
    int index = (int)u;
    if (index > t.gs_n_u - 1) index = t.gs_n_u - 1;
    const float4 c =
        __ldg(t.gs4 + ((long long)ix * (t.gs_n_theta2 - 1) + iy) * t.gs_n_u + index);
    const float w_lo = c.x * (1.0f - tx) + c.y * tx;
    const float w_hi = c.z * (1.0f - tx) + c.w * tx;
    const float w = w_lo * (1.0f - ty) + w_hi * ty;
    return fmaxf(-1.0f, 1.0f - w * gs_one_minus_cos(ms));
}

// physics/rayleigh.py — ascending-abscissa interpolation, flat outside.
__device__ inline float interp_increasing(float q, const float* xs, const float* ys, int n) {
    if (q <= __ldg(xs)) return __ldg(ys);
    if (q >= __ldg(xs + n - 1)) return __ldg(ys + n - 1);
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(xs + mid) <= q) lo = mid;
        else hi = mid;
    }
    const float x_lo = __ldg(xs + lo), x_hi = __ldg(xs + hi);
    const float tt = (q - x_lo) / (x_hi - x_lo);
    return __ldg(ys + lo) * (1.0f - tt) + __ldg(ys + hi) * tt;
}

// physics/rayleigh.py:43 — coherent cosine from the form-factor cumulative.
__device__ inline float sample_coherent_cos_theta(const Tables& t, int mat, float e, Rng& rng) {
    const float* cum = t.coh_cum + (long long)mat * t.n_coherent;
    const float x_max = kRayleighPerMeV * e;
    const float a_max = interp_increasing(x_max, t.coh_x, cum, t.n_coherent);
    for (int round = 0; round < (1 << 20); ++round) {
        const float target = rng.uniform() * a_max;
        const float x = interp_increasing(target, cum, t.coh_x, t.n_coherent);
        const float ratio = x / x_max;
        const float mu = 1.0f - 2.0f * ratio * ratio;
        if (2.0f * rng.uniform() <= 1.0f + mu * mu) return mu;
    }
    return 1.0f;
}

// transport/electron.py:169 substep_pieces — ceil(length / resolution) in [1, 1024].
__device__ __forceinline__ int substep_pieces(float length, float resolution) {
    if (resolution <= 0.0f) return 1;
    const int n = (int)ceilf(length / resolution);
    if (n < 1) return 1;
    if (n > 1024) return 1024;
    return n;
}

}  // namespace pmc
