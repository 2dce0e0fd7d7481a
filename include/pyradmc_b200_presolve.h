/*
 * pyradmc_b200_presolve.h — C-ABI of the treatment-head pre-solve on the GPU
 * (libpmc_b200.so).
 *
 * Replaces pyRadMC's device pre-solve (backends/warp/presolve.py:356-544, the
 * kernel, and :572-687, presolve_head_device) and follows its host oracle
 * (geometry/head.py:373-575, presolve_head): primaries sampled on the host
 * from a planar photon source are traced through a beam-limiting stack of jaw
 * pairs and multi-leaf collimators (geometry/collimation.py:280-490, the
 * scalar chord-length twins) and an optional air column, one thread per
 * primary, and the exit-plane particles are appended to an output buffer:
 *   - every primary's transmitted copy, weight w exp(-tau_stack - tau_air);
 *   - mode 1 (first Compton), when the stack's optical depth is positive:
 *     one forced Compton photon from the device sampled by its share of the
 *     optical depth, at that device's mid-plane crossing, weight
 *     w (1 - e^-tau) (mu_compton / mu_total) e^-tau_out, rouletted below the
 *     weight floor;
 *   - mode 1 with an air column, for forward primaries with tau_air > 0: the
 *     Compton photon and the recoil electron of a forced interaction at an
 *     exponentially sampled depth, each rouletted separately.
 * Particles fly straight to the plane w = exit_z; backward-going ones, those
 * below the cutoff (pcut photons, ecut electrons) and zero weights are
 * dropped, their weight x energy summed into *dropped.  Weights are NOT
 * normalized per primary (the caller scales them by count / n, as
 * _Population.build does).  The random streams are the project's Philox
 * streams keyed by (seed, primary index): the result agrees with the host
 * oracle in distribution, never bit for bit (as pyRadMC's own device twin).
 *
 * Geometry (all float64 on the host, float32 on the device): the beam frame
 * has its origin at the focal spot and rows u, v, w of `rotation`; a point p
 * maps to rotation . (p - origin).  Device j is a jaw pair (kind 0) or an MLC
 * (kind 1) occupying z_top[j] <= w <= z_bottom[j]; the fields are those of
 * pyRadMC's CompiledStack (collimation.py:871-903).
 *
 * Macroscopic attenuation: mu tables per row (the stack's devices in order,
 * then the air column), log-log on n_table energies: log_total[row][k] and
 * log_compton[row][k] at log_energy[k] (head.py:119-180), interpolated
 * linearly in log energy and clamped at the ends.
 *
 * Return codes as in pyradmc_b200.h: PMC_OK, PMC_ERR_INVALID for bad
 * arguments, PMC_ERR_CAPACITY (and *count = the particles produced) when more
 * than `capacity` particles were produced, PMC_ERR_CUDA for a CUDA failure.
 * Every call allocates and frees its own device buffers and synchronizes.
 */
#ifndef PYRADMC_B200_PRESOLVE_H
#define PYRADMC_B200_PRESOLVE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pmc_head_stack {
    int32_t n_devices;
    double origin[3];
    double rotation[9];          /* rows u, v, w */
    const int32_t* kind;         /* [n_devices] 0 jaw pair, 1 MLC */
    const double* z_top;         /* [n_devices] */
    const double* z_bottom;
    const int32_t* jaw_axis;     /* 0 u, 1 v */
    const double* jaw_edge_neg;
    const double* jaw_edge_pos;
    const int32_t* jaw_focused;
    const double* mlc_tip_radius;
    const int32_t* mlc_focused_sides;
    const int32_t* mlc_n_pairs;
    const int32_t* mlc_edges_off; /* into leaf_edges_v */
    const int32_t* mlc_tips_off;  /* into tips_neg / tips_pos */
    const double* leaf_edges_v;   /* [n_leaf_edges] */
    int64_t n_leaf_edges;
    const double* tips_neg;       /* [n_tips] */
    const double* tips_pos;
    int64_t n_tips;
} pmc_head_stack;

typedef struct pmc_head_mu {
    int32_t n_rows;               /* stack devices, then the air column (if any) */
    int32_t n_table;
    const double* log_energy;     /* [n_table] ascending */
    const double* log_total;      /* [n_rows][n_table] */
    const double* log_compton;    /* [n_rows][n_table] */
} pmc_head_mu;

typedef struct pmc_head_params {
    int32_t first_compton;        /* 0 attenuation only, 1 forced first Compton */
    int32_t has_air;
    int32_t air_row;              /* mu row of the air column */
    int32_t outputs_on_device;    /* 1: the out_* arrays of pmc_presolve_head are device
                                     pointers of the current device (no copy back) */
    double air_z_start, air_z_end;
    double exit_z;
    double pcut, ecut;
    double weight_floor;          /* roulette of forced secondaries below it; 0 off */
    uint64_t seed;
} pmc_head_params;

/* The chord length (cm) of each engine-frame ray (pos, dir: [n][3] float32)
 * through each device of the stack: out[i][j], float32 [n][n_devices].  With
 * from_origin != 0 only the forward half-line t >= 0 counts.  A ray trapped
 * inside a block parallel to its slab has an infinite length. */
int pmc_head_path_lengths(const pmc_head_stack* stack, int64_t n, const float* pos, const float* dir,
                          int32_t from_origin, float* out);

/* The pre-solve of n primaries (host arrays: energy [n], pos [n][3], dir [n][3],
 * weight [n], all photons) into at most `capacity` exit-plane particles (arrays
 * kind [capacity] with 1 photon, 2 electron, energy, pos [capacity][3], dir,
 * weight: host arrays, or device arrays when params->outputs_on_device).
 * *count = particles written; *dropped = dropped weight x energy (MeV).
 * capacity >= n * (1 + first_compton * (1 + 2 * has_air)) always suffices. */
int pmc_presolve_head(const pmc_head_stack* stack, const pmc_head_mu* mu, const pmc_head_params* params,
                      int64_t n, const float* energy, const float* pos, const float* dir,
                      const float* weight, int64_t capacity, int32_t* out_kind, float* out_energy,
                      float* out_pos, float* out_dir, float* out_weight, int64_t* count,
                      double* dropped);

#ifdef __cplusplus
}
#endif

#endif /* PYRADMC_B200_PRESOLVE_H */
