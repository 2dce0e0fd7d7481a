/*
 * pyradmc_b200.h — C-ABI of the B200 Monte Carlo dose backend (libpmc_b200.so).
 *
 * The library replaces the device side of pyRadMC's Warp backend
 * (pyradmc/backends/warp/engine.py, pyradmc/backends/warp/kernels.py): photon
 * Woodcock transport, Class II condensed-history electron transport with
 * Goudsmit-Saunderson multiple scattering, int64 fixed-point beamlet-tagged
 * scoring, the per-batch float64 fold, finalize, and the truncation + CSC
 * compaction of the dose-influence matrix.  Everything here is plain C types:
 * host pointers and sizes in, host buffers out.  A Python host binds it with
 * ctypes (pyradmc_b200/engine.py); any other FFI can bind it the same way.
 *
 * Conventions
 *   - Every entry point returns 0 (PMC_OK) or a negative PMC_ERR_* code; the
 *     message of the last failure is pmc_last_error(engine).
 *   - Host buffers are caller-owned.  Device memory is engine-owned.
 *   - One engine per host thread; calls on one engine are not re-entrant.  All
 *     device work of a call is ordered on the engine's own CUDA stream, and a
 *     call returns only after that work has finished.
 *   - No call waits without bound: every device loop carries a step cap and a
 *     round cap, and a tripped cap is reported as PMC_ERR_STEP_CAP.
 */
#ifndef PYRADMC_B200_H
#define PYRADMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PMC_ABI_VERSION 2

/* Return codes.  The Python host maps them onto the reference's exceptions:
 * INVALID -> ValueError (engine.py:512-550), MAJORANT and QUEUE_OVERFLOW ->
 * RuntimeError (engine.py:685-690, engine.py:347-351). */
#define PMC_OK 0
#define PMC_ERR_INVALID (-1)
#define PMC_ERR_MAJORANT (-2)
#define PMC_ERR_QUEUE_OVERFLOW (-3)
#define PMC_ERR_STEP_CAP (-4)
#define PMC_ERR_CUDA (-5)
#define PMC_ERR_OOM (-6)
#define PMC_ERR_STATE (-7)
#define PMC_ERR_CAPACITY (-8) /* a caller-sized output buffer is too small */

/* Particle kinds: pyradmc/transport/particles.py:23-25. */
#define PMC_PHOTON 0
#define PMC_ELECTRON 1
#define PMC_POSITRON 2

/* Primary generators.  PENCIL/PARALLEL/SPECTRAL mirror the Warp generators
 * generate_pencil_beam (kernels.py:1888), generate_parallel_beam (:2035) and
 * generate_spectral_beam (:2071); UPLOAD mirrors generate_from_upload (:1922),
 * the host pre-sampling route of Source.sample_batch. */
#define PMC_SRC_PENCIL 0
#define PMC_SRC_PARALLEL 1
#define PMC_SRC_SPECTRAL 2
#define PMC_SRC_UPLOAD 3
/* A phase space kept resident on the device: history h draws record
 * floor(r * n_records), r a 64-bit draw of its own stream, the per-history
 * sampling of PhaseSpaceSource.emit (geometry/phasespace.py:546). */
#define PMC_SRC_PHASESPACE 4
/* The same, with the up_* arrays already in the engine device's memory (a
 * head pre-solve's output, pmc_presolve_head with outputs on the device): no
 * upload and no host check; every up_kind must be PMC_PHOTON, PMC_ELECTRON or
 * PMC_POSITRON, and the arrays must stay valid until the call returns (the
 * hand-off of generate_from_exit_buffer, kernels.py:1963-2032). */
#define PMC_SRC_PHASESPACE_DEVICE 5
/* The spectral fan seen through a 0..1 transmission mask on a plane rectangle
 * (TransmissionMaskSource wrapping SpectralBeamSource, geometry/collimation.py:
 * 987-1080 and 1205; the device twin generate_spectral_masked_beam,
 * kernels.py:2137-2244): the four uniforms of PMC_SRC_SPECTRAL, then the ray's
 * full line meets the mask plane and the primary's weight is the mask value
 * there, bilinear between pixel centres and clamped in the half-pixel border.
 * A ray parallel to the plane or crossing it outside the rectangle, or a zero
 * value, emits nothing (the history still counts in the batch mean).  The
 * mask_* fields describe the plane; mask[i * mask_n_v + j] is pixel i along
 * mask_u_axis and j along mask_v_axis, every value finite and in 0..1. */
#define PMC_SRC_SPECTRAL_MASKED 6

/* Beamlet generators: generate_beamlet_lattice (kernels.py:2248),
 * generate_spectral_beamlets (kernels.py:2322), per-beamlet records (fans and
 * lattice rectangles of any geometry, and per-beamlet mixtures of them:
 * CompositeBeamletSource, geometry/source.py:239-277), and the host
 * pre-sampling route of BeamletSource.sample_beamlet_batch
 * (engine.py:3224-3335 _generate_group_presampled). */
#define PMC_BEAMLET_LATTICE 0
#define PMC_BEAMLET_SPECTRAL 1
#define PMC_BEAMLET_RECORDS 2
#define PMC_BEAMLET_UPLOAD 3

typedef struct pmc_engine pmc_engine;

/* Flattened cross-section tables: the fields of CrossSectionTables
 * (pyradmc/data/tables.py:140-219).  Per-material arrays are row-major
 * [n_materials][n_points] float64; the engine casts to float32 on upload, as
 * WarpEngine._upload_tables does (engine.py:3368-3429). */
typedef struct pmc_tables_desc {
    int32_t n_materials;
    int32_t n_points;
    double photon_log_e_min, photon_inv_dlog;
    double electron_log_e_min, electron_inv_dlog;
    double range_log_r_min, range_inv_dlog;
    const double* mu_compton;
    const double* mu_photo;
    const double* mu_pair;
    const double* mu_rayleigh;
    const double* majorant; /* [n_points] */
    const double* stopping_restricted;
    const double* stopping_radiative;
    const double* moller;
    const double* csda_range;
    const double* scattering_power;
    const double* log_eta;
    const double* restricted_range;
    const double* energy_of_restricted_range;
    int32_t n_coherent;
    const double* coherent_x;          /* [n_coherent] */
    const double* coherent_cumulative; /* [n_materials][n_coherent] */
} pmc_tables_desc;

/* Scoring geometry: a rectilinear grid (pyradmc/scoring/grid.py:67) or, with
 * mode 1, depth bins by radial shells about an axis parallel to z
 * (CylindricalScoringGrid, pyradmc/scoring/cylinder.py:172; device side
 * _scoring_index, kernels.py:492-533).  A deposit outside it is booked to the
 * unscored ledger (kernels.py:536-585). */
typedef struct pmc_scoring_desc {
    int32_t nx, ny, nz;
    double origin[3];
    double spacing[3];
    const double* voxel_mass; /* [nx*ny*nz] grams, C order; mode 1: [n_depth][n_shells] */
    int32_t mode;             /* 0 rectilinear, 1 cylindrical */
    double axis[2];           /* mode 1: (x, y) of the axis */
    int32_t n_depth, n_shells;
    const double* depth_edges;  /* mode 1: [n_depth + 1], increasing */
    const double* radial_edges; /* mode 1: [n_shells + 1], increasing, >= 0 */
} pmc_scoring_desc;

/* Open-field primary source (WarpEngine.run, engine.py:454). */
struct pmc_head_stack;
struct pmc_head_mu;

typedef struct pmc_source_desc {
    int32_t type; /* PMC_SRC_* */
    int32_t kind; /* PMC_PHOTON or PMC_ELECTRON for the analytic beams */
    double energy;
    double position[3]; /* pencil */
    double direction[3];
    double z0, x_lo, x_extent, y_lo, y_extent; /* parallel */
    /* spectral fan (geometry/source.py:479 _DivergentFan.emit_through) */
    int32_t n_bins;
    const double* edges; /* [n_bins+1] */
    const double* cdf;   /* [n_bins] */
    double focal[3], center[3], u_axis[3], v_axis[3];
    double width_u, width_v;
    /* upload: one record per history, in history order */
    const int32_t* up_kind; /* PMC_PHOTON / PMC_ELECTRON / PMC_POSITRON */
    const float* up_energy;
    const float* up_pos;    /* [n][3] */
    const float* up_dir;    /* [n][3] */
    const float* up_weight;
    int64_t n_records; /* PMC_SRC_PHASESPACE: records in the up_* arrays */
    /* PMC_SRC_SPECTRAL_MASKED: the mask plane (engine frame, cm; unit axes).
     * A non-NULL mask on PMC_SRC_PENCIL, _PARALLEL or _SPECTRAL weights those
     * primaries the same way (TransmissionMaskSource over any built-in). */
    const double* mask; /* [mask_n_u][mask_n_v] */
    int32_t mask_n_u, mask_n_v;
    double mask_center[3], mask_u_axis[3], mask_v_axis[3];
    double mask_width_u, mask_width_v;
    /* Optional (NULL: none): a beam-limiting stack the primaries are seen
     * through, CollimatedSource (geometry/collimation.py:1154): each analytic
     * primary's weight is multiplied by exp(-sum_j mu_j(E) t_j), t_j the chord
     * of its full line through device j, mu_j row j of stack_mu's log_total
     * (macroscopic, density included; the log energies log-uniform).  A zero
     * transmission emits nothing.  Types declared in pyradmc_b200_presolve.h. */
    const struct pmc_head_stack* stack;
    const struct pmc_head_mu* stack_mu;
} pmc_source_desc;

/* One beamlet of a PMC_BEAMLET_RECORDS source: a lattice rectangle
 * (BeamletGridSource.emit, geometry/source.py:420: two uniforms, +z travel) or
 * a divergent fan through an aperture (_DivergentFan.emit_through, :479: four
 * uniforms, energy from the record's spectrum). */
typedef struct pmc_beamlet_rec {
    int32_t type;     /* PMC_BEAMLET_LATTICE or PMC_BEAMLET_SPECTRAL */
    int32_t spectrum; /* fan: index into the descriptor's spectra */
    double energy, z0;                             /* lattice */
    double x_lo, x_extent, y_lo, y_extent;         /* lattice */
    double focal[3], center[3], u_axis[3], v_axis[3]; /* fan (unit axes) */
    double width_u, width_v;                       /* fan */
} pmc_beamlet_rec;

/* Host pre-sampling callback of PMC_BEAMLET_UPLOAD: write the n primaries of
 * column `beamlet` (an index into this call's descriptor) whose transport
 * streams are keyed key_offset .. key_offset + n - 1, as
 * BeamletSource.sample_beamlet_batch(seed, key_offset, n, beamlet) does.
 * position and direction are [n][3]; every primary is a photon.  Return 0, or
 * non-zero to abort the call with PMC_ERR_INVALID. */
typedef int (*pmc_sample_fn)(void* user, int32_t beamlet, int64_t key_offset, int64_t n,
                             float* energy, float* position, float* direction, float* weight);

/* Beamlet source for run_dij (engine.py:948). */
typedef struct pmc_beamlet_desc {
    int32_t type; /* PMC_BEAMLET_* */
    int32_t n_beamlets;
    double energy, z0;                     /* lattice */
    const double* x_lo;                    /* [n_beamlets] */
    const double* x_extent;
    const double* y_lo;
    const double* y_extent;
    int32_t n_bins;                        /* spectral beamlets */
    const double* edges;
    const double* cdf;
    double focal[3], u_axis[3], v_axis[3];
    double width_u, width_v;
    const double* centers; /* [n_beamlets][3] */
    /* Optional [n_beamlets] first global history of each beamlet; NULL means the
     * exclusive prefix sum of counts.  Lets a caller run a range of beamlets
     * (one device's share) with the streams the whole matrix would use. */
    const int64_t* history_offsets;
    /* PMC_BEAMLET_RECORDS: records [n_beamlets][n_components]; with several
     * components a beamlet is a mixture: one uniform u picks the first
     * component whose component_cdf entry is >= u, then that record emits. */
    int32_t n_components;
    const pmc_beamlet_rec* records;
    const double* component_cdf;  /* [n_components], ends at 1 */
    int32_t n_spectra;
    const int32_t* spectrum_bins; /* [n_spectra] */
    const double* spectrum_edges; /* concatenated, spectrum_bins[k] + 1 each */
    const double* spectrum_cdf;   /* concatenated, spectrum_bins[k] each */
    /* PMC_BEAMLET_UPLOAD */
    pmc_sample_fn sample;
    void* sample_user;
    /* Optional stack transmission of every in-kernel beamlet primary, the
     * same fields as in pmc_source_desc: CollimatedBeamletSource,
     * geometry/collimation.py:1185 */
    const struct pmc_head_stack* stack;
    const struct pmc_head_mu* stack_mu;
    /* Optional (NULL: none) transmission mask of every in-kernel beamlet
     * primary, the fields of pmc_source_desc's mask:
     * TransmissionMaskBeamletSource, geometry/collimation.py:1264 */
    const double* mask;
    int32_t mask_n_u, mask_n_v;
    double mask_center[3], mask_u_axis[3], mask_v_axis[3];
    double mask_width_u, mask_width_v;
} pmc_beamlet_desc;

/* Run options: the keyword arguments of WarpEngine.run / run_dij plus the
 * scheduling knobs.  Scheduling knobs never change a result (bit-inert). */
typedef struct pmc_run_params {
    int64_t n_histories; /* run: total histories (divisible by n_batches) */
    int32_t n_batches;
    uint64_t seed;
    double pcut, ecut;
    int32_t transport_electrons;
    int32_t msc_gs; /* 1 Goudsmit-Saunderson, 0 Gaussian hinge */
    double step_energy_fraction;
    double deposit_resolution; /* <= 0: single midpoint deposit */
    int32_t dose_to_water;
    int32_t photon_split_n; /* Compton splitting of primaries; 1 = off */
    double truncation;      /* run_dij */
    int32_t correlated;     /* run_dij */
    int32_t beamlet_group_size; /* 0: auto */
    /* scheduling */
    int64_t chunk_size; /* new primaries admitted per transport round; 0: auto */
    int32_t queue_factor;
    int32_t block_size;     /* transport threads per block; 0: auto */
    int32_t blocks_per_sm;  /* transport blocks per SM; 0: auto */
    int32_t use_graph;      /* drain each batch inside one CUDA graph */
    int64_t max_steps;      /* per-particle step cap; 0: default */
    int32_t tail_steps;     /* steps a particle may take after its round's input ran dry
                               before it is parked for the next round; 0: default,
                               < 0: never park */
    int32_t smem_tables;    /* 1: stage the photon and electron table rows in shared
                               memory, -1: read them through L1, 0: auto */
} pmc_run_params;

/* Exact integer energy books of a call, in quanta of 1e-9 MeV
 * (kernels.py:96 ENERGY_QUANTUM_MEV). */
typedef struct pmc_books {
    int64_t deposited;
    int64_t escaped;
    int64_t unscored;
    int64_t emitted; /* booked per primary by the spectral/upload routes */
    int64_t majorant_violations;
} pmc_books;

/* Device event counters of the last call (for the roofline figures). */
typedef struct pmc_counters {
    int64_t photon_flights;
    int64_t photon_interactions;
    int64_t electron_substeps;
    int64_t deposits;
    int64_t queue_pushes;
    int64_t primaries;
    int64_t rounds;
    int64_t transport_launches; /* graph launches (or host-loop rounds) */
    int64_t reduce_launches;
    int64_t kernel_launches;    /* every kernel of this library the call ran */
    double transport_ms; /* device time of the transport kernels */
    double reduce_ms;    /* device time of fold/finalize/truncation */
    int64_t h2d_bytes_total; /* host-to-device bytes over the engine's life */
    int64_t d2h_bytes_total; /* device-to-host bytes over the engine's life */
} pmc_counters;

int pmc_abi_version(void);
int pmc_device_count(void);

/* Engine lifetime.  Replaces the per-call uploads WarpEngine performs
 * (_upload_grid engine.py:3336, _upload_tables :3368) with a resident engine. */
int pmc_create(pmc_engine** out, int device_ordinal);
void pmc_destroy(pmc_engine* engine);
const char* pmc_last_error(const pmc_engine* engine);

/* Transport grid: VoxelGrid (geometry/grid.py:227).  density float32 and
 * material uint8 per voxel, C order (x slowest), as _upload_grid casts them. */
int pmc_upload_grid(pmc_engine* engine, int32_t nx, int32_t ny, int32_t nz,
                    const double origin[3], const double spacing[3],
                    const float* density, const uint8_t* material);

/* Cross-section tables (data/tables.py:222 build_cross_section_tables). */
int pmc_upload_tables(pmc_engine* engine, const pmc_tables_desc* tables);

/* Goudsmit-Saunderson node grid (data/goudsmit_saunderson.py:1108
 * build_gs_grid): values [n_eta][n_theta2][n_u] float32, window origin
 * (ix0, iy0), bins_per_log nodes per natural log. */
int pmc_upload_gs(pmc_engine* engine, const float* values, int32_t ix0, int32_t iy0,
                  int32_t n_eta, int32_t n_theta2, int32_t n_u, double bins_per_log);

/* Scoring geometry; a call with NULL restores "score on the transport grid"
 * (ScoringGrid.for_grid, scoring/grid.py:113). */
int pmc_set_scoring(pmc_engine* engine, const pmc_scoring_desc* scoring);

/* Open-field run: WarpEngine.run (engine.py:454).  dose and dose_sigma are
 * caller buffers of n_scoring_voxels float64 (MeV/g per emitted history). */
int pmc_run_forward(pmc_engine* engine, const pmc_source_desc* source,
                    const pmc_run_params* params, double* dose, double* dose_sigma,
                    pmc_books* books);

/* Dij: WarpEngine.run_dij (engine.py:948).  counts[j] is beamlet j's history
 * count (each divisible by n_batches); equal counts reproduce the reference
 * mapping h = j * n_per + r (backends/ref/engine.py:410-442).  The CSC result
 * stays on the engine; *nnz receives its entry count. */
int pmc_run_dij(pmc_engine* engine, const pmc_beamlet_desc* source, const int64_t* counts,
                const pmc_run_params* params, int64_t* nnz, pmc_books* books);

/* Copy the CSC of the last pmc_run_dij into caller buffers:
 * indptr[n_beamlets+1], indices[nnz], dose[nnz], sigma[nnz]
 * (DijResult fields, scoring/dij.py:195-229). */
int pmc_dij_fetch(pmc_engine* engine, int64_t* indptr, int64_t* indices, double* dose,
                  double* sigma);

/* The CSC of the last pmc_run_dij left on the device (no counterpart in the
 * reference, whose Dij is always assembled on the host): indptr[n_beamlets+1]
 * is copied into the caller's host buffer, and *indices, *dose, *sigma receive
 * DEVICE pointers to the nnz entries, owned by the engine and valid until its
 * next run or pmc_destroy.  For device-side consumers of the Dij (the
 * denoiser) that would otherwise copy it to the host and back. */
int pmc_dij_device_view(pmc_engine* engine, int64_t* indptr, const int64_t** indices,
                        const double** dose, const double** sigma);

int pmc_get_counters(const pmc_engine* engine, pmc_counters* counters);

/* Run the engine's work on the caller's CUDA stream (a cudaStream_t passed as
 * void*), e.g. to bracket it with the caller's own events; NULL restores the
 * engine's private stream. */
int pmc_set_stream(pmc_engine* engine, void* stream);

/* Progress: fn(user, histories) is called from the calling thread after each
 * completed batch of pmc_run_forward and each completed beamlet group of
 * pmc_run_dij, with the histories that completed (progress.py:71 tick).  A
 * NULL fn disables it. */
typedef void (*pmc_progress_fn)(void* user, int64_t histories);
int pmc_set_progress(pmc_engine* engine, pmc_progress_fn fn, void* user);

/* Device reduction entry points, exposed on their own for the parity tests
 * against the host scorers.  All pointers are host buffers.
 *   fold:   BatchedBeamletScorer.end_batch (scoring/dij.py:155-174) over
 *           batches of int64 quanta maps [n_batches][n_cols][n_vox];
 *   finalize + truncate + compact: BatchedBeamletScorer.finalize
 *           (scoring/dij.py:176-191) then DijAssembler.add_block (:351-366). */
int pmc_reduce_dense(pmc_engine* engine, const int64_t* quanta, int32_t n_batches,
                     int32_t n_cols, int64_t n_vox, const double* voxel_mass,
                     const double* histories_per_batch, double* mean, double* sigma,
                     int64_t* total_quanta);
int pmc_truncate_dense(pmc_engine* engine, const double* mean, const double* sigma,
                       int32_t n_cols, int64_t n_vox, double truncation, int64_t* counts,
                       int64_t* nnz);

/* Allocation-free truncation + CSC compaction.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc (an application
 * whose device memory all comes from its own pool or allocator, or a process
 * that fixes its device footprint at start-up and forbids allocation after
 * that).  It is the truncation and compaction of pmc_truncate_dense over
 * caller-owned DEVICE buffers, with no allocation of any kind: its scratch is
 * a static device array of about 3.2 MB that every GPU loading the library
 * holds until exit.
 *   mean, sigma  [n_cols][n_vox] float64 dose means and sigmas (device)
 *   col_counts   [n_cols] int64 kept entries per column (device)
 *   out_*        [out_capacity] CSC rows, doses, sigmas (device)
 *   *nnz         the entry total (host).  When it exceeds out_capacity the
 *                call returns PMC_ERR_CAPACITY and writes neither out_* nor
 *                col_counts; retry with out_capacity >= *nnz.  On every
 *                other failure *nnz is left as it was.
 * Limits: n_cols <= 4096 and n_cols * ceil(n_vox / 4096) <= 262144; larger
 * sizes return PMC_ERR_INVALID.
 * Work runs on `stream` (a cudaStream_t, NULL = the default stream) of the
 * current device.  The call reads the entry total back to the host and
 * synchronizes `stream` (twice), so it must not be called while `stream` is
 * being captured into a CUDA graph.  The first call on a device looks up the
 * scratch array's device address and keeps it for the life of the process; a
 * cudaDeviceReset of that device invalidates the kept address, so do not call
 * this entry point after resetting the device.  All calls share the one array:
 * calls that overlap on the GPU (other threads or streams) race. */
int pmc_dij_compact_static(const double* mean, const double* sigma, int32_t n_cols,
                           int64_t n_vox, double truncation, int64_t out_capacity,
                           int64_t* col_counts, int64_t* out_indices, double* out_dose,
                           double* out_sigma, int64_t* nnz, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PYRADMC_B200_H */
