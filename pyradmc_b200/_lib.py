"""ctypes binding of ``libpmc_b200.so`` (the C-ABI of ``include/pyradmc_b200.h``).

The structures below mirror the header field for field.  Loading fails loudly:
there is no CPU fallback anywhere in this package — a missing or unbuildable
library raises, it never degrades to another implementation.
"""

from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

from pyradmc_b200.build import LIBRARY, build

PMC_OK = 0
PMC_ERR_INVALID = -1
PMC_ERR_MAJORANT = -2
PMC_ERR_QUEUE_OVERFLOW = -3
PMC_ERR_STEP_CAP = -4
PMC_ERR_CUDA = -5
PMC_ERR_OOM = -6
PMC_ERR_STATE = -7
PMC_ERR_CAPACITY = -8

PMC_PHOTON, PMC_ELECTRON, PMC_POSITRON = 0, 1, 2
PMC_SRC_PENCIL, PMC_SRC_PARALLEL, PMC_SRC_SPECTRAL, PMC_SRC_UPLOAD, PMC_SRC_PHASESPACE = 0, 1, 2, 3, 4
PMC_SRC_PHASESPACE_DEVICE = 5
PMC_SRC_SPECTRAL_MASKED = 6
PMC_BEAMLET_LATTICE, PMC_BEAMLET_SPECTRAL, PMC_BEAMLET_RECORDS, PMC_BEAMLET_UPLOAD = 0, 1, 2, 3

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)
_u8p = C.POINTER(C.c_uint8)
_d3 = C.c_double * 3


class TablesDesc(C.Structure):
    _fields_ = [
        ("n_materials", C.c_int32),
        ("n_points", C.c_int32),
        ("photon_log_e_min", C.c_double),
        ("photon_inv_dlog", C.c_double),
        ("electron_log_e_min", C.c_double),
        ("electron_inv_dlog", C.c_double),
        ("range_log_r_min", C.c_double),
        ("range_inv_dlog", C.c_double),
        ("mu_compton", _dp),
        ("mu_photo", _dp),
        ("mu_pair", _dp),
        ("mu_rayleigh", _dp),
        ("majorant", _dp),
        ("stopping_restricted", _dp),
        ("stopping_radiative", _dp),
        ("moller", _dp),
        ("csda_range", _dp),
        ("scattering_power", _dp),
        ("log_eta", _dp),
        ("restricted_range", _dp),
        ("energy_of_restricted_range", _dp),
        ("n_coherent", C.c_int32),
        ("coherent_x", _dp),
        ("coherent_cumulative", _dp),
    ]


class ScoringDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32),
        ("ny", C.c_int32),
        ("nz", C.c_int32),
        ("origin", _d3),
        ("spacing", _d3),
        ("voxel_mass", _dp),
        ("mode", C.c_int32),
        ("axis", C.c_double * 2),
        ("n_depth", C.c_int32),
        ("n_shells", C.c_int32),
        ("depth_edges", _dp),
        ("radial_edges", _dp),
    ]


class SourceDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("kind", C.c_int32),
        ("energy", C.c_double),
        ("position", _d3),
        ("direction", _d3),
        ("z0", C.c_double),
        ("x_lo", C.c_double),
        ("x_extent", C.c_double),
        ("y_lo", C.c_double),
        ("y_extent", C.c_double),
        ("n_bins", C.c_int32),
        ("edges", _dp),
        ("cdf", _dp),
        ("focal", _d3),
        ("center", _d3),
        ("u_axis", _d3),
        ("v_axis", _d3),
        ("width_u", C.c_double),
        ("width_v", C.c_double),
        ("up_kind", _ip),
        ("up_energy", _fp),
        ("up_pos", _fp),
        ("up_dir", _fp),
        ("up_weight", _fp),
        ("n_records", C.c_int64),
        ("mask", _dp),
        ("mask_n_u", C.c_int32),
        ("mask_n_v", C.c_int32),
        ("mask_center", _d3),
        ("mask_u_axis", _d3),
        ("mask_v_axis", _d3),
        ("mask_width_u", C.c_double),
        ("mask_width_v", C.c_double),
        ("stack", C.c_void_p),
        ("stack_mu", C.c_void_p),
    ]


SAMPLE_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int32, C.c_int64, C.c_int64,
                        C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float),
                        C.POINTER(C.c_float))


class BeamletRec(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("spectrum", C.c_int32),
        ("energy", C.c_double),
        ("z0", C.c_double),
        ("x_lo", C.c_double),
        ("x_extent", C.c_double),
        ("y_lo", C.c_double),
        ("y_extent", C.c_double),
        ("focal", _d3),
        ("center", _d3),
        ("u_axis", _d3),
        ("v_axis", _d3),
        ("width_u", C.c_double),
        ("width_v", C.c_double),
    ]


class BeamletDesc(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("n_beamlets", C.c_int32),
        ("energy", C.c_double),
        ("z0", C.c_double),
        ("x_lo", _dp),
        ("x_extent", _dp),
        ("y_lo", _dp),
        ("y_extent", _dp),
        ("n_bins", C.c_int32),
        ("edges", _dp),
        ("cdf", _dp),
        ("focal", _d3),
        ("u_axis", _d3),
        ("v_axis", _d3),
        ("width_u", C.c_double),
        ("width_v", C.c_double),
        ("centers", _dp),
        ("history_offsets", _lp),
        ("n_components", C.c_int32),
        ("records", C.POINTER(BeamletRec)),
        ("component_cdf", _dp),
        ("n_spectra", C.c_int32),
        ("spectrum_bins", C.POINTER(C.c_int32)),
        ("spectrum_edges", _dp),
        ("spectrum_cdf", _dp),
        ("sample", SAMPLE_FN),
        ("sample_user", C.c_void_p),
        ("stack", C.c_void_p),
        ("stack_mu", C.c_void_p),
        ("mask", _dp),
        ("mask_n_u", C.c_int32),
        ("mask_n_v", C.c_int32),
        ("mask_center", _d3),
        ("mask_u_axis", _d3),
        ("mask_v_axis", _d3),
        ("mask_width_u", C.c_double),
        ("mask_width_v", C.c_double),
    ]


class RunParams(C.Structure):
    _fields_ = [
        ("n_histories", C.c_int64),
        ("n_batches", C.c_int32),
        ("seed", C.c_uint64),
        ("pcut", C.c_double),
        ("ecut", C.c_double),
        ("transport_electrons", C.c_int32),
        ("msc_gs", C.c_int32),
        ("step_energy_fraction", C.c_double),
        ("deposit_resolution", C.c_double),
        ("dose_to_water", C.c_int32),
        ("photon_split_n", C.c_int32),
        ("truncation", C.c_double),
        ("correlated", C.c_int32),
        ("beamlet_group_size", C.c_int32),
        ("chunk_size", C.c_int64),
        ("queue_factor", C.c_int32),
        ("block_size", C.c_int32),
        ("blocks_per_sm", C.c_int32),
        ("use_graph", C.c_int32),
        ("max_steps", C.c_int64),
        ("tail_steps", C.c_int32),
        ("smem_tables", C.c_int32),
    ]


class Books(C.Structure):
    _fields_ = [
        ("deposited", C.c_int64),
        ("escaped", C.c_int64),
        ("unscored", C.c_int64),
        ("emitted", C.c_int64),
        ("majorant_violations", C.c_int64),
    ]


class Counters(C.Structure):
    _fields_ = [
        ("photon_flights", C.c_int64),
        ("photon_interactions", C.c_int64),
        ("electron_substeps", C.c_int64),
        ("deposits", C.c_int64),
        ("queue_pushes", C.c_int64),
        ("primaries", C.c_int64),
        ("rounds", C.c_int64),
        ("transport_launches", C.c_int64),
        ("reduce_launches", C.c_int64),
        ("kernel_launches", C.c_int64),
        ("transport_ms", C.c_double),
        ("reduce_ms", C.c_double),
        ("h2d_bytes_total", C.c_int64),
        ("d2h_bytes_total", C.c_int64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


# Every symbol the header declares, with its ctypes signature.
SIGNATURES: dict[str, tuple[object, list]] = {
    "pmc_abi_version": (C.c_int, []),
    "pmc_device_count": (C.c_int, []),
    "pmc_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int]),
    "pmc_destroy": (None, [C.c_void_p]),
    "pmc_last_error": (C.c_char_p, [C.c_void_p]),
    "pmc_upload_grid": (
        C.c_int,
        [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, _dp, _dp, _fp, _u8p],
    ),
    "pmc_upload_tables": (C.c_int, [C.c_void_p, C.POINTER(TablesDesc)]),
    "pmc_upload_gs": (
        C.c_int,
        [C.c_void_p, _fp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_double],
    ),
    "pmc_set_scoring": (C.c_int, [C.c_void_p, C.POINTER(ScoringDesc)]),
    "pmc_run_forward": (
        C.c_int,
        [C.c_void_p, C.POINTER(SourceDesc), C.POINTER(RunParams), _dp, _dp, C.POINTER(Books)],
    ),
    "pmc_run_dij": (
        C.c_int,
        [C.c_void_p, C.POINTER(BeamletDesc), _lp, C.POINTER(RunParams), _lp, C.POINTER(Books)],
    ),
    "pmc_dij_fetch": (C.c_int, [C.c_void_p, _lp, _lp, _dp, _dp]),
    "pmc_dij_device_view": (
        C.c_int,
        [C.c_void_p, _lp, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)],
    ),
    "pmc_get_counters": (C.c_int, [C.c_void_p, C.POINTER(Counters)]),
    "pmc_set_progress": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pmc_set_stream": (C.c_int, [C.c_void_p, C.c_void_p]),
    "pmc_reduce_dense": (
        C.c_int,
        [C.c_void_p, _lp, C.c_int32, C.c_int32, C.c_int64, _dp, _dp, _dp, _dp, _lp],
    ),
    "pmc_truncate_dense": (
        C.c_int,
        [C.c_void_p, _dp, _dp, C.c_int32, C.c_int64, C.c_double, _lp, _lp],
    ),
    "pmc_dij_compact_static": (
        C.c_int,
        [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_double, C.c_int64, C.c_void_p,
         C.c_void_p, C.c_void_p, C.c_void_p, _lp, C.c_void_p],
    ),
}

# The head pre-solve (include/pyradmc_b200_presolve.h): host arrays throughout.
_dp = C.POINTER(C.c_double)


class HeadStack(C.Structure):
    _fields_ = [
        ("n_devices", C.c_int32),
        ("origin", C.c_double * 3),
        ("rotation", C.c_double * 9),
        ("kind", _ip), ("z_top", _dp), ("z_bottom", _dp),
        ("jaw_axis", _ip), ("jaw_edge_neg", _dp), ("jaw_edge_pos", _dp), ("jaw_focused", _ip),
        ("mlc_tip_radius", _dp), ("mlc_focused_sides", _ip), ("mlc_n_pairs", _ip),
        ("mlc_edges_off", _ip), ("mlc_tips_off", _ip),
        ("leaf_edges_v", _dp), ("n_leaf_edges", C.c_int64),
        ("tips_neg", _dp), ("tips_pos", _dp), ("n_tips", C.c_int64),
    ]


class HeadMu(C.Structure):
    _fields_ = [("n_rows", C.c_int32), ("n_table", C.c_int32), ("log_energy", _dp),
                ("log_total", _dp), ("log_compton", _dp)]


class HeadParams(C.Structure):
    _fields_ = [("first_compton", C.c_int32), ("has_air", C.c_int32), ("air_row", C.c_int32),
                ("outputs_on_device", C.c_int32), ("air_z_start", C.c_double), ("air_z_end", C.c_double),
                ("exit_z", C.c_double), ("pcut", C.c_double), ("ecut", C.c_double),
                ("weight_floor", C.c_double), ("seed", C.c_uint64)]


SIGNATURES.update({
    "pmc_head_path_lengths": (C.c_int, [C.POINTER(HeadStack), C.c_int64, _fp, _fp, C.c_int32, _fp]),
    "pmc_presolve_head": (C.c_int, [C.POINTER(HeadStack), C.POINTER(HeadMu), C.POINTER(HeadParams),
                                    C.c_int64, _fp, _fp, _fp, _fp, C.c_int64, _ip, _fp, _fp, _fp, _fp,
                                    _lp, _dp]),
})

# The denoiser's entry points (include/pyradmc_b200_denoise.h); every pointer is
# a device address.
_v = C.c_void_p
_i = C.c_int
_l = C.c_int64
_f = C.c_float
SIGNATURES.update({
    "pmd_conv3d": (_i, [_v, _v, _v, _v, _i, _i, _i, _i, _i, _i, _i, _i, _v]),
    "pmd_conv3d_wgrad": (_i, [_v, _v, _v, _v, _i, _i, _i, _i, _i, _i, _i, _v]),
    "pmd_conv3d_impl": (_i, [_i]),
    "pmd_conv3d_plan": (_i, [_i, _i, _i, _i, _i, _i, _ip]),
    "pmd_conv3d_wgrad_plan": (_i, [_i, _i, _i, _i, _i, _i, _ip]),
    "pmd_conv3d_head": (_i, [_v, _v, _v, _v, _v, _v, _v, _i, _i, _i, _i, _i, _i, _i, _i, _v]),
    "pmd_gather_windows_oriented": (_i, [_v, _l, _i, _i, _i, _v, _i, _i, _i, _i, _v, _v]),
    "pmd_scatter_windows_oriented": (_i, [_v, _v, _i, _i, _i, _v, _i, _i, _i, _i, _v, _l, _v]),
    "pmd_conv3d_failures": (_i, []),
    "pmd_flip_weights": (_i, [_v, _v, _i, _i, _i, _i, _v]),
    "pmd_relu_mask": (_i, [_v, _v, _l, _v]),
    "pmd_avgpool": (_i, [_v, _v, _i, _i, _i, _i, _i, _v]),
    "pmd_avgpool_grad": (_i, [_v, _v, _i, _i, _i, _i, _i, _i, _v]),
    "pmd_upcat": (_i, [_v, _v, _v, _i, _i, _i, _i, _i, _i, _v]),
    "pmd_upcat_grad": (_i, [_v, _v, _v, _i, _i, _i, _i, _i, _i, _i, _v]),
    "pmd_head": (_i, [_v, _v, _v, _v, _v, _l, _i, _v]),
    "pmd_head_grad": (_i, [_v, _v, _v, _v, _v, _v, _l, _i, _v]),
    "pmd_loss": (_i, [_v, _v, _v, _f, _v, _v, _l, _v]),
    "pmd_adam": (_i, [_v, _v, _v, _v, _v, _l, _f, _f, _f, _f, _i, _v]),
    "pmd_pack_input": (_i, [_v, _v, _v, _v, _l, _i, _v, _v, _l, _v]),
    "pmd_csc_to_dense": (_i, [_v, _v, _v, _i, _l, _v, _v, _v]),
    "pmd_unscale": (_i, [_v, _v, _l, _v, _l, _v]),
    "pmd_csc_to_dense_f64": (_i, [_v, _v, _v, _i, _l, _v, _v]),
    "pmd_gather_windows": (_i, [_v, _l, _i, _i, _i, _v, _i, _i, _i, _i, _v, _v]),
    "pmd_scatter_windows": (_i, [_v, _v, _i, _i, _i, _v, _i, _i, _i, _i, _v, _l, _v]),
})

PROGRESS_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int64)

_lib: C.CDLL | None = None
_lock = threading.Lock()


def library_path() -> Path:
    return LIBRARY


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load (building first if needed) the shared library and bind every symbol."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if build_if_missing:
            build()
        if not LIBRARY.exists():
            raise RuntimeError(
                f"the B200 backend library {LIBRARY} is missing; build it with "
                "`python -m pyradmc_b200.build` (there is no CPU fallback)"
            )
        lib = C.CDLL(str(LIBRARY))
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
        return lib


def ptr(array, ctype):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if array is None:
        return None
    return array.ctypes.data_as(C.POINTER(ctype))
