"""``B200Engine``: the B200 backend of pyRadMC, a drop-in for ``WarpEngine``.

Same constructor fields and the same ``run`` / ``run_dij`` signatures, argument
meanings, validation messages and result types as
``pyradmc/backends/warp/engine.py`` (``WarpEngine``: :369, ``run``: :454,
``run_dij``: :948).  The work runs in ``libpmc_b200.so`` (hand-written sm_100a
CUDA behind the C-ABI of ``include/pyradmc_b200.h``); this module validates,
flattens the host data through the caller's ``CrossSectionSource``, packs the
call descriptors and wraps the results.  There is no CPU path: without the
library and a CUDA device every run raises.
"""

from __future__ import annotations

import ctypes as C
import math
import threading
from collections import deque
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from pyradmc_b200 import _lib, model

__all__ = ["B200Engine", "DIJ_TRUNCATION_RELATIVE", "DeviceDij", "ECUT_MEV", "PCUT_MEV",
           "column_shards", "merge_shards"]

ECUT_MEV = 0.200  # pyradmc/__init__.py:22
PCUT_MEV = 0.050  # pyradmc/__init__.py:25
DIJ_TRUNCATION_RELATIVE = 1.0e-3  # pyradmc/__init__.py:28
ENERGY_QUANTUM_MEV = 1.0e-9  # kernels.py:96
_E_MAX_MARGIN = 1.0 + 1.0e-6  # engine.py:80
GS_STEP_ENERGY_FRACTION = 0.20  # transport/electron.py:85
STEP_ENERGY_FRACTION = 0.05  # transport/electron.py:73
VERSION = "0.2.1"  # the pyRadMC release whose API this backend mirrors


def default_step_energy_fraction(msc_model: str) -> float:
    """transport/electron.py:97 — the per-model validated substep fraction."""
    return GS_STEP_ENERGY_FRACTION if msc_model == "gs" else STEP_ENERGY_FRACTION


def _validate_msc_model(msc_model: str) -> int:
    if msc_model not in ("gaussian", "gs"):
        raise ValueError(f"unknown msc_model {msc_model!r}; expected 'gaussian' or 'gs'")
    return 1 if msc_model == "gs" else 0


def validate_scoring_mode(scoring_mode: str, transport_electrons: bool) -> bool:
    """scoring/dose_to_water.py:48 — True selects dose-to-water."""
    if scoring_mode not in ("dose_to_medium", "dose_to_water"):
        raise ValueError(
            f"unknown scoring_mode {scoring_mode!r}; expected 'dose_to_medium' or 'dose_to_water'"
        )
    if scoring_mode == "dose_to_water" and not transport_electrons:
        raise ValueError(
            "dose_to_water requires electron transport: KERMA mode deposits carry no "
            "electron to evaluate the stopping-power ratio on (it would need "
            "mass-energy-absorption ratios instead)"
        )
    return scoring_mode == "dose_to_water"


def _result_types():
    """pyRadMC's own result classes when importable (a true drop-in), else the mirror."""
    try:
        from pyradmc.backends.results import RunProvenance, TransportResult
        from pyradmc.scoring.dij import DijResult

        return RunProvenance, TransportResult, DijResult
    except ImportError:
        return model.RunProvenance, model.TransportResult, model.DijResult


def _progress_emitter(progress, total):
    try:
        from pyradmc.progress import ProgressEmitter

        return ProgressEmitter(progress, total)
    except ImportError:
        return model.ProgressEmitter(progress, total)


def _type_name(obj) -> str:
    return type(obj).__name__


class NativeError(RuntimeError):
    """A failure reported by the C-ABI that has no reference exception type."""


def _raise_for(code: int, message: str) -> None:
    if code == _lib.PMC_OK:
        return
    if code == _lib.PMC_ERR_INVALID:
        raise ValueError(message)
    if code in (_lib.PMC_ERR_MAJORANT, _lib.PMC_ERR_QUEUE_OVERFLOW, _lib.PMC_ERR_STEP_CAP):
        raise RuntimeError(message)
    if code == _lib.PMC_ERR_OOM:
        raise MemoryError(message)
    raise NativeError(f"B200 backend error {code}: {message}")


class _Native:
    """One native engine (one CUDA device); calls are serialized by a lock."""

    def __init__(self, device: str) -> None:
        if not device.startswith("cuda"):
            raise ValueError(
                f"the B200 backend runs on CUDA devices only, got device={device!r} "
                "(there is no CPU path)"
            )
        ordinal = int(device.split(":")[1]) if ":" in device else 0
        self.lib = _lib.load()
        if self.lib.pmc_device_count() <= ordinal:
            raise RuntimeError(f"no CUDA device {device!r} visible to the B200 backend")
        handle = C.c_void_p()
        code = self.lib.pmc_create(C.byref(handle), ordinal)
        if code != _lib.PMC_OK:
            raise NativeError(f"pmc_create failed with code {code} on {device}")
        self.handle = handle
        self.device = device
        self.lock = threading.Lock()
        self.grid_key = None
        self.table_key = None
        self.gs_key = None
        self.scoring_key = None
        self._keep: list = []

    def check(self, code: int) -> None:
        if code != _lib.PMC_OK:
            msg = self.lib.pmc_last_error(self.handle)
            _raise_for(code, msg.decode() if msg else "")

    def __del__(self) -> None:
        handle = getattr(self, "handle", None)
        if handle is not None and handle.value:
            try:
                self.lib.pmc_destroy(handle)
            except Exception:
                pass
            self.handle = None


@dataclass
class DeviceDij:
    """A Dij left on the device by :meth:`B200Engine.run_dij_device`.

    ``indptr`` is host memory; ``indices`` (int64), ``dose`` and ``sigma``
    (float64) are device addresses of ``nnz`` entries owned by the engine and
    valid until its next run.
    """

    n_beamlets: int
    nnz: int
    indptr: np.ndarray
    indices: int
    dose: int
    sigma: int
    books: tuple
    grid_shape: tuple = ()
    counts: np.ndarray | None = None
    n_batches: int = 0
    device: str = "cuda:0"


def _pinned_array(n: int, dtype) -> np.ndarray:
    """A numpy array in page-locked host memory (torch's caching host allocator,
    so repeated Dijs reuse the blocks): the CSC readback then runs at the full
    host link rate instead of through the driver's pageable staging.  Plain
    numpy memory when pinning is unavailable."""
    if n >= 1 << 16:
        try:
            import torch

            tdt = {np.dtype(np.int64): torch.int64, np.dtype(np.float64): torch.float64,
                   np.dtype(np.float32): torch.float32, np.dtype(np.uint8): torch.uint8}[np.dtype(dtype)]
            return torch.empty(int(n), dtype=tdt, pin_memory=True).numpy()
        except Exception:
            pass
    return np.empty(n, dtype=dtype)


def _pinned_copy(a, dtype) -> np.ndarray:
    """`a` converted to a contiguous `dtype` array in page-locked host memory
    (same shape): the arrays the engine uploads again on every drop of the
    device copies then cross the bus by DMA at the full link rate."""
    a = np.asarray(a)
    out = _pinned_array(a.size, dtype).reshape(a.shape)
    np.copyto(out, a, casting="unsafe")
    return out


def column_shards(counts, world: int) -> list[tuple[int, int]]:
    """Contiguous Dij column ranges, one per rank, with near-equal history totals
    (some empty when there are more ranks than columns)."""
    c = np.asarray(counts, dtype=np.int64)
    if world < 1:
        raise ValueError(f"need at least one rank, got {world}")
    cum = np.cumsum(c)
    total = int(cum[-1]) if c.size else 0
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        j = int(np.searchsorted(cum, target))  # first column whose running total reaches target
        if j < c.size and j > 0 and abs(cum[j - 1] - target) <= abs(cum[j] - target):
            j -= 1
        bounds.append(min(max(bounds[-1], j + 1), c.size))
    bounds.append(int(c.size))
    return list(zip(bounds[:-1], bounds[1:]))


def merge_shards(parts):
    """One Dij from ``(DijResult, (first, stop))`` shards that cover every column
    once (in any order): the CSC concatenated in column order, energies summed."""
    parts = sorted(parts, key=lambda p: p[1][0])
    if not parts:
        raise ValueError("no shards to merge")
    expect = 0
    for _, (a, b) in parts:
        if a != expect or b < a:
            raise ValueError(f"shards do not tile the columns: expected {expect}, got ({a}, {b})")
        expect = b
    first = parts[0][0]
    indptr = [np.zeros(1, dtype=np.int64)]
    base = 0
    for dij, _ in parts:
        indptr.append(np.asarray(dij.indptr[1:], dtype=np.int64) + base)
        base += int(dij.indptr[-1])
    _, _, DijResult = _result_types()
    real = [d for d, (a, b) in parts if b > a]
    return DijResult(
        grid_shape=first.grid_shape, n_beamlets=expect,
        n_histories_per_beamlet=max(int(d.n_histories_per_beamlet) for d in real),
        n_batches=first.n_batches, truncation=first.truncation,
        indptr=np.concatenate(indptr),
        indices=np.concatenate([np.asarray(d.indices, dtype=np.int64) for d, _ in parts]),
        dose=np.concatenate([np.asarray(d.dose) for d, _ in parts]),
        sigma=np.concatenate([np.asarray(d.sigma) for d, _ in parts]),
        energy_emitted=sum(float(d.energy_emitted) for d in real),
        energy_deposited=sum(float(d.energy_deposited) for d in real),
        energy_escaped=sum(float(d.energy_escaped) for d in real),
        energy_unscored=sum(float(d.energy_unscored) for d in real),
        correlated=first.correlated, scoring_mode=first.scoring_mode,
        provenance=first.provenance)


# ---- beamlet sources beyond the two built-in generators ------------------------------
_IN_KERNEL_BEAMLETS = ("BeamletGridSource", "SpectralBeamletSource")


def _simple_records(src, spectra: list) -> list | None:
    """Per-beamlet record tuples of a built-in beamlet source (None otherwise);
    `spectra` collects the distinct spectra the fans draw from."""
    name = _type_name(src)
    if name == "BeamletGridSource":
        out = []
        for j in range(int(src.n_beamlets)):
            x0, x1, y0, y1 = src.beamlet_bounds(j)
            out.append(("lattice", float(src.energy), float(src.z), x0, x1 - x0, y0, y1 - y0))
        return out
    if name == "SpectralBeamletSource":
        k = next((i for i, sp in enumerate(spectra) if sp is src.spectrum), None)
        if k is None:
            spectra.append(src.spectrum)
            k = len(spectra) - 1
        return [("fan", k, tuple(src.focal_point), tuple(c), tuple(src.u_axis), tuple(src.v_axis),
                 float(src.width_u), float(src.width_v)) for c in src.centers]
    return None


def _records_plan(source, spectra: list | None = None):
    """(rows, component cdf or None, spectra) when every beamlet of `source`
    is a built-in lattice rectangle or fan, or a fixed mixture of them
    (CompositeBeamletSource); a ConcatenatedBeamletSource joins such parts when
    they share one mixture.  None when the source needs host pre-sampling."""
    spectra = [] if spectra is None else spectra
    name = _type_name(source)
    if name in _IN_KERNEL_BEAMLETS:
        return [[r] for r in _simple_records(source, spectra)], None, spectra
    if name == "CompositeBeamletSource":
        comps = [_simple_records(c, spectra) for c in source._sources]
        if any(c is None for c in comps):
            return None
        n = int(source.n_beamlets)
        return [[c[j] for c in comps] for j in range(n)], np.asarray(source._cdf, float), spectra
    if name == "ConcatenatedBeamletSource":
        rows, cdf = [], None
        for part in source.sources:
            plan = _records_plan(part, spectra)
            if plan is None:
                return None
            part_rows, part_cdf, _ = plan
            if rows and (len(part_rows[0]) != len(rows[0]) or
                         (part_cdf is None) != (cdf is None) or
                         (cdf is not None and not np.array_equal(cdf, part_cdf))):
                return None  # differently mixed parts: pre-sampled instead
            rows += part_rows
            cdf = part_cdf
        return rows, cdf, spectra
    return None


def _fill_general_desc(desc, source, records, sl: slice, seed: int, keep: list) -> None:
    """PMC_BEAMLET_RECORDS for `records`, else PMC_BEAMLET_UPLOAD through the
    source's ``sample_beamlet_batch`` (the Warp engine's pre-sampling route,
    engine.py:3224-3335), for the columns `sl` of the call."""
    if records is not None:
        rows, cdf, spectra = records
        rows = rows[sl]
        nc = len(rows[0])
        arr = (_lib.BeamletRec * (len(rows) * nc))()
        for i, row in enumerate(rows):
            for c, r in enumerate(row):
                rec = arr[i * nc + c]
                if r[0] == "lattice":
                    rec.type = _lib.PMC_BEAMLET_LATTICE
                    rec.energy, rec.z0, rec.x_lo, rec.x_extent, rec.y_lo, rec.y_extent = r[1:]
                else:
                    rec.type = _lib.PMC_BEAMLET_SPECTRAL
                    rec.spectrum = r[1]
                    rec.focal[:], rec.center[:], rec.u_axis[:], rec.v_axis[:] = r[2:6]
                    rec.width_u, rec.width_v = r[6], r[7]
        bins = np.array([int(np.asarray(sp.cdf).size) for sp in spectra] or [0], dtype=np.int32)
        edges = np.ascontiguousarray(np.concatenate([np.asarray(sp.edges, float) for sp in spectra])
                                     if spectra else np.zeros(1))
        cdfs = np.ascontiguousarray(np.concatenate([np.asarray(sp.cdf, float) for sp in spectra])
                                    if spectra else np.zeros(1))
        comp = np.ascontiguousarray(cdf if cdf is not None else np.ones(1))
        keep += [arr, bins, edges, cdfs, comp]
        desc.type = _lib.PMC_BEAMLET_RECORDS
        desc.n_components = nc
        desc.records = C.cast(arr, C.POINTER(_lib.BeamletRec))
        desc.component_cdf = _lib.ptr(comp, C.c_double)
        desc.n_spectra = len(spectra)
        desc.spectrum_bins = _lib.ptr(bins, C.c_int32)
        desc.spectrum_edges = _lib.ptr(edges, C.c_double)
        desc.spectrum_cdf = _lib.ptr(cdfs, C.c_double)
        return
    first = sl.start or 0
    errors: list = []

    def sample(_user, beamlet, key_offset, n, energy, position, direction, weight):
        try:
            cols = source.sample_beamlet_batch(seed, int(key_offset), int(n), first + int(beamlet))
            np.ctypeslib.as_array(energy, (n,))[:] = cols["energy"]
            np.ctypeslib.as_array(weight, (n,))[:] = cols["weight"]
            pos = np.ctypeslib.as_array(position, (n, 3))
            dirs = np.ctypeslib.as_array(direction, (n, 3))
            for k, (a, b) in enumerate((("x", "ux"), ("y", "uy"), ("z", "uz"))):
                pos[:, k] = cols[a]
                dirs[:, k] = cols[b]
            return 0
        except Exception as exc:  # reported after the call returns
            errors.append(exc)
            return 1

    callback = _lib.SAMPLE_FN(sample)
    keep += [callback, errors]
    desc.type = _lib.PMC_BEAMLET_UPLOAD
    desc.sample = callback


def _forward_in_kernel(source) -> bool:
    name = _type_name(source)
    if name in ("PencilBeamSource", "ParallelBeamSource", "SpectralBeamSource"):
        return True
    return _collimated_inner(source, _forward_in_kernel) is not None


def _attach_stack(desc, source, keep: list):
    """Point `desc` (a pmc_source_desc or pmc_beamlet_desc) at the stack
    transmission of a collimated `source`; the structures go into `keep`."""
    from .collimation import stack_transmission_tables

    _, stack, log_energy, log_total = stack_transmission_tables(source)
    hs = stack.to_c()
    arrs = [np.ascontiguousarray(log_energy, dtype=np.float64),
            np.ascontiguousarray(log_total, dtype=np.float64)]
    mu = _lib.HeadMu(n_rows=int(arrs[1].shape[0]), n_table=int(arrs[0].size),
                     log_energy=_lib.ptr(arrs[0], C.c_double), log_total=_lib.ptr(arrs[1], C.c_double),
                     log_compton=_lib.ptr(arrs[1], C.c_double))
    keep += [stack, hs, mu, arrs]
    desc.stack = C.cast(C.pointer(hs), C.c_void_p)
    desc.stack_mu = C.cast(C.pointer(mu), C.c_void_p)


_MASKS = ("TransmissionMaskSource", "TransmissionMaskBeamletSource")


def _wrapped(source):
    """The source a weight wrapper wraps (pyRadMC's beamlet wrappers keep it
    private, geometry/collimation.py:1126-1128)."""
    return getattr(source, "inner", None) or getattr(source, "_inner", None)


def _mask_params(source):
    """(mask, centre, width_u, width_v, u_axis, v_axis) of a mask wrapper: its
    properties, or the _MaskTransmission model of pyRadMC's beamlet wrapper
    (geometry/collimation.py:1024-1029), which exposes none."""
    if hasattr(source, "mask"):
        return (source.mask, source.plane_center, source.width_u, source.width_v, source.u_axis,
                source.v_axis)
    m = source._model
    return m._mask, m._center, m._widths[0], m._widths[1], m._u_axis, m._v_axis


def _collimated_inner(source, in_kernel):
    """The inner source of a collimated or masked `source` when
    `in_kernel(inner)` says the engine generates it on the device, else None."""
    from .collimation import stack_transmission_tables

    if _type_name(source) in _MASKS:
        inner = _wrapped(source)
        return inner if inner is not None and in_kernel(inner) else None
    found = stack_transmission_tables(source)
    return found[0] if found is not None and in_kernel(found[0]) else None


def _beamlets_in_kernel(source) -> bool:
    name = _type_name(source)
    if name in ("BeamletGridSource", "SpectralBeamletSource") or _records_plan(source) is not None:
        return True
    return _collimated_inner(source, _beamlets_in_kernel) is not None


def _attach_mask(desc, source, keep: list) -> None:
    """Point `desc` at the transmission mask of a TransmissionMask(Beamlet)Source
    (geometry/collimation.py:987-1080, 1205-1284)."""
    if desc.mask:
        raise ValueError("one transmission mask per source: nested masks are not supported")
    values, center, width_u, width_v, u_axis, v_axis = _mask_params(source)
    mask = np.ascontiguousarray(values, dtype=np.float64)
    if mask.ndim != 2:
        raise ValueError(f"the mask must be a non-empty 2D array, got shape {mask.shape}")
    keep.append(mask)
    desc.mask = _lib.ptr(mask, C.c_double)
    desc.mask_n_u, desc.mask_n_v = (int(n) for n in mask.shape)
    desc.mask_center[:] = [float(c) for c in center]
    desc.mask_u_axis[:] = [float(c) for c in u_axis]
    desc.mask_v_axis[:] = [float(c) for c in v_axis]
    desc.mask_width_u = float(width_u)
    desc.mask_width_v = float(width_v)


def _attach_weights(desc, source, keep: list) -> None:
    if _type_name(source) in _MASKS:
        _attach_mask(desc, source, keep)
    else:
        _attach_stack(desc, source, keep)


def beamlet_arrays(source):
    """(per-beamlet arrays of a built-in generator or None, records plan or None):
    the host-side flattening of a beamlet source for ``pmc_run_dij``."""
    inner = _collimated_inner(source, _beamlets_in_kernel)
    if inner is not None:
        return beamlet_arrays(inner)
    name = _type_name(source)
    n = int(source.n_beamlets)
    if name == "BeamletGridSource":
        bounds = np.array([source.beamlet_bounds(j) for j in range(n)], dtype=np.float64)
        return dict(x_lo=bounds[:, 0], x_extent=bounds[:, 1] - bounds[:, 0],
                    y_lo=bounds[:, 2], y_extent=bounds[:, 3] - bounds[:, 2]), None
    if name == "SpectralBeamletSource":
        return dict(centers=np.asarray(source.centers, dtype=np.float64).reshape(n, 3)), None
    records = _records_plan(source)
    if records is None and not hasattr(source, "sample_beamlet_batch"):
        raise ValueError(f"unsupported beamlet source type {name}")
    return None, records


def beamlet_descriptor(source, sl: slice, seed: int, keep: list, per=None, records=None):
    """The ``pmc_beamlet_desc`` of columns `sl` of `source` (the arrays it
    points to are appended to `keep`, which must outlive the call)."""
    inner = _collimated_inner(source, _beamlets_in_kernel)
    if inner is not None:  # the inner generator, its primaries weighted by the stack or mask
        desc = beamlet_descriptor(inner, sl, seed, keep, per, records)
        _attach_weights(desc, source, keep)
        return desc
    if per is None and records is None:
        per, records = beamlet_arrays(source)
    desc = _lib.BeamletDesc(n_beamlets=sl.stop - sl.start)
    name = _type_name(source)
    if per is None:
        _fill_general_desc(desc, source, records, sl, seed, keep)
    elif name == "BeamletGridSource":
        desc.type = _lib.PMC_BEAMLET_LATTICE
        desc.energy = float(source.energy)
        desc.z0 = float(source.z)
        for key in ("x_lo", "x_extent", "y_lo", "y_extent"):
            arr = np.ascontiguousarray(per[key][sl])
            keep.append(arr)
            setattr(desc, key, _lib.ptr(arr, C.c_double))
    else:
        spectrum = source.spectrum
        edges = np.ascontiguousarray(spectrum.edges, dtype=np.float64)
        cdf = np.ascontiguousarray(spectrum.cdf, dtype=np.float64)
        centers = np.ascontiguousarray(per["centers"][sl])
        keep += [edges, cdf, centers]
        desc.type = _lib.PMC_BEAMLET_SPECTRAL
        desc.n_bins = int(cdf.size)
        desc.edges = _lib.ptr(edges, C.c_double)
        desc.cdf = _lib.ptr(cdf, C.c_double)
        desc.focal[:] = [float(v) for v in source.focal_point]
        desc.u_axis[:] = [float(v) for v in source.u_axis]
        desc.v_axis[:] = [float(v) for v in source.v_axis]
        desc.width_u = float(source.width_u)
        desc.width_v = float(source.width_v)
        desc.centers = _lib.ptr(centers, C.c_double)
    return desc


def _device_dij(native: "_Native", n_cols: int, nnz: int, books) -> DeviceDij:
    indptr = np.zeros(n_cols + 1, dtype=np.int64)
    ptrs = [C.c_void_p() for _ in range(3)]
    native.check(native.lib.pmc_dij_device_view(native.handle, _lib.ptr(indptr, C.c_int64),
                                                *(C.byref(p) for p in ptrs)))
    return DeviceDij(n_beamlets=n_cols, nnz=nnz, indptr=indptr,
                     indices=ptrs[0].value or 0, dose=ptrs[1].value or 0, sigma=ptrs[2].value or 0,
                     books=(books.deposited, books.escaped, books.unscored, books.emitted))


@dataclass(frozen=True)
class B200Engine:
    """The B200 Monte Carlo dose engine over a voxel grid.

    Parameters
    ----------
    grid, cross_sections
        As in ``WarpEngine``: a ``VoxelGrid`` and a ``CrossSectionSource``
        (pyRadMC's own, or this package's :class:`~pyradmc_b200.model.VoxelGrid`
        and :class:`~pyradmc_b200.model.AnalyticWaterTables` mirrors).
    device
        ``"cuda:N"``.
    chunk_size
        Fresh primaries admitted per transport round (``None``: four per resident
        transport thread).  Bit-inert: streams are pure functions of
        ``(seed, history)`` and scoring is integer, so it only trades memory
        for occupancy.
    queue_factor
        Queue slots per admitted primary; overflow raises, never drops.
    block_size, blocks_per_sm, use_graph
        Launch shape of the persistent transport kernels and whether each batch
        drains inside one CUDA graph (a conditional WHILE node) or under a host
        loop.  All bit-inert.
    tail_steps
        Steps a particle may still take once its transport round has no input
        left before it is parked, state and all, for the next round (``None``:
        the library default; a negative value never parks).  Bit-inert.
    smem_tables
        Stage the photon and electron table rows in each block's shared memory
        (True), read them through L1 (False) or let the library decide (None).
        Bit-inert: the same values either way.
    """

    grid: object
    cross_sections: object
    device: str = "cuda:0"
    chunk_size: int | None = None
    queue_factor: int = 16
    block_size: int | None = None
    blocks_per_sm: int | None = None
    use_graph: bool = True
    max_steps: int | None = None
    tail_steps: int | None = None
    smem_tables: bool | None = None
    _natives: dict = field(default_factory=dict, init=False, repr=False, compare=False)
    _table_cache: dict = field(default_factory=dict, init=False, repr=False, compare=False)
    _host_arrays: dict = field(default_factory=dict, init=False, repr=False, compare=False)
    _streams: dict = field(default_factory=dict, init=False, repr=False, compare=False)
    _table_cache_lock: threading.Lock = field(
        default_factory=threading.Lock, init=False, repr=False, compare=False
    )

    # ---- host data ------------------------------------------------------------
    def _native(self, device: str | None = None) -> _Native:
        key = device or self.device
        with self._table_cache_lock:
            native = self._natives.get(key)
            if native is None:
                native = _Native(key)
                stream = self._streams.get(key)
                if stream:
                    native.check(native.lib.pmc_set_stream(native.handle, C.c_void_p(stream)))
                self._natives[key] = native
        return native

    def _grid_arrays(self):
        """The transport grid as the C-ABI takes it (float32 density, uint8
        material), converted once per grid object, like the uploads."""
        key = ("grid", id(self.grid))
        hit = self._host_arrays.get(key)
        if hit is None:
            hit = (_pinned_copy(self.grid.density, np.float32),
                   _pinned_copy(np.asarray(self.grid.material).astype(np.uint8), np.uint8))
            self._host_arrays[key] = hit
        return hit

    def _default_mass(self):
        """Voxel masses of the default scoring grid (density x volume, float64,
        ScoringGrid.for_grid's arithmetic), computed once per grid object."""
        key = ("mass", id(self.grid))
        hit = self._host_arrays.get(key)
        if hit is None:
            hit = _pinned_copy(np.asarray(model.ScoringGrid.for_grid(self.grid).voxel_mass).reshape(-1),
                               np.float64)
            self._host_arrays[key] = hit
        return hit

    def _host_tables(self, e_max: float, pcut: float, ecut: float):
        key = (ecut, pcut, e_max)
        with self._table_cache_lock:
            host = self._table_cache.get(key)
            if host is None:
                host = self.cross_sections.build_tables(
                    ecut=ecut, pcut=pcut, e_max=e_max * _E_MAX_MARGIN
                )
                self._table_cache[key] = host
        return host

    def _gs_host(self, host, ecut: float, e_max: float):
        """The GS node grid, built once per (ecut, e_max) before any launch."""
        key = ("gs", ecut, e_max)
        with self._table_cache_lock:
            gs = self._table_cache.get(key)
            if gs is None:
                present = np.unique(np.asarray(self.grid.material)).astype(int).tolist()
                if hasattr(self.cross_sections, "gs_grid_for"):
                    gs = self.cross_sections.gs_grid_for(host, present)
                else:
                    from pyradmc.data.goudsmit_saunderson import (
                        build_gs_grid,
                        gs_window_from_tables,
                    )

                    gs = build_gs_grid(*gs_window_from_tables(host, present))
                self._table_cache[key] = gs
        return gs

    def _upload(self, native: _Native, e_max: float, pcut: float, ecut: float, with_gs: bool,
                scoring) -> None:
        lib = native.lib
        grid = self.grid
        gkey = id(grid)
        if native.grid_key != gkey:
            if getattr(self.cross_sections, "n_materials", 1) > 256:
                raise ValueError(
                    "the B200 backend addresses at most 256 materials (uint8 voxel map); "
                    f"this source declares {self.cross_sections.n_materials}"
                )
            shape = tuple(int(n) for n in grid.shape)
            density, material = self._grid_arrays()
            origin = np.asarray(grid.origin, dtype=np.float64)
            spacing = np.asarray(grid.spacing, dtype=np.float64)
            native.check(lib.pmc_upload_grid(
                native.handle, shape[0], shape[1], shape[2], _lib.ptr(origin, C.c_double),
                _lib.ptr(spacing, C.c_double), _lib.ptr(density, C.c_float),
                _lib.ptr(material, C.c_uint8)))
            native.grid_key = gkey
            native.scoring_key = None
        host = self._host_tables(e_max, pcut, ecut)
        tkey = (id(host), ecut, pcut, e_max)
        if native.table_key != tkey:
            arrays = {}
            for name in ("mu_compton", "mu_photo", "mu_pair", "mu_rayleigh", "majorant",
                         "stopping_restricted", "stopping_radiative", "moller", "csda_range",
                         "scattering_power", "log_eta", "restricted_range",
                         "energy_of_restricted_range", "coherent_x", "coherent_cumulative"):
                arrays[name] = np.ascontiguousarray(np.asarray(getattr(host, name)), dtype=np.float64)
            n_mat = arrays["mu_compton"].shape[0]
            desc = _lib.TablesDesc(
                n_materials=n_mat,
                n_points=int(host.n_points),
                photon_log_e_min=float(host.photon_log_e_min),
                photon_inv_dlog=float(host.photon_inv_dlog),
                electron_log_e_min=float(host.electron_log_e_min),
                electron_inv_dlog=float(host.electron_inv_dlog),
                range_log_r_min=float(host.range_log_r_min),
                range_inv_dlog=float(host.range_inv_dlog),
                n_coherent=int(host.n_coherent),
            )
            for name, arr in arrays.items():
                setattr(desc, name, _lib.ptr(arr, C.c_double))
            native.check(lib.pmc_upload_tables(native.handle, C.byref(desc)))
            native.table_key = tkey
        if with_gs:
            gs = self._gs_host(host, ecut, e_max)
            gkey2 = id(gs)
            if native.gs_key != gkey2:
                vkey = ("gs_values", gkey2)
                values = self._host_arrays.get(vkey)
                if values is None:  # converted once per GS grid, in page-locked memory
                    values = self._host_arrays[vkey] = _pinned_copy(gs.values, np.float32)
                n_eta, n_t2, n_u = values.shape
                native.check(lib.pmc_upload_gs(native.handle, _lib.ptr(values, C.c_float),
                                               int(gs.ix0), int(gs.iy0), n_eta, n_t2, n_u,
                                               float(gs.bins_per_log)))
                native.gs_key = gkey2
        skey = id(scoring) if scoring is not None else ("default", gkey)
        if native.scoring_key != skey:
            if scoring is None:  # the transport grid itself (ScoringGrid.for_grid)
                mass = self._default_mass()
            else:
                mass = np.ascontiguousarray(np.asarray(scoring.voxel_mass).reshape(-1), dtype=np.float64)
            if scoring is not None and _type_name(scoring) == "CylindricalScoringGrid":  # scoring/cylinder.py:172
                depth = np.ascontiguousarray(scoring.depth_edges, dtype=np.float64)
                radial = np.ascontiguousarray(scoring.radial_edges, dtype=np.float64)
                native._keep = [mass, depth, radial]
                sdesc = _lib.ScoringDesc(mode=1, n_depth=depth.size - 1, n_shells=radial.size - 1)
                sdesc.axis[:] = [float(v) for v in scoring.axis]
                sdesc.depth_edges = _lib.ptr(depth, C.c_double)
                sdesc.radial_edges = _lib.ptr(radial, C.c_double)
            else:
                box = grid if scoring is None else scoring
                sdesc = _lib.ScoringDesc(nx=int(box.shape[0]), ny=int(box.shape[1]),
                                         nz=int(box.shape[2]))
                sdesc.origin[:] = [float(v) for v in box.origin]
                sdesc.spacing[:] = [float(v) for v in box.spacing]
            sdesc.voxel_mass = _lib.ptr(mass, C.c_double)
            native.check(lib.pmc_set_scoring(native.handle, C.byref(sdesc)))
            native.scoring_key = skey

    def _params(self, *, n_histories=0, n_batches, seed, pcut, ecut, transport_electrons,
                msc_gs, step_energy_fraction, deposit_resolution, dose_to_water,
                truncation=0.0, correlated=True, beamlet_group_size=None) -> _lib.RunParams:
        return _lib.RunParams(
            n_histories=int(n_histories),
            n_batches=int(n_batches),
            seed=int(seed) & 0xFFFFFFFFFFFFFFFF,
            pcut=float(pcut),
            ecut=float(ecut),
            transport_electrons=1 if transport_electrons else 0,
            msc_gs=msc_gs,
            step_energy_fraction=float(step_energy_fraction),
            deposit_resolution=float(deposit_resolution),
            dose_to_water=dose_to_water,
            photon_split_n=1,
            truncation=float(truncation),
            correlated=1 if correlated else 0,
            beamlet_group_size=int(beamlet_group_size or 0),
            chunk_size=int(self.chunk_size or 0),
            queue_factor=int(self.queue_factor),
            block_size=int(self.block_size or 0),
            blocks_per_sm=int(self.blocks_per_sm or 0),
            use_graph=1 if self.use_graph else 0,
            max_steps=int(self.max_steps or 0),
            tail_steps=int(self.tail_steps or 0),
            smem_tables=0 if self.smem_tables is None else (1 if self.smem_tables else -1),
        )

    def _provenance(self, seed, pcut, ecut, msc_model, step_energy_fraction,
                    deposit_resolution_cm, devices=None):
        RunProvenance, _, _ = _result_types()
        return RunProvenance(
            version=VERSION,
            backend="b200",
            device="+".join(devices) if devices else self.device,
            seed=seed,
            pcut_mev=pcut,
            ecut_mev=ecut,
            msc_model=msc_model,
            step_energy_fraction=step_energy_fraction,
            cross_sections=getattr(self.cross_sections, "provenance", type(self.cross_sections).__name__),
            deposit_resolution_cm=deposit_resolution_cm,
        )

    def use_stream(self, stream: int | None, device: str | None = None) -> None:
        """Run this engine's work on the caller's CUDA stream (a ``cudaStream_t``
        as an int, e.g. ``torch.cuda.current_stream().cuda_stream``); None
        restores the engine's own stream."""
        native = self._native(device)
        self._streams[device or self.device] = stream or 0
        with native.lock:
            native.check(native.lib.pmc_set_stream(native.handle, C.c_void_p(stream or 0)))

    def release_device_memory(self, device: str | None = None) -> None:
        """Free every device buffer of this engine on ``device`` (all devices
        when None): maps, queues, tables, the last Dij's CSC (a ``DeviceDij``
        of it is no longer valid).  The next call allocates and uploads again,
        on the stream set by :meth:`use_stream`."""
        with self._table_cache_lock:
            keys = [k for k in self._natives if device is None or k == device]
            natives = [self._natives.pop(k) for k in keys]
        for native in natives:
            with native.lock:
                native.__del__()

    def drop_uploads(self, device: str | None = None) -> None:
        """Forget what is resident, so the next call uploads grid, tables, GS
        grid and scoring geometry again (an end-to-end timing from host data)."""
        native = self._native(device)
        with native.lock:
            native.grid_key = native.table_key = native.gs_key = native.scoring_key = None

    def last_counters(self, device: str | None = None) -> dict:
        """Device event counters and device times of the last call on ``device``."""
        native = self._native(device)
        c = _lib.Counters()
        native.check(native.lib.pmc_get_counters(native.handle, C.byref(c)))
        return c.as_dict()

    # ---- run ----------------------------------------------------------------------
    def run(
        self,
        source,
        n_histories: int,
        n_batches: int,
        seed: int,
        pcut: float = PCUT_MEV,
        ecut: float = ECUT_MEV,
        transport_electrons: bool = True,
        primary_kind: str = "photon",
        scoring_grid=None,
        scoring_mode: str = "dose_to_medium",
        step_energy_fraction: float | None = None,
        deposit_resolution_cm: float | None = None,
        msc_model: str = "gs",
        progress=None,
        concurrent_batches: int = 1,
    ):
        """Transport ``n_histories`` primaries; the contract of ``WarpEngine.run``.

        ``concurrent_batches`` is accepted for API compatibility and is inert:
        a batch already drains inside one device-side graph with no host gaps
        to hide, and the float64 fold stays in batch order either way.
        """
        if n_histories < 1:
            raise ValueError(f"need at least one history, got {n_histories}")
        if concurrent_batches < 1:
            raise ValueError(f"need at least one lane, got concurrent_batches={concurrent_batches}")
        if n_batches < 1:
            raise ValueError(f"need at least one batch, got {n_batches}")
        if n_histories % n_batches != 0:
            raise ValueError(
                f"n_histories={n_histories} not divisible by n_batches={n_batches}; "
                "unequal batches would weight batch means inconsistently"
            )
        wrappers = []  # stack and mask wrappers around an in-kernel source, outermost first
        while (inner := _collimated_inner(source, _forward_in_kernel)) is not None:
            wrappers.append(source)
            source = inner
        name = _type_name(source)
        in_kernel = name in ("PencilBeamSource", "ParallelBeamSource")
        if in_kernel and primary_kind not in ("photon", "electron"):
            raise ValueError(f"unknown primary_kind {primary_kind!r}")
        dose_to_water = 1 if validate_scoring_mode(scoring_mode, transport_electrons) else 0
        msc_gs = _validate_msc_model(msc_model)
        if step_energy_fraction is None:
            step_energy_fraction = default_step_energy_fraction(msc_model)
        if deposit_resolution_cm is not None and deposit_resolution_cm <= 0.0:
            raise ValueError(f"deposit resolution must be positive, got {deposit_resolution_cm}")
        deposit_resolution = 0.0 if deposit_resolution_cm is None else deposit_resolution_cm

        src = _lib.SourceDesc()
        keep = []
        energy_emitted = None
        if name == "PencilBeamSource":
            src.type = _lib.PMC_SRC_PENCIL
            src.kind = _lib.PMC_PHOTON if primary_kind == "photon" else _lib.PMC_ELECTRON
            src.energy = float(source.energy)
            src.position[:] = [float(v) for v in source.position]
            src.direction[:] = [float(v) for v in source.direction]
            energy_emitted = n_histories * source.max_energy
        elif name == "ParallelBeamSource":
            src.type = _lib.PMC_SRC_PARALLEL
            src.kind = _lib.PMC_PHOTON if primary_kind == "photon" else _lib.PMC_ELECTRON
            src.energy = float(source.energy)
            src.z0 = float(source.z)
            src.x_lo = float(source.x_range[0])
            src.x_extent = float(source.x_range[1] - source.x_range[0])
            src.y_lo = float(source.y_range[0])
            src.y_extent = float(source.y_range[1] - source.y_range[0])
            energy_emitted = n_histories * source.max_energy
        elif name == "SpectralBeamSource":
            spectrum = source.spectrum
            edges = np.ascontiguousarray(spectrum.edges, dtype=np.float64)
            cdf = np.ascontiguousarray(spectrum.cdf, dtype=np.float64)
            keep += [edges, cdf]
            src.type = _lib.PMC_SRC_SPECTRAL
            src.kind = _lib.PMC_PHOTON
            src.n_bins = int(cdf.size)
            src.edges = _lib.ptr(edges, C.c_double)
            src.cdf = _lib.ptr(cdf, C.c_double)
            src.focal[:] = [float(v) for v in source.focal_point]
            src.center[:] = [float(v) for v in source.center]
            src.u_axis[:] = [float(v) for v in source.u_axis]
            src.v_axis[:] = [float(v) for v in source.v_axis]
            src.width_u = float(source.width_u)
            src.width_v = float(source.width_v)
        elif name == "DevicePhaseSpace" and hasattr(source, "energy"):
            # a pre-solve's phase space already on the device (presolve.py):
            # the records are read in place, no copy to the host and back
            import torch

            dev = torch.device(self.device)
            if torch.device(source.device) != dev:
                raise ValueError(f"the phase space lives on {source.device}, the run on {dev}")
            kind = (source.particle_type - 1).to(torch.int32).contiguous()  # IAEA code -> PMC_* kind
            cols = [t.contiguous() for t in (source.energy, source.pos, source.dir, source.weight)]
            keep += [kind, *cols]
            dptr = lambda t, ct: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ct))  # noqa: E731
            src.type = _lib.PMC_SRC_PHASESPACE_DEVICE
            src.n_records = int(kind.shape[0])
            src.up_kind = dptr(kind, C.c_int32)
            src.up_energy = dptr(cols[0], C.c_float)
            src.up_pos = dptr(cols[1], C.c_float)
            src.up_dir = dptr(cols[2], C.c_float)
            src.up_weight = dptr(cols[3], C.c_float)
        elif name in ("PhaseSpaceSource", "InMemoryPhaseSpaceSource") and hasattr(source, "columns"):
            # The whole phase space resident on the device, one record drawn per
            # history from its own stream (PhaseSpaceSource.emit, geometry/phasespace.py:546).
            cols = source.columns()
            iaea_to_kind = np.array([-1, 0, 1, 2], dtype=np.int32)
            kind = np.ascontiguousarray(iaea_to_kind[np.asarray(cols["particle_type"], dtype=np.int32)])
            energy = np.ascontiguousarray(cols["energy"], dtype=np.float32)
            pos = np.ascontiguousarray(np.stack([cols["x"], cols["y"], cols["z"]], axis=1), dtype=np.float32)
            dirs = np.ascontiguousarray(np.stack([cols["ux"], cols["uy"], cols["uz"]], axis=1), dtype=np.float32)
            weight = np.ascontiguousarray(cols["weight"], dtype=np.float32)
            keep += [kind, energy, pos, dirs, weight]
            src.type = _lib.PMC_SRC_PHASESPACE
            src.n_records = int(energy.size)
            src.up_kind = _lib.ptr(kind, C.c_int32)
            src.up_energy = _lib.ptr(energy, C.c_float)
            src.up_pos = _lib.ptr(pos, C.c_float)
            src.up_dir = _lib.ptr(dirs, C.c_float)
            src.up_weight = _lib.ptr(weight, C.c_float)
        elif hasattr(source, "sample_batch"):
            # Host pre-sampling route (Source.sample_batch): records in history order.
            cols = source.sample_batch(seed, 0, n_histories)
            codes = np.asarray(cols["particle_type"], dtype=np.int32)
            iaea_to_kind = np.array([-1, 0, 1, 2], dtype=np.int32)
            kind = np.ascontiguousarray(iaea_to_kind[codes])
            energy = np.ascontiguousarray(cols["energy"], dtype=np.float32)
            pos = np.ascontiguousarray(np.stack([cols["x"], cols["y"], cols["z"]], axis=1), dtype=np.float32)
            dirs = np.ascontiguousarray(np.stack([cols["ux"], cols["uy"], cols["uz"]], axis=1), dtype=np.float32)
            weight = np.ascontiguousarray(cols["weight"], dtype=np.float32)
            keep += [kind, energy, pos, dirs, weight]
            src.type = _lib.PMC_SRC_UPLOAD
            src.up_kind = _lib.ptr(kind, C.c_int32)
            src.up_energy = _lib.ptr(energy, C.c_float)
            src.up_pos = _lib.ptr(pos, C.c_float)
            src.up_dir = _lib.ptr(dirs, C.c_float)
            src.up_weight = _lib.ptr(weight, C.c_float)
        else:
            raise ValueError(f"unsupported source type {name}")
        for wrapper in wrappers:  # weights from a stack or a mask (the Warp engine's
            # generate_spectral_masked_beam for a masked fan): emitted energy booked per primary
            _attach_weights(src, wrapper, keep)
            energy_emitted = None

        params = self._params(
            n_histories=n_histories, n_batches=n_batches, seed=seed, pcut=pcut, ecut=ecut,
            transport_electrons=transport_electrons, msc_gs=msc_gs,
            step_energy_fraction=step_energy_fraction, deposit_resolution=deposit_resolution,
            dose_to_water=dose_to_water,
        )
        emitter = _progress_emitter(progress, n_histories)
        scoring = scoring_grid
        n_vox = (int(np.prod(scoring.shape)) if scoring is not None
                 else int(np.prod(self.grid.shape)))
        shape = tuple(scoring.shape) if scoring is not None else tuple(self.grid.shape)
        dose = np.zeros(n_vox, dtype=np.float64)
        sigma = np.zeros(n_vox, dtype=np.float64)
        books = _lib.Books()
        tick = _lib.PROGRESS_FN(lambda _u, n: emitter.tick(int(n)))
        native = self._native()
        lib = native.lib
        with native.lock:
            self._upload(native, source.max_energy, pcut, ecut, msc_gs == 1, scoring)
            native.check(lib.pmc_set_progress(native.handle, C.cast(tick, C.c_void_p), None))
            try:
                code = lib.pmc_run_forward(native.handle, C.byref(src), C.byref(params),
                                           _lib.ptr(dose, C.c_double), _lib.ptr(sigma, C.c_double),
                                           C.byref(books))
            finally:
                lib.pmc_set_progress(native.handle, None, None)
            native.check(code)
        if energy_emitted is None:
            energy_emitted = float(books.emitted) * ENERGY_QUANTUM_MEV
        _, TransportResult, _ = _result_types()
        return TransportResult(
            dose=dose.reshape(shape),
            dose_sigma=sigma.reshape(shape),
            energy_emitted=energy_emitted,
            energy_deposited=float(books.deposited) * ENERGY_QUANTUM_MEV,
            energy_escaped=float(books.escaped) * ENERGY_QUANTUM_MEV,
            energy_unscored=float(books.unscored) * ENERGY_QUANTUM_MEV,
            n_histories=n_histories,
            n_batches=n_batches,
            scoring_mode=scoring_mode,
            provenance=self._provenance(seed, pcut, ecut, msc_model, step_energy_fraction,
                                        deposit_resolution_cm),
        )

    # ---- run_dij ------------------------------------------------------------------
    def run_dij(
        self,
        source,
        n_histories_per_beamlet,
        n_batches: int,
        seed: int,
        pcut: float = PCUT_MEV,
        ecut: float = ECUT_MEV,
        transport_electrons: bool = True,
        truncation: float = DIJ_TRUNCATION_RELATIVE,
        correlated: bool = True,
        beamlet_group_size: int | None = None,
        scoring_grid=None,
        scoring_mode: str = "dose_to_medium",
        step_energy_fraction: float | None = None,
        deposit_resolution_cm: float | None = None,
        msc_model: str = "gs",
        devices=None,
        concurrent_batches: int = 1,
        progress=None,
    ):
        """The Dij over the beamlets; the contract of ``WarpEngine.run_dij``.

        Extension: ``n_histories_per_beamlet`` may be a sequence of per-beamlet
        counts (each divisible by ``n_batches``).  Beamlet ``j`` then owns the
        histories ``offset_j + r`` with ``offset_j`` the exclusive prefix sum of
        the counts, so equal counts reproduce the reference mapping
        ``h = j * n_per + r`` exactly.  ``DijResult.n_histories_per_beamlet``
        carries the integer when the counts are equal and the maximum otherwise.
        """
        return self._run_dij(
            source, n_histories_per_beamlet, n_batches, seed, pcut=pcut, ecut=ecut,
            transport_electrons=transport_electrons, truncation=truncation, correlated=correlated,
            beamlet_group_size=beamlet_group_size, scoring_grid=scoring_grid,
            scoring_mode=scoring_mode, step_energy_fraction=step_energy_fraction,
            deposit_resolution_cm=deposit_resolution_cm, msc_model=msc_model, devices=devices,
            concurrent_batches=concurrent_batches, progress=progress, device_view=False)

    def run_dij_shard(self, source, n_histories_per_beamlet, n_batches: int, seed: int, *,
                      rank: int, world: int, **kwargs):
        """This rank's share of a Dij computed by `world` processes (one GPU
        each): ``(DijResult of columns first..stop-1, (first, stop))`` from
        :func:`column_shards`.  Beamlets keep their global history numbers, so
        the shards are bit-identical to the same columns of the whole Dij and
        :func:`merge_shards` rebuilds it; no data-path collective is needed."""
        n = int(source.n_beamlets)
        counts = (np.full(n, int(n_histories_per_beamlet), dtype=np.int64)
                  if np.ndim(n_histories_per_beamlet) == 0
                  else np.asarray(n_histories_per_beamlet, dtype=np.int64))
        if not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside a world of {world}")
        span = column_shards(counts, world)[rank]
        dij = self._run_dij(source, counts, n_batches, seed, columns=span, **kwargs)
        return dij, span

    def run_dij_device(self, source, n_histories_per_beamlet, n_batches: int, seed: int,
                       **kwargs) -> "DeviceDij":
        """``run_dij`` on this engine's device, leaving the CSC there.

        Same arguments as :meth:`run_dij` (one device, one beamlet group).  The
        result's device arrays belong to the engine and stay valid until its
        next run; the denoiser reads them without a host round trip.
        """
        if kwargs.get("devices") not in (None, [self.device], (self.device,)):
            raise ValueError("run_dij_device runs on the engine's own device only")
        if kwargs.get("beamlet_group_size") not in (None, int(source.n_beamlets)):
            raise ValueError("run_dij_device runs the beamlets as one group")
        kwargs.pop("devices", None)
        return self._run_dij(source, n_histories_per_beamlet, n_batches, seed, device_view=True,
                             **kwargs)

    def _run_dij(
        self,
        source,
        n_histories_per_beamlet,
        n_batches: int,
        seed: int,
        pcut: float = PCUT_MEV,
        ecut: float = ECUT_MEV,
        transport_electrons: bool = True,
        truncation: float = DIJ_TRUNCATION_RELATIVE,
        correlated: bool = True,
        beamlet_group_size: int | None = None,
        scoring_grid=None,
        scoring_mode: str = "dose_to_medium",
        step_energy_fraction: float | None = None,
        deposit_resolution_cm: float | None = None,
        msc_model: str = "gs",
        devices=None,
        concurrent_batches: int = 1,
        progress=None,
        device_view: bool = False,
        columns: tuple[int, int] | None = None,
    ):
        n_beamlets = int(source.n_beamlets)
        if np.ndim(n_histories_per_beamlet) == 0:
            counts = np.full(n_beamlets, int(n_histories_per_beamlet), dtype=np.int64)
        else:
            counts = np.asarray(n_histories_per_beamlet, dtype=np.int64).copy()
            if counts.shape != (n_beamlets,):
                raise ValueError(f"need {n_beamlets} per-beamlet history counts, got {counts.shape}")
        for c in counts:
            if c < 1:
                raise ValueError(f"need at least one history per beamlet, got {int(c)}")
            if c % n_batches != 0:
                raise ValueError(
                    f"n_histories_per_beamlet={int(c)} not divisible by "
                    f"n_batches={n_batches}; unequal batches would weight batch means inconsistently"
                )
        if beamlet_group_size is not None and beamlet_group_size < 1:
            raise ValueError(f"need a positive beamlet group size, got {beamlet_group_size}")
        if concurrent_batches < 1:
            raise ValueError(f"need at least one lane, got concurrent_batches={concurrent_batches}")
        if truncation < 0.0:
            raise ValueError(f"negative truncation {truncation}")
        dose_to_water = 1 if validate_scoring_mode(scoring_mode, transport_electrons) else 0
        msc_gs = _validate_msc_model(msc_model)
        if step_energy_fraction is None:
            step_energy_fraction = default_step_energy_fraction(msc_model)
        if deposit_resolution_cm is not None and deposit_resolution_cm <= 0.0:
            raise ValueError(f"deposit resolution must be positive, got {deposit_resolution_cm}")
        deposit_resolution = 0.0 if deposit_resolution_cm is None else deposit_resolution_cm
        device_list = [self.device] if devices is None else list(dict.fromkeys(devices))
        if not device_list:
            raise ValueError("devices must name at least one device")

        name = _type_name(source)
        offsets = np.zeros(n_beamlets, dtype=np.int64)
        np.cumsum(counts[:-1], out=offsets[1:])
        col_lo, col_hi = (0, n_beamlets) if columns is None else (int(columns[0]), int(columns[1]))
        if not 0 <= col_lo <= col_hi <= n_beamlets:
            raise ValueError(f"column range {columns} outside 0..{n_beamlets}")
        if columns is not None and len(device_list) > 1:
            raise ValueError("a column range runs on one device")
        per, records = beamlet_arrays(source)
        energy_emitted = (float(np.sum(counts[col_lo:col_hi])) * source.max_energy
                          if name == "BeamletGridSource" else None)

        params = self._params(
            n_batches=n_batches, seed=seed, pcut=pcut, ecut=ecut,
            transport_electrons=transport_electrons, msc_gs=msc_gs,
            step_energy_fraction=step_energy_fraction, deposit_resolution=deposit_resolution,
            dose_to_water=dose_to_water, truncation=truncation, correlated=correlated,
            beamlet_group_size=beamlet_group_size,
        )
        emitter = _progress_emitter(progress, int(np.sum(counts)))
        group = beamlet_group_size or n_beamlets
        group_starts = list(range(0, n_beamlets, group)) if len(device_list) > 1 else [col_lo]
        span = group if len(device_list) > 1 else col_hi - col_lo
        if col_hi == col_lo:
            group_starts = []
        pending = deque(group_starts)
        pending_lock = threading.Lock()

        def next_group():
            with pending_lock:
                return pending.popleft() if pending else None

        def shard(device: str):
            native = self._native(device)
            lib = native.lib
            blocks = {}
            totals = np.zeros(4, dtype=np.int64)
            tick = _lib.PROGRESS_FN(lambda _u, n: emitter.tick(int(n)))
            while (g0 := next_group()) is not None:
                g1 = min(g0 + span, col_hi)
                sl = slice(g0, g1)
                keep = []
                desc = beamlet_descriptor(source, sl, seed, keep, per=per, records=records)
                sub_counts = np.ascontiguousarray(counts[sl])
                sub_offsets = np.ascontiguousarray(offsets[sl])
                keep += [sub_counts, sub_offsets]
                desc.history_offsets = _lib.ptr(sub_offsets, C.c_int64)
                nnz = C.c_int64()
                books = _lib.Books()
                with native.lock:
                    self._upload(native, source.max_energy, pcut, ecut, msc_gs == 1, scoring_grid)
                    native.check(lib.pmc_set_progress(native.handle, C.cast(tick, C.c_void_p), None))
                    try:
                        code = lib.pmc_run_dij(native.handle, C.byref(desc),
                                               _lib.ptr(sub_counts, C.c_int64), C.byref(params),
                                               C.byref(nnz), C.byref(books))
                    finally:
                        lib.pmc_set_progress(native.handle, None, None)
                    for item in keep:  # an exception the host sampler raised inside the call
                        if isinstance(item, list) and item and isinstance(item[0], Exception):
                            raise item[0]
                    native.check(code)
                    if device_view:
                        return _device_dij(native, g1 - g0, nnz.value, books), None
                    indptr = np.zeros(g1 - g0 + 1, dtype=np.int64)
                    indices = _pinned_array(nnz.value, np.int64)
                    dose = _pinned_array(nnz.value, np.float64)
                    sigma = _pinned_array(nnz.value, np.float64)
                    native.check(lib.pmc_dij_fetch(native.handle, _lib.ptr(indptr, C.c_int64),
                                                   _lib.ptr(indices, C.c_int64),
                                                   _lib.ptr(dose, C.c_double),
                                                   _lib.ptr(sigma, C.c_double)))
                blocks[g0] = (np.diff(indptr), indices, dose, sigma)
                totals += np.array([books.deposited, books.escaped, books.unscored, books.emitted])
            return blocks, totals

        if device_view:
            view, _ = shard(device_list[0])
            view.grid_shape = (tuple(scoring_grid.shape) if scoring_grid is not None
                               else tuple(self.grid.shape))
            view.counts = counts
            view.n_batches = n_batches
            view.device = device_list[0]
            return view
        if len(device_list) == 1:
            results = [shard(device_list[0])]
        else:
            with ThreadPoolExecutor(max_workers=len(device_list)) as pool:
                results = [f.result() for f in [pool.submit(shard, d) for d in device_list]]
        blocks = {g: b for r, _ in results for g, b in r.items()}
        totals = sum((t for _, t in results), np.zeros(4, dtype=np.int64))
        counts_all, idx_all, dose_all, sig_all = [], [], [], []
        for g0 in group_starts:
            c, i, d, s = blocks[g0]
            counts_all.append(c)
            idx_all.append(i)
            dose_all.append(d)
            sig_all.append(s)
        n_out = col_hi - col_lo
        col_counts = np.concatenate(counts_all) if counts_all else np.zeros(0, dtype=np.int64)
        indptr = np.zeros(n_out + 1, dtype=np.int64)
        np.cumsum(col_counts, out=indptr[1:])

        def joined(parts, dtype=np.float64):  # one block (one device) needs no copy
            if not parts:
                return np.zeros(0, dtype=dtype)
            return parts[0] if len(parts) == 1 else np.concatenate(parts)

        counts = counts[col_lo:col_hi] if n_out else counts[:1]

        if energy_emitted is None:
            energy_emitted = float(totals[3]) * ENERGY_QUANTUM_MEV
        shape = tuple(scoring_grid.shape) if scoring_grid is not None else tuple(self.grid.shape)
        _, _, DijResult = _result_types()
        equal = bool(np.all(counts == counts[0]))
        return DijResult(
            grid_shape=shape,
            n_beamlets=n_out,
            n_histories_per_beamlet=int(counts[0]) if equal else int(counts.max()),
            n_batches=n_batches,
            truncation=truncation,
            indptr=indptr,
            indices=joined(idx_all, np.int64),
            dose=joined(dose_all),
            sigma=joined(sig_all),
            energy_emitted=energy_emitted,
            energy_deposited=float(totals[0]) * ENERGY_QUANTUM_MEV,
            energy_escaped=float(totals[1]) * ENERGY_QUANTUM_MEV,
            energy_unscored=float(totals[2]) * ENERGY_QUANTUM_MEV,
            correlated=correlated,
            scoring_mode=scoring_mode,
            provenance=self._provenance(seed, pcut, ecut, msc_model, step_energy_fraction,
                                        deposit_resolution_cm, devices=device_list),
        )
