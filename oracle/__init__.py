"""TEST INFRASTRUCTURE — the oracle of the B200 backend's parity tests.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of
``bench.py`` may import this package, and only as the checker (or the timed CPU
baseline); the product (``pyradmc_b200``) never imports, links or calls it.

Contents
--------
``transport.c``  CPU restatement of pyRadMC's coupled transport (float64,
                 one history at a time on a LIFO stack), built by ``Makefile``
                 into ``_build/liboracle.so`` and driven by :func:`run`.
``reduction.py`` numpy restatement of the batch fold, finalize, truncation and
                 CSC assembly (scoring/dij.py:155-434).
``stats.py``     the reference's statistical detection oracles
                 (tests/conftest.py:45-196 of pyRadMC).

Pinning: ``reduction.py`` is checked bit-for-bit against pyRadMC's own scorer
outputs (``tests/golden/reduction.npz``); ``transport.c`` is checked by batched
chi-squared against pyRadMC ``ReferenceEngine`` runs (``tests/golden/ref_*.npz``),
both generated by ``tests/golden/make_golden.py``.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
import threading
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

_dp = C.POINTER(C.c_double)
_d3 = C.c_double * 3


class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("origin", _d3),
                ("spacing", _d3), ("density", _dp), ("material", C.POINTER(C.c_uint8))]


class _Tables(C.Structure):
    _fields_ = [("n_materials", C.c_int), ("n_points", C.c_int),
                ("p_log_min", C.c_double), ("p_inv_dlog", C.c_double),
                ("e_log_min", C.c_double), ("e_inv_dlog", C.c_double),
                ("r_log_min", C.c_double), ("r_inv_dlog", C.c_double)] + [
        (n, _dp) for n in ("mu_compton", "mu_photo", "mu_pair", "mu_rayleigh", "majorant",
                           "stopping_radiative", "moller", "csda_range", "scattering_power",
                           "log_eta", "restricted_range", "energy_of_restricted_range")
    ] + [("n_coherent", C.c_int), ("coherent_x", _dp), ("coherent_cumulative", _dp)]


class _GS(C.Structure):
    _fields_ = [("values", C.POINTER(C.c_float)), ("ix0", C.c_int), ("iy0", C.c_int),
                ("n_eta", C.c_int), ("n_theta2", C.c_int), ("n_u", C.c_int),
                ("bins_per_log", C.c_double)]


class _Source(C.Structure):
    _fields_ = [("type", C.c_int), ("kind", C.c_int), ("energy", C.c_double),
                ("position", _d3), ("direction", _d3), ("z0", C.c_double),
                ("x_lo", _dp), ("x_extent", _dp), ("y_lo", _dp), ("y_extent", _dp),
                ("n_bins", C.c_int), ("edges", _dp), ("cdf", _dp), ("focal", _d3),
                ("u_axis", _d3), ("v_axis", _d3), ("width_u", C.c_double),
                ("width_v", C.c_double), ("centers", _dp), ("mask", _dp),
                ("mask_n_u", C.c_int), ("mask_n_v", C.c_int), ("mask_center", _d3),
                ("mask_u", _d3), ("mask_v", _d3), ("mask_width_u", C.c_double),
                ("mask_width_v", C.c_double)]


class _Params(C.Structure):
    _fields_ = [("forward", C.c_int), ("n_cols", C.c_int), ("counts", C.POINTER(C.c_int64)),
                ("n_batches", C.c_int), ("seed", C.c_uint64), ("pcut", C.c_double),
                ("ecut", C.c_double), ("transport_electrons", C.c_int), ("msc_gs", C.c_int),
                ("correlated", C.c_int), ("step_energy_fraction", C.c_double),
                ("n_threads", C.c_int), ("first_history", C.c_int64),
                ("max_histories", C.c_int64)]


_lib = None
_lock = threading.Lock()


def load():
    """Build (make) and load the C oracle."""
    global _lib
    with _lock:
        if _lib is None:
            src = HERE / "transport.c"
            if not LIB.exists() or LIB.stat().st_mtime < src.stat().st_mtime:
                subprocess.run(["make", "-s", "-f", str(HERE / "Makefile")], check=True)
            lib = C.CDLL(str(LIB))
            lib.oracle_transport.restype = C.c_int
            lib.oracle_transport.argtypes = [C.POINTER(_Grid), C.POINTER(_Tables), C.POINTER(_GS),
                                             C.POINTER(_Source), C.POINTER(_Params), _dp, _dp,
                                             C.POINTER(C.c_int64)]
            lib.oracle_philox.restype = None
            lib.oracle_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                          C.POINTER(C.c_uint32)]
            lib.oracle_max_threads.restype = C.c_int
            _lib = lib
    return _lib


def philox(counter, key) -> np.ndarray:
    """Philox4x32-10 of one counter block, for the known-answer tests."""
    lib = load()
    c = (C.c_uint32 * 4)(*counter)
    k = (C.c_uint32 * 2)(*key)
    out = (C.c_uint32 * 4)()
    lib.oracle_philox(c, k, out)
    return np.array(list(out), dtype=np.uint32)


def max_threads() -> int:
    return int(load().oracle_max_threads())


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def run(grid, tables, gs, source, *, counts, n_batches, seed, forward=True, pcut=0.05,
        ecut=0.2, transport_electrons=True, msc_model="gs", correlated=True,
        step_energy_fraction=None, primary_kind="photon", n_threads=None, first_history=0,
        max_histories=0):
    """Run the CPU oracle on one source; returns (mean, sigma, books) per column.

    ``grid`` needs shape/spacing/origin/density/material; ``tables`` the
    CrossSectionTables fields; ``gs`` values/ix0/iy0/bins_per_log; ``source`` is a
    pencil, parallel, lattice, spectral (optionally masked) or spectral-beamlet source (the same
    classes the engine takes).  ``counts`` gives each column's histories.
    """
    lib = load()
    keep = []
    density = _d(grid.density).reshape(-1)
    material = np.ascontiguousarray(np.asarray(grid.material).reshape(-1), dtype=np.uint8)
    keep += [density, material]
    g = _Grid(nx=int(grid.shape[0]), ny=int(grid.shape[1]), nz=int(grid.shape[2]))
    g.origin[:] = [float(v) for v in grid.origin]
    g.spacing[:] = [float(v) for v in grid.spacing]
    g.density = density.ctypes.data_as(_dp)
    g.material = material.ctypes.data_as(C.POINTER(C.c_uint8))
    t = _Tables(n_materials=int(np.asarray(tables.mu_compton).shape[0]),
                n_points=int(tables.n_points), p_log_min=float(tables.photon_log_e_min),
                p_inv_dlog=float(tables.photon_inv_dlog),
                e_log_min=float(tables.electron_log_e_min),
                e_inv_dlog=float(tables.electron_inv_dlog),
                r_log_min=float(tables.range_log_r_min), r_inv_dlog=float(tables.range_inv_dlog),
                n_coherent=int(tables.n_coherent))
    for name in ("mu_compton", "mu_photo", "mu_pair", "mu_rayleigh", "majorant",
                 "stopping_radiative", "moller", "csda_range", "scattering_power", "log_eta",
                 "restricted_range", "energy_of_restricted_range", "coherent_x",
                 "coherent_cumulative"):
        arr = _d(getattr(tables, name)).reshape(-1)
        keep.append(arr)
        setattr(t, name, arr.ctypes.data_as(_dp))
    values = np.ascontiguousarray(np.asarray(gs.values), dtype=np.float32)
    keep.append(values)
    gsd = _GS(values=values.ctypes.data_as(C.POINTER(C.c_float)), ix0=int(gs.ix0),
              iy0=int(gs.iy0), n_eta=values.shape[0], n_theta2=values.shape[1],
              n_u=values.shape[2], bins_per_log=float(gs.bins_per_log))
    s = _Source(kind=0 if primary_kind == "photon" else 1)
    name = type(source).__name__
    n_cols = len(counts)

    def arr(x):
        a = _d(x)
        keep.append(a)
        return a.ctypes.data_as(_dp)

    if name == "TransmissionMaskSource" and type(source.inner).__name__ == "SpectralBeamSource":
        # the spectral fan, its primaries weighted by the mask
        mask = _d(source.mask)
        keep.append(mask)
        s.mask = mask.ctypes.data_as(_dp)
        s.mask_n_u, s.mask_n_v = (int(n) for n in mask.shape)
        s.mask_center[:] = list(map(float, source.plane_center))
        s.mask_u[:] = list(map(float, source.u_axis))
        s.mask_v[:] = list(map(float, source.v_axis))
        s.mask_width_u, s.mask_width_v = float(source.width_u), float(source.width_v)
        source, name = source.inner, "SpectralBeamSource"
    if name == "PencilBeamSource":
        s.type = 0
        s.energy = float(source.energy)
        s.position[:] = list(map(float, source.position))
        s.direction[:] = list(map(float, source.direction))
    elif name in ("ParallelBeamSource", "BeamletGridSource"):
        s.type = 1
        s.energy = float(source.energy)
        s.z0 = float(source.z)
        if name == "ParallelBeamSource":
            b = np.array([[source.x_range[0], source.x_range[1], source.y_range[0], source.y_range[1]]])
        else:
            b = np.array([source.beamlet_bounds(j) for j in range(n_cols)], dtype=np.float64)
        s.x_lo, s.x_extent = arr(b[:, 0]), arr(b[:, 1] - b[:, 0])
        s.y_lo, s.y_extent = arr(b[:, 2]), arr(b[:, 3] - b[:, 2])
    elif name in ("SpectralBeamSource", "SpectralBeamletSource"):
        s.type = 2
        centers = ([source.center] if name == "SpectralBeamSource" else list(source.centers))
        s.centers = arr(np.asarray(centers, dtype=np.float64).reshape(-1))
        s.n_bins = int(np.asarray(source.spectrum.cdf).size)
        s.edges, s.cdf = arr(source.spectrum.edges), arr(source.spectrum.cdf)
        s.focal[:] = list(map(float, source.focal_point))
        s.u_axis[:] = list(map(float, source.u_axis))
        s.v_axis[:] = list(map(float, source.v_axis))
        s.width_u, s.width_v = float(source.width_u), float(source.width_v)
    else:
        raise ValueError(f"unsupported source {name}")
    cnt = np.ascontiguousarray(counts, dtype=np.int64)
    keep.append(cnt)
    if step_energy_fraction is None:
        step_energy_fraction = 0.20 if msc_model == "gs" else 0.05
    p = _Params(forward=1 if forward else 0, n_cols=n_cols,
                counts=cnt.ctypes.data_as(C.POINTER(C.c_int64)), n_batches=int(n_batches),
                seed=int(seed), pcut=float(pcut), ecut=float(ecut),
                transport_electrons=1 if transport_electrons else 0,
                msc_gs=1 if msc_model == "gs" else 0, correlated=1 if correlated else 0,
                step_energy_fraction=float(step_energy_fraction),
                n_threads=int(n_threads or os.cpu_count() or 1),
                first_history=int(first_history), max_histories=int(max_histories))
    n_vox = int(np.prod(grid.shape))
    mean = np.zeros(n_cols * n_vox)
    sigma = np.zeros(n_cols * n_vox)
    books = (C.c_int64 * 3)()
    code = lib.oracle_transport(C.byref(g), C.byref(t), C.byref(gsd), C.byref(s), C.byref(p),
                                mean.ctypes.data_as(_dp), sigma.ctypes.data_as(_dp), books)
    if code != 0:
        raise RuntimeError(f"oracle transport failed with code {code}")
    return (mean.reshape(n_cols, n_vox), sigma.reshape(n_cols, n_vox),
            dict(deposited=books[0] * 1e-9, escaped=books[1] * 1e-9, emitted=books[2] * 1e-9))
