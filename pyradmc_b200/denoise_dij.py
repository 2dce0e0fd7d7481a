"""Dij columns through the denoiser: device-side conversion, windows, training
pairs, the denoised Dij and its error against high-statistics Monte Carlo.

No counterpart in pyRadMC.  Every step runs on the device through the C-ABI of
``include/pyradmc_b200_denoise.h`` (plus ``pmc_dij_compact_static`` for the
final truncation + CSC); torch allocates the buffers and supplies the stream.

Columns are dense volumes in the Dij's voxel order (x-major, z fastest).  Each
column is denoised in windows that follow its beamlet: the grid axis closest
to the beamlet's direction is the window's depth axis (read from the far end
when the beam travels towards lower indices, so that every window sees the
beam enter at its first depth plane), the lateral axes shift with depth along
the beamlet (whole voxels, no resampling), the depth is cut into chunks, and
each chunk's window is centred on the column's dose within the chunk.  Voxels
outside every window keep their Monte Carlo values.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .denoiser import LEVELS, UNet3D, _check


def _torch():
    import torch

    return torch


def _stream(device) -> int:
    return _torch().cuda.current_stream(device).cuda_stream


def _device_density(engine, device):
    """The engine grid's density as float32 [vox] on `device`, converted and
    uploaded once per (grid, device) and kept on the engine: the conversion
    and a pageable upload cost milliseconds of host time per Dij."""
    torch = _torch()
    key = ("density_on_device", id(engine.grid), str(device))
    rho = engine._host_arrays.get(key)  # the engine's per-grid cache
    if rho is None:
        rho = engine._host_arrays[key] = torch.from_numpy(
            np.ascontiguousarray(engine.grid.density, dtype=np.float32).ravel()).to(device)
    return rho


def dense_columns(view, device, with_sigma: bool = False):
    """(dose f32 [C, vox], colmax f32 [C], sigma f32 [C, vox] or None) of a
    :class:`DeviceDij` on its device."""
    torch = _torch()
    lib = _lib.load()
    n_cols = view.n_beamlets
    vox = int(np.prod(view.grid_shape))
    indptr = torch.from_numpy(view.indptr).to(device)
    dose = torch.zeros((n_cols, vox), dtype=torch.float32, device=device)
    colmax = torch.zeros(n_cols, dtype=torch.float32, device=device)
    st = _stream(device)
    if view.nnz:
        _check(lib.pmd_csc_to_dense(indptr.data_ptr(), view.indices, view.dose, n_cols, vox,
                                    dose.data_ptr(), colmax.data_ptr(), st), "csc to dense")
    sigma = None
    if with_sigma:
        sigma = torch.zeros((n_cols, vox), dtype=torch.float32, device=device)
        if view.nnz:
            _check(lib.pmd_csc_to_dense(indptr.data_ptr(), view.indices, view.sigma, n_cols, vox,
                                        sigma.data_ptr(), torch.zeros_like(colmax).data_ptr(), st),
                   "csc to dense")
    return dose, colmax, sigma


def dense_columns_f64(view, device):
    """(mean f64 [C, vox], sigma f64 [C, vox]) of a :class:`DeviceDij`."""
    torch = _torch()
    lib = _lib.load()
    n_cols = view.n_beamlets
    vox = int(np.prod(view.grid_shape))
    indptr = torch.from_numpy(view.indptr).to(device)
    mean = torch.zeros((n_cols, vox), dtype=torch.float64, device=device)
    sigma = torch.zeros((n_cols, vox), dtype=torch.float64, device=device)
    if view.nnz:
        st = _stream(device)
        _check(lib.pmd_csc_to_dense_f64(indptr.data_ptr(), view.indices, view.dose, n_cols, vox,
                                        mean.data_ptr(), st), "csc to dense")
        _check(lib.pmd_csc_to_dense_f64(indptr.data_ptr(), view.indices, view.sigma, n_cols, vox,
                                        sigma.data_ptr(), st), "csc to dense")
    return mean, sigma


def gather(src, grid_shape, origins, window, shared: bool = False):
    """Windows [C, wx, wy, wz] of src ([C, vox], or one shared [vox] volume)."""
    torch = _torch()
    nx, ny, nz = grid_shape
    wx, wy, wz = window
    n = origins.shape[0]
    out = torch.empty((n, wx, wy, wz), dtype=torch.float32, device=src.device)
    stride = 0 if shared else int(np.prod(grid_shape))
    _check(_lib.load().pmd_gather_windows(src.data_ptr(), stride, nx, ny, nz, origins.data_ptr(), n,
                                          wx, wy, wz, out.data_ptr(), _stream(src.device)),
           "gather windows")
    return out


def scatter(win, scale, grid_shape, origins, dst) -> None:
    """dst[c] (f64 [C, vox]) <- max(win, 0) * scale[c] inside each window."""
    nx, ny, nz = grid_shape
    n, wx, wy, wz = win.shape
    _check(_lib.load().pmd_scatter_windows(win.data_ptr(), None if scale is None else scale.data_ptr(),
                                           nx, ny, nz, origins.data_ptr(), n, wx, wy, wz,
                                           dst.data_ptr(), int(np.prod(grid_shape)),
                                           _stream(win.device)), "scatter windows")


def beam_directions(source) -> np.ndarray:
    """Unit travel direction [n_beamlets, 3] of every column's central ray:
    aperture centre minus focal spot for a divergent fan, +z for a lattice
    (and for sources whose geometry is not known here), part by part for a
    concatenation."""
    parts = getattr(source, "sources", None)
    if parts is not None and hasattr(source, "part_of"):
        return np.concatenate([beam_directions(p) for p in parts]) if parts else np.zeros((0, 3))
    n = int(source.n_beamlets)
    focal, centers = getattr(source, "focal_point", None), getattr(source, "centers", None)
    if focal is None or centers is None:
        return np.tile([0.0, 0.0, 1.0], (n, 1))
    d = np.asarray(centers, dtype=np.float64) - np.asarray(focal, dtype=np.float64)[None, :]
    return d / np.linalg.norm(d, axis=1, keepdims=True)


def orientation_codes(directions) -> np.ndarray:
    """int32 [n]: 2 * (axis of the largest |component|) + (1 if it is negative)."""
    d = np.asarray(directions, dtype=np.float64).reshape(-1, 3)
    axis = np.argmax(np.abs(d), axis=1)
    neg = d[np.arange(d.shape[0]), axis] < 0
    return (2 * axis + neg).astype(np.int32)


def _frame(orient: int):
    """(lateral axis 1, lateral axis 2, depth axis, reversed) of an orientation code."""
    d, f = orient >> 1, orient & 1
    lat = [a for a in range(3) if a != d]
    return lat[0], lat[1], d, bool(f)


WIN_INTS = 7      # (ox, oy, oz, orient, col, shear1, shear2) per oriented window
SHEAR_ONE = 65536  # shear unit: 1/65536 voxel per depth plane


SHEAR_MIN = 0.1  # voxels per depth plane: beamlets closer to their axis keep plain windows


def oriented_windows(dose, grid_shape, directions, window, starts=None, spacing=None):
    """int32 [W, 7] oriented windows (ox, oy, oz, orient, col, shear1, shear2)
    of dense columns dose [C, vox] (pmd_gather_windows_oriented).
    `directions` [C, 3] are the beamlets' travel directions and `window` =
    (wa, wb, wd) the lateral and depth extent.  A window's depth axis is the
    grid axis closest to its beamlet, read from the beam's entry side, and for
    a beamlet that drifts at least SHEAR_MIN voxels per depth plane its lateral
    axes shear with depth along the beamlet (1/65536-voxel steps), so an
    oblique beamlet runs straight down the window (a near-axial one keeps the
    plain window: whole-voxel steps ten or more planes apart would only add
    jitter).  Without `starts` every
    column is covered along its whole depth by consecutive depth chunks of wd
    planes (the last may reach past the grid); with `starts` ([C], depth planes
    counted from the entry side) each column gets one window there.  A
    window's lateral position is the dose-weighted mean of the beamlet's
    sheared axis over its depth range (the column's own where that range
    holds no dose), clamped so that its middle plane lies inside the grid."""
    torch = _torch()
    dev = dose.device
    n_cols = dose.shape[0]
    dirs = np.asarray(directions, dtype=np.float64).reshape(n_cols, 3)
    orient = orientation_codes(dirs)
    sp = np.ones(3) if spacing is None else np.asarray(spacing, dtype=np.float64)
    wa, wb, wd = window
    vol = dose.view(n_cols, *grid_shape)
    out = []
    for code in np.unique(orient):
        cols = np.nonzero(orient == code)[0]
        l1, l2, d, rev = _frame(int(code))
        n1, n2, nd = grid_shape[l1], grid_shape[l2], grid_shape[d]
        idx = torch.from_numpy(cols).to(dev)
        # voxels moved along l1, l2 per plane of depth, and the same in 1/65536 units
        per_depth = np.abs(dirs[cols, d]) / sp[d]
        slope1 = (dirs[cols, l1] / sp[l1]) / per_depth
        slope2 = (dirs[cols, l2] / sp[l2]) / per_depth
        sheared = np.maximum(np.abs(slope1), np.abs(slope2)) >= SHEAR_MIN
        q1 = np.where(sheared, np.round(slope1 * SHEAR_ONE), 0).astype(np.int64)
        q2 = np.where(sheared, np.round(slope2 * SHEAR_ONE), 0).astype(np.int64)
        # lateral marginals per depth plane, a few columns at a time (no copy
        # of the columns): m1 [c, n1, nd], m2 [c, n2, nd], depth from the entry side
        m1 = torch.empty((len(cols), n1, nd), dtype=torch.float32, device=dev)
        m2 = torch.empty((len(cols), n2, nd), dtype=torch.float32, device=dev)
        j = 0
        while j < len(cols):  # runs of consecutive columns, 16 at a time, as views
            k = j + 1
            while k < len(cols) and k - j < 16 and cols[k] == cols[k - 1] + 1:
                k += 1
            v = vol[int(cols[j]):int(cols[k - 1]) + 1].permute(0, 1 + l1, 1 + l2, 1 + d)
            m1[j:k] = v.sum(dim=2)
            m2[j:k] = v.sum(dim=1)
            j = k
        if rev:
            m1, m2 = m1.flip(2), m2.flip(2)
        t = torch.arange(nd, device=dev, dtype=torch.float32)
        x1 = torch.arange(n1, device=dev, dtype=torch.float32)
        x2 = torch.arange(n2, device=dev, dtype=torch.float32)
        mass = m1.sum(dim=1)                                   # [c, nd] dose per depth plane
        s1 = torch.as_tensor(q1, dtype=torch.float32, device=dev).view(-1, 1) / SHEAR_ONE
        s2 = torch.as_tensor(q2, dtype=torch.float32, device=dev).view(-1, 1) / SHEAR_ONE
        # first moments of the sheared lateral coordinates x - s * t, per plane
        f1 = (m1 * x1.view(1, -1, 1)).sum(dim=1) - s1 * t * mass
        f2 = (m2 * x2.view(1, -1, 1)).sum(dim=1) - s2 * t * mass
        if starts is None:
            n_ch = -(-nd // wd)
            lo = (torch.arange(n_ch, device=dev) * wd).expand(len(cols), n_ch)
        else:
            lo = torch.as_tensor(np.asarray(starts)[cols], dtype=torch.int64, device=dev).view(-1, 1)
        tt = torch.arange(nd, device=dev).view(1, 1, -1)
        mask = ((tt >= lo.unsqueeze(2)) & (tt < lo.unsqueeze(2) + wd)).float()  # [c, chunks, nd]
        w_ch = torch.einsum("ct,cjt->cj", mass, mask)
        i1 = torch.einsum("ct,cjt->cj", f1, mask)
        i2 = torch.einsum("ct,cjt->cj", f2, mask)
        whole = mass.sum(dim=1, keepdim=True).clamp_min(1e-30)
        ok = w_ch > 0
        c1 = torch.where(ok, i1 / w_ch.clamp_min(1e-30), f1.sum(dim=1, keepdim=True) / whole)
        c2 = torch.where(ok, i2 / w_ch.clamp_min(1e-30), f2.sum(dim=1, keepdim=True) / whole)
        # window origin at its first plane; the middle plane is kept inside the grid
        mid = lo.float() + wd / 2
        o1 = torch.clamp(torch.round(c1 + s1 * mid - wa / 2), 0, max(n1 - wa, 0)) - torch.round(s1 * wd / 2)
        o2 = torch.clamp(torch.round(c2 + s2 * mid - wb / 2), 0, max(n2 - wb, 0)) - torch.round(s2 * wd / 2)
        od = (nd - (lo + wd)) if rev else lo
        w = torch.zeros((*o1.shape, WIN_INTS), dtype=torch.int32, device=dev)
        w[..., l1] = o1.to(torch.int32)
        w[..., l2] = o2.to(torch.int32)
        w[..., d] = od.to(torch.int32)
        w[..., 3] = int(code)
        w[..., 4] = idx.to(torch.int32).view(-1, 1)
        w[..., 5] = torch.as_tensor(q1, dtype=torch.int32, device=dev).view(-1, 1)
        w[..., 6] = torch.as_tensor(q2, dtype=torch.int32, device=dev).view(-1, 1)
        out.append(w.view(-1, WIN_INTS))
    if not out:
        return torch.zeros((0, WIN_INTS), dtype=torch.int32, device=dev)
    win = torch.cat(out)
    order = torch.argsort(win[:, 4], stable=True)  # windows of a column together, in depth order
    return win[order].contiguous()


def gather_oriented(src, grid_shape, win, window, shared: bool = False):
    """Oriented windows [W, wa, wb, wd] of src ([C, vox] read through each
    window's column, or one shared [vox] volume)."""
    torch = _torch()
    nx, ny, nz = grid_shape
    wa, wb, wd = window
    n = win.shape[0]
    out = torch.empty((n, wa, wb, wd), dtype=torch.float32, device=src.device)
    stride = 0 if shared else int(np.prod(grid_shape))
    _check(_lib.load().pmd_gather_windows_oriented(src.data_ptr(), stride, nx, ny, nz, win.data_ptr(),
                                                   n, wa, wb, wd, out.data_ptr(), _stream(src.device)),
           "gather oriented windows")
    return out


def scatter_oriented(data, scale, grid_shape, win, dst) -> None:
    """dst[col] (f64 [C, vox]) <- max(data, 0) * scale[w] inside each window."""
    nx, ny, nz = grid_shape
    n, wa, wb, wd = data.shape
    _check(_lib.load().pmd_scatter_windows_oriented(
        data.data_ptr(), None if scale is None else scale.data_ptr(), nx, ny, nz, win.data_ptr(), n,
        wa, wb, wd, dst.data_ptr(), int(np.prod(grid_shape)), _stream(data.device)),
        "scatter oriented windows")


# ---- training pairs --------------------------------------------------------------------
@dataclass
class PairSet:
    """Training pairs on the device, each [N, wx, wy, wz] float32: the
    low-history input and the high-history target (both divided by the input
    column's maximum), the target's sigma on the same scale, the density, the
    loss weight, and the input's Monte Carlo sigma."""

    inputs: object
    targets: object
    sigma: object
    density: object
    weight: object
    noise: object  # the input's Monte Carlo sigma, on the input's scale

    def __len__(self) -> int:
        return int(self.inputs.shape[0])

    def subset(self, idx) -> "PairSet":
        return PairSet(*(getattr(self, f)[idx] for f in PAIR_FIELDS))


PAIR_FIELDS = ("inputs", "targets", "sigma", "density", "weight", "noise")


def make_pairs(grid, cross_sections, source, *, n_low, n_high: int, n_batches: int,
               seed: int, window=(64, 64, 64), device="cuda:0", precision=0.02,
               rng=None) -> PairSet:
    """Pairs of one phantom: the engine runs the beamlets at n_high histories
    each and at every count of n_low (an int or a sequence; independent
    seeds), and each (low run, column) gives one window along the column's
    beamlet (:func:`oriented_windows`, centred on the high-history dose) at a
    random depth."""
    from .denoiser import loss_weight
    from .engine import B200Engine

    torch = _torch()
    rng = rng if rng is not None else np.random.default_rng(seed)
    engine = B200Engine(grid=grid, cross_sections=cross_sections, device=device)
    shape = tuple(grid.shape)
    hi = engine.run_dij_device(source, n_high, n_batches, seed + 7919, truncation=0.0)
    hi_dose, _, hi_sigma = dense_columns(hi, device, with_sigma=True)
    rho = torch.from_numpy(np.ascontiguousarray(grid.density, dtype=np.float32).ravel()).to(device)
    directions = beam_directions(source)
    depth_extent = np.array([shape[o >> 1] for o in orientation_codes(directions)])
    sets = []
    for k, n in enumerate(np.atleast_1d(n_low)):
        lo = engine.run_dij_device(source, int(n), n_batches, seed + 31 * k, truncation=0.0)
        lo_dose, lo_max, lo_sigma = dense_columns(lo, device, with_sigma=True)
        starts = rng.integers(0, np.maximum(depth_extent - window[2], 0) + 1)
        win = oriented_windows(hi_dose, shape, directions, window, starts, spacing=grid.spacing)
        scale = (1.0 / lo_max.clamp_min(1e-30))[win[:, 4].to(torch.int64)].view(-1, 1, 1, 1)
        x = gather_oriented(lo_dose, shape, win, window) * scale
        t = gather_oriented(hi_dose, shape, win, window) * scale
        s = gather_oriented(hi_sigma, shape, win, window) * scale
        d = gather_oriented(rho, shape, win, window, shared=True)
        e = gather_oriented(lo_sigma, shape, win, window) * scale
        sets.append(PairSet(x, t, s, d, loss_weight(t, s, precision), e))
        del lo_dose, lo_sigma
    del hi_dose, hi_sigma
    engine.drop_uploads()
    return concat(sets)


def concat(sets: list[PairSet]) -> PairSet:
    """One PairSet from many, field by field, releasing each field of the parts
    as soon as it is joined (peak memory: the parts plus one joined field)."""
    torch = _torch()
    out = {}
    for f in PAIR_FIELDS:
        out[f] = torch.cat([getattr(p, f) for p in sets])
        for p in sets:
            setattr(p, f, None)
    return PairSet(**out)


def train(net: UNet3D, pairs: PairSet, *, steps: int, batch: int = 4, seed: int = 0,
          lr_final: float | None = None, log_every: int = 100, log=None,
          keep_best: bool = True, warmup: int = 0) -> list[float]:
    """Adam steps over random mini-batches of the pairs; returns the mean loss of
    every ``log_every`` steps.  With lr_final the learning rate decays
    geometrically from net.lr to lr_final; the first ``warmup`` steps ramp it
    up linearly from zero (Adam's first steps move every parameter by about the
    learning rate, too far for a network that is already trained).  With
    keep_best the network ends with the parameters of the interval whose mean
    loss was lowest (a late divergence cannot lose a good network)."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    lr0 = net.lr
    history, acc = [], torch.zeros((), device=net.device)
    best, best_params = float("inf"), None
    n = len(pairs)
    for step in range(steps):
        net.lr = lr0
        if lr_final is not None:
            net.lr = lr0 * (lr_final / lr0) ** (step / max(steps - 1, 1))
        if step < warmup:
            net.lr *= (step + 1) / warmup
        idx = torch.randint(0, n, (batch,), generator=g).to(net.device)
        acc += net.train_step(pairs.inputs[idx].contiguous(), pairs.density[idx].contiguous(),
                              pairs.targets[idx].contiguous(), pairs.weight[idx].contiguous(),
                              pairs.noise[idx].contiguous())[0]
        if (step + 1) % log_every == 0:
            history.append(float(acc.item()) / log_every)
            acc.zero_()
            if keep_best and history[-1] < best:
                best, best_params = history[-1], net.p32.clone()
            if log is not None:
                log(f"step {step + 1}: loss {history[-1]:.5f} lr {net.lr:.2e}")
    net.lr = lr0
    if best_params is not None:
        net.p32.copy_(best_params)
        net.p16.copy_(best_params.to(net.p16.dtype))
    return history


# ---- the denoised Dij ------------------------------------------------------------------
def inference_window(grid_shape, lateral: int = 64, depth: int | None = None) -> tuple[int, int, int]:
    """The denoising window (wa, wb, wd): `lateral` voxels across (at most the
    smallest grid extent, a multiple of 8) and `depth` planes deep (default:
    the z extent rounded up to a multiple of 8, one chunk for beams along z)."""
    smallest = min(grid_shape)
    wa = min(lateral, smallest - smallest % 8) or 8
    wd = depth if depth is not None else -(-grid_shape[2] // 8) * 8
    return wa, wa, wd


def chunk_windows(n_win: int, window, chunk: int) -> int:
    """Windows per U-Net pass: at most `chunk`, equal passes (no padded work),
    and few enough that the network's widest activation — the level-0
    concatenation, LEVELS[0] + LEVELS[1] channels — stays below 2^31 elements
    (its element-wise kernels index 32-bit)."""
    per_window = int(np.prod(window)) * (LEVELS[0] + LEVELS[1])
    chunk = max(1, min(int(chunk), (2 ** 31 - 1) // per_window, max(1, n_win)))
    return -(-max(1, n_win) // -(-max(1, n_win) // chunk))


def denoise_dense(net: UNet3D, dose, colmax, density, grid_shape, *, sigma=None, window=None,
                  chunk: int = 100, out=None, directions=None, spacing=None):
    """Denoised dense columns, float64 [C, vox]: the Monte Carlo columns
    (float32 dose [C, vox] with their maxima and, optionally, their sigma; or
    `out`, float64, written in place) with every window along each column's
    beamlet replaced by the network's estimate.  `density` is the shared [vox]
    volume; `directions` [C, 3] the beamlets' travel directions (default +z)
    and `spacing` the voxel size (default isotropic)."""
    torch = _torch()
    window = window or inference_window(grid_shape)
    n = dose.shape[0]
    dirs = np.tile([0.0, 0.0, 1.0], (n, 1)) if directions is None else np.asarray(directions)
    win = oriented_windows(dose, grid_shape, dirs, window, spacing=spacing)
    if out is None:
        out = dose.to(torch.float64)
    scale = colmax[win[:, 4].to(torch.int64)].contiguous()
    n_win = win.shape[0]
    chunk = chunk_windows(n_win, window, chunk)
    for w0 in range(0, n_win, chunk):
        w1 = min(w0 + chunk, n_win)
        idx = torch.arange(w0, w0 + chunk, device=dose.device).clamp_max(n_win - 1)  # fixed batch shape
        wsel = win[idx].contiguous()
        x = gather_oriented(dose, grid_shape, wsel, window)
        rho = gather_oriented(density, grid_shape, wsel, window, shared=True)
        sg = None if sigma is None else gather_oriented(sigma, grid_shape, wsel, window)
        cm = scale[idx].contiguous()
        y = net.predict(x, rho, colmax=cm, sigma=sg)
        scatter_oriented(y[: w1 - w0], cm[: w1 - w0], grid_shape, wsel[: w1 - w0].contiguous(), out)
    return out


_COMPACT_CAPACITY: dict = {}  # (columns, voxels, device) -> entries to reserve next time


def compact(mean, sigma, truncation: float, to_host: bool = True):
    """Truncation + CSC of dense float64 columns on the device, through the
    allocation-free compaction entry point: (indptr, indices, dose, sigma) on
    the host, or (with to_host False) indptr on the host and the entries as
    device tensors."""
    torch = _torch()
    lib = _lib.load()
    n_cols, vox = mean.shape
    dev = mean.device
    # capacity: the last call's entry count of this shape plus slack (a call
    # that needs more is told so and runs again with the exact size); no
    # counting pass over the dense columns
    key = (n_cols, vox, str(dev))
    cap = _COMPACT_CAPACITY.get(key, 1 << 20)
    for _ in range(2):
        counts = torch.zeros(n_cols, dtype=torch.int64, device=dev)
        idx = torch.empty(cap, dtype=torch.int64, device=dev)
        dose = torch.empty(cap, dtype=torch.float64, device=dev)
        sig = torch.empty(cap, dtype=torch.float64, device=dev)
        nnz = C.c_int64()
        code = lib.pmc_dij_compact_static(C.c_void_p(mean.data_ptr()), C.c_void_p(sigma.data_ptr()),
                                          n_cols, vox, float(truncation), cap,
                                          C.c_void_p(counts.data_ptr()), C.c_void_p(idx.data_ptr()),
                                          C.c_void_p(dose.data_ptr()), C.c_void_p(sig.data_ptr()),
                                          C.byref(nnz), C.c_void_p(_stream(dev)))
        if code != _lib.PMC_ERR_CAPACITY:
            break
        cap = int(nnz.value) + 1  # the size this call needs
    if code != _lib.PMC_OK:
        raise RuntimeError(f"pmc_dij_compact_static failed ({code})")
    k = nnz.value
    _COMPACT_CAPACITY[key] = k + k // 16 + 1024
    indptr = np.zeros(n_cols + 1, dtype=np.int64)
    np.cumsum(counts.cpu().numpy(), out=indptr[1:])
    if not to_host:  # views: the capacity is at most ~6 % above the entries
        return indptr, idx[:k], dose[:k], sig[:k]
    return indptr, idx[:k].cpu().numpy(), dose[:k].cpu().numpy(), sig[:k].cpu().numpy()


def run_dij_denoised(engine, net: UNet3D | None, source, n_histories_per_beamlet, n_batches: int,
                     seed: int, *, truncation: float = 1.0e-3, lateral: int = 64,
                     depth: int | None = None, chunk: int = 100, to_host: bool = True,
                     timings: dict | None = None, group_columns: int | None = None,
                     overlap: bool = False):
    """A Dij from low-history Monte Carlo plus the denoiser: the engine runs the
    beamlets (``run_dij_device``), the windows along every column's beamlet
    (``lateral`` voxels across, ``depth`` planes per chunk; see
    :func:`oriented_windows`) are replaced by the network's estimate, and the
    dense columns are truncated and compacted to CSC on the device.  Columns
    go through in groups of ``group_columns`` (all at once when None: the dense
    maps of a group must fit the device), each group with the same history
    keys as in the whole Dij.  With ``overlap`` a group's denoising and
    compaction run on a second stream while the engine transports the next
    group (the engine's kernels are latency-bound, the U-Net's tensor-bound);
    ``timings`` then holds the whole call only.  With ``to_host`` False the
    CSC entries stay on the device (torch tensors in the result).  With ``net``
    None this is plain Monte Carlo (``engine.run_dij``), the method's fallback.

    The per-entry ``sigma`` of the result is the batch sigma of the
    low-history Monte Carlo input, not an uncertainty of the denoised value:
    the network's estimate is smoother than its input and is judged against
    high-statistics Monte Carlo instead (:func:`sigma_equivalent_error`,
    :func:`relative_bias`).  A consumer that weights entries by ``sigma``
    (a robust optimizer) reads the input's noise level."""
    import torch

    from .engine import ENERGY_QUANTUM_MEV, _result_types

    if net is None:
        return engine.run_dij(source, n_histories_per_beamlet, n_batches, seed,
                              truncation=truncation)
    n_cols = int(source.n_beamlets)
    counts = (np.full(n_cols, int(n_histories_per_beamlet), dtype=np.int64)
              if np.ndim(n_histories_per_beamlet) == 0
              else np.asarray(n_histories_per_beamlet, dtype=np.int64))
    directions = beam_directions(source)
    group = n_cols if not group_columns else int(group_columns)
    marks = []

    def mark(name):  # CUDA events between the stages, read when `timings` is given
        if timings is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            marks.append((name, ev))

    pieces, books, shape = [], np.zeros(4, dtype=np.int64), None
    rho = None
    pipelined = overlap and group < n_cols
    main = torch.cuda.current_stream()
    side = torch.cuda.Stream(device=main.device) if pipelined else None
    pending = None  # the previous group's dense mean and sigma, denoised on `side`

    def finish(item):
        with torch.cuda.stream(side):
            pieces.append(compact(item[0], item[1], truncation, to_host=False))

    mark("start")
    for lo in range(0, n_cols, group):
        hi = min(lo + group, n_cols)
        view = engine.run_dij_device(source, counts, n_batches, seed, truncation=0.0,
                                     columns=(lo, hi))
        device = torch.device(view.device)
        shape = tuple(view.grid_shape)
        if not pipelined:
            mark("monte_carlo")
        dose, colmax, sigma32 = dense_columns(view, device, with_sigma=True)
        mean, sigma = dense_columns_f64(view, device)
        books += np.asarray(view.books, dtype=np.int64)
        if rho is None:
            rho = _device_density(engine, device)
        window = inference_window(shape, lateral, depth)
        if pipelined:
            ready = torch.cuda.Event()
            ready.record(main)
            ready.synchronize()  # the engine's next run overwrites the CSC these were read from
            if pending is not None:
                finish(pending)
            side.wait_event(ready)
            for t in (dose, colmax, sigma32, mean, sigma, rho):
                t.record_stream(side)
            with torch.cuda.stream(side):
                denoise_dense(net, dose, colmax, rho, shape, sigma=sigma32, window=window,
                              chunk=chunk, out=mean, directions=directions[lo:hi],
                              spacing=engine.grid.spacing)
            pending = (mean, sigma)
            del dose, sigma32, mean, sigma
            continue
        mark("dense_columns")
        denoise_dense(net, dose, colmax, rho, shape, sigma=sigma32, window=window, chunk=chunk,
                      out=mean, directions=directions[lo:hi], spacing=engine.grid.spacing)
        del dose, sigma32
        mark("unet")
        pieces.append(compact(mean, sigma, truncation, to_host=False))
        del mean, sigma
        mark("compaction")
    if pipelined:
        finish(pending)
        pending = None
        main.wait_stream(side)
        for piece in pieces:
            for t in piece[1:]:
                t.record_stream(main)
        mark("pipelined")
    if timings is not None:
        marks[-1][1].synchronize()
        for (_, a), (name, b) in zip(marks, marks[1:]):
            timings[name] = timings.get(name, 0.0) + a.elapsed_time(b)
    indptr = np.zeros(n_cols + 1, dtype=np.int64)
    col = 0
    for ptr, *_ in pieces:
        k = len(ptr) - 1
        indptr[col + 1:col + k + 1] = indptr[col] + ptr[1:]
        col += k
    joined = [torch.cat([p[i] for p in pieces]) for i in (1, 2, 3)]
    if to_host:
        joined = [t.cpu().numpy() for t in joined]
    indices, dose_v, sigma_v = joined
    deposited, escaped, unscored, emitted = books
    _, _, DijResult = _result_types()
    return DijResult(
        grid_shape=shape, n_beamlets=n_cols,
        n_histories_per_beamlet=int(counts.max()), n_batches=n_batches, truncation=truncation,
        indptr=indptr, indices=indices, dose=dose_v, sigma=sigma_v,
        energy_emitted=float(emitted) * ENERGY_QUANTUM_MEV,
        energy_deposited=float(deposited) * ENERGY_QUANTUM_MEV,
        energy_escaped=float(escaped) * ENERGY_QUANTUM_MEV,
        energy_unscored=float(unscored) * ENERGY_QUANTUM_MEV,
        correlated=True)


# ---- error against high-statistics Monte Carlo ------------------------------------------
def sigma_equivalent_error(estimate, reference, reference_sigma=None, threshold: float = 0.5):
    """Per-column sigma-equivalent relative error of dense columns [C, vox]
    against a high-statistics reference, over the voxels where the reference is
    at least `threshold` of its column maximum: the median |est - ref| / ref
    divided by 0.6745 (the median of |N(0, 1)|), with the reference's own
    median relative sigma removed in quadrature.  For plain Monte Carlo this is
    the per-beamlet sigma (mean over columns of the median sigma/dose over the
    same voxels).  Returns a float64 numpy array, one value per column."""
    torch = _torch()
    est = estimate.to(torch.float64)
    ref = reference.to(torch.float64)
    out = np.zeros(ref.shape[0])
    for c in range(ref.shape[0]):
        r = ref[c]
        sel = r >= threshold * r.max()
        if not bool(sel.any()) or float(r.max()) <= 0.0:
            out[c] = np.nan
            continue
        rel = ((est[c][sel] - r[sel]).abs() / r[sel]).median().item() / 0.6745
        if reference_sigma is not None:
            own = (reference_sigma[c].to(torch.float64)[sel] / r[sel]).median().item()
            rel = float(np.sqrt(max(rel * rel - own * own, 0.0)))
        out[c] = rel
    return out


def relative_bias(estimate, reference, threshold: float = 0.1):
    """Per-column signed bias of dense columns [C, vox] against a
    high-statistics reference over the voxels where the reference is at least
    `threshold` of its column maximum: (mean of (est - ref) / ref, and the
    integral (sum est - sum ref) / sum ref).  Returns two float64 arrays."""
    torch = _torch()
    est = estimate.to(torch.float64)
    ref = reference.to(torch.float64)
    mean_rel = np.zeros(ref.shape[0])
    integral = np.zeros(ref.shape[0])
    for c in range(ref.shape[0]):
        r = ref[c]
        if float(r.max()) <= 0.0:
            mean_rel[c] = integral[c] = np.nan
            continue
        sel = r >= threshold * r.max()
        d = est[c][sel] - r[sel]
        mean_rel[c] = (d / r[sel]).mean().item()
        integral[c] = (d.sum() / r[sel].sum()).item()
    return mean_rel, integral


def error_report(estimate, reference, reference_sigma, thresholds=(0.5, 0.1, 0.01)) -> dict:
    """Sigma-equivalent error and signed bias (mean over columns) at each
    threshold of the column maximum: the beamlet core (0.5), the penumbra
    (0.1) and the low-dose tail the truncation keeps (0.01)."""
    out = {}
    for t in thresholds:
        err = sigma_equivalent_error(estimate, reference, reference_sigma, threshold=t)
        mean_rel, integral = relative_bias(estimate, reference, threshold=t)
        out[f"{t:g}"] = {"sigma_eq": float(np.nanmean(err)), "bias_mean": float(np.nanmean(mean_rel)),
                         "bias_integral": float(np.nanmean(integral))}
    return out
