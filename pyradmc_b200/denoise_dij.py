"""Dij columns through the denoiser: device-side conversion, windows, training
pairs, the denoised Dij and its error against high-statistics Monte Carlo.

No counterpart in pyRadMC.  Every step runs on the device through the C-ABI of
``include/pyradmc_b200_denoise.h`` (plus ``pmc_dij_compact_static`` for the
final truncation + CSC); torch allocates the buffers and supplies the stream.

Columns are dense volumes in the Dij's voxel order (x-major, z fastest).  Each
column is denoised in a lateral window centred on the column's dose centroid
over the full depth (the beamlets travel along +z); voxels outside the window
keep their Monte Carlo values.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from .denoiser import UNet3D, _check


def _torch():
    import torch

    return torch


def _stream(device) -> int:
    return _torch().cuda.current_stream(device).cuda_stream


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


def lateral_origins(dose, grid_shape, window: tuple[int, int, int], z0=None):
    """int32 [C, 3] window origins: laterally centred on each column's dose
    centroid (clamped into the grid), at depth z0 (0 when None; an array gives
    one depth per column)."""
    torch = _torch()
    nx, ny, nz = grid_shape
    wx, wy, _ = window
    vol = dose.view(-1, nx, ny, nz)
    lateral = vol.sum(dim=3)                                   # [C, nx, ny]
    total = lateral.sum(dim=(1, 2)).clamp_min(1e-30)
    xs = torch.arange(nx, device=dose.device, dtype=torch.float32)
    ys = torch.arange(ny, device=dose.device, dtype=torch.float32)
    cx = (lateral.sum(dim=2) * xs).sum(dim=1) / total
    cy = (lateral.sum(dim=1) * ys).sum(dim=1) / total
    ox = torch.clamp(torch.round(cx - wx / 2), 0, max(nx - wx, 0)).to(torch.int32)
    oy = torch.clamp(torch.round(cy - wy / 2), 0, max(ny - wy, 0)).to(torch.int32)
    if z0 is None:
        oz = torch.zeros_like(ox)
    else:
        oz = torch.as_tensor(z0, dtype=torch.int32, device=dose.device).expand_as(ox).contiguous()
    return torch.stack([ox, oy, oz], dim=1).contiguous()


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
    seeds), and each (low run, column) gives one window, laterally centred on
    the column's dose and at a random depth."""
    from .denoiser import loss_weight
    from .engine import B200Engine

    torch = _torch()
    rng = rng if rng is not None else np.random.default_rng(seed)
    engine = B200Engine(grid=grid, cross_sections=cross_sections, device=device)
    shape = tuple(grid.shape)
    hi = engine.run_dij_device(source, n_high, n_batches, seed + 7919, truncation=0.0)
    hi_dose, _, hi_sigma = dense_columns(hi, device, with_sigma=True)
    rho = torch.from_numpy(np.ascontiguousarray(grid.density, dtype=np.float32).ravel()).to(device)
    sets = []
    for k, n in enumerate(np.atleast_1d(n_low)):
        lo = engine.run_dij_device(source, int(n), n_batches, seed + 31 * k, truncation=0.0)
        lo_dose, lo_max, lo_sigma = dense_columns(lo, device, with_sigma=True)
        n_cols = lo.n_beamlets
        z0 = rng.integers(0, max(shape[2] - window[2], 0) + 1, size=n_cols)
        origins = lateral_origins(hi_dose, shape, window, z0)
        scale = (1.0 / lo_max.clamp_min(1e-30)).view(-1, 1, 1, 1)
        x = gather(lo_dose, shape, origins, window) * scale
        t = gather(hi_dose, shape, origins, window) * scale
        s = gather(hi_sigma, shape, origins, window) * scale
        d = gather(rho, shape, origins, window, shared=True)
        e = gather(lo_sigma, shape, origins, window) * scale
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
          keep_best: bool = True) -> list[float]:
    """Adam steps over random mini-batches of the pairs; returns the mean loss of
    every ``log_every`` steps.  With lr_final the learning rate decays
    geometrically from net.lr to lr_final.  With keep_best the network ends
    with the parameters of the interval whose mean loss was lowest (a late
    divergence cannot lose a good network)."""
    torch = _torch()
    g = torch.Generator(device="cpu").manual_seed(seed)
    lr0 = net.lr
    history, acc = [], torch.zeros((), device=net.device)
    best, best_params = float("inf"), None
    n = len(pairs)
    for step in range(steps):
        if lr_final is not None:
            net.lr = lr0 * (lr_final / lr0) ** (step / max(steps - 1, 1))
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
def inference_window(grid_shape, lateral: int = 64) -> tuple[int, int, int]:
    """The denoising window: `lateral` voxels (at most the grid, a multiple of 8)
    across, the full depth rounded up to a multiple of 8."""
    nx, ny, nz = grid_shape
    wx = min(lateral, nx - nx % 8) or 8
    wy = min(lateral, ny - ny % 8) or 8
    return wx, wy, -(-nz // 8) * 8


def denoise_dense(net: UNet3D, dose, colmax, density, grid_shape, *, sigma=None, window=None,
                  chunk: int = 32, out=None):
    """Denoised dense columns, float64 [C, vox]: the Monte Carlo columns
    (float32 dose [C, vox] with their maxima and, optionally, their sigma; or
    `out`, float64, written in place) with every column's window replaced by
    the network's estimate.  `density` is the shared [vox] volume."""
    torch = _torch()
    window = window or inference_window(grid_shape)
    origins = lateral_origins(dose, grid_shape, window)
    if out is None:
        out = dose.to(torch.float64)
    n = dose.shape[0]
    chunk = -(-n // -(-n // chunk))  # equal chunks of at most `chunk` windows: no padded work
    for c0 in range(0, n, chunk):
        c1 = min(c0 + chunk, n)
        idx = torch.arange(c0, c0 + chunk, device=dose.device).clamp_max(n - 1)  # fixed batch shape
        org = origins[idx].contiguous()
        x = gather(dose[idx].contiguous(), grid_shape, org, window)
        rho = gather(density, grid_shape, org, window, shared=True)
        sg = None if sigma is None else gather(sigma[idx].contiguous(), grid_shape, org, window)
        cm = colmax[idx].contiguous()
        y = net.predict(x, rho, colmax=cm, sigma=sg)
        scatter(y[: c1 - c0], cm[: c1 - c0], grid_shape, org[: c1 - c0].contiguous(),
                out[c0:c1])
    return out


def compact(mean, sigma, truncation: float, to_host: bool = True):
    """Truncation + CSC of dense float64 columns on the device, through the
    allocation-free compaction entry point: (indptr, indices, dose, sigma) on
    the host, or (with to_host False) indptr on the host and the entries as
    device tensors."""
    torch = _torch()
    lib = _lib.load()
    n_cols, vox = mean.shape
    dev = mean.device
    cap = int(torch.count_nonzero(mean).item()) + 1  # kept entries are non-zero
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
    if code != _lib.PMC_OK:
        raise RuntimeError(f"pmc_dij_compact_static failed ({code})")
    k = nnz.value
    indptr = np.zeros(n_cols + 1, dtype=np.int64)
    np.cumsum(counts.cpu().numpy(), out=indptr[1:])
    if not to_host:
        return indptr, idx[:k], dose[:k], sig[:k]
    return indptr, idx[:k].cpu().numpy(), dose[:k].cpu().numpy(), sig[:k].cpu().numpy()


def run_dij_denoised(engine, net: UNet3D | None, source, n_histories_per_beamlet, n_batches: int,
                     seed: int, *, truncation: float = 1.0e-3, lateral: int = 64, chunk: int = 32,
                     to_host: bool = True, timings: dict | None = None):
    """A Dij from low-history Monte Carlo plus the denoiser: the engine runs the
    beamlets (``run_dij_device``), every column's window around its beamlet is
    replaced by the network's estimate, and the dense columns are truncated and
    compacted to CSC on the device.  With ``to_host`` False the CSC entries
    stay on the device (torch tensors in the result).  With ``net`` None this is
    plain Monte Carlo (``engine.run_dij``), the method's fallback.

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
    marks = []

    def mark(name):  # CUDA events between the stages, read when `timings` is given
        if timings is not None:
            ev = torch.cuda.Event(enable_timing=True)
            ev.record()
            marks.append((name, ev))

    mark("start")
    view = engine.run_dij_device(source, n_histories_per_beamlet, n_batches, seed, truncation=0.0)
    device = torch.device(view.device)
    shape = tuple(view.grid_shape)
    mark("monte_carlo")
    dose, colmax, sigma32 = dense_columns(view, device, with_sigma=True)
    mean, sigma = dense_columns_f64(view, device)
    rho = torch.from_numpy(np.ascontiguousarray(engine.grid.density, dtype=np.float32).ravel()).to(device)
    mark("dense_columns")
    denoise_dense(net, dose, colmax, rho, shape, sigma=sigma32,
                  window=inference_window(shape, lateral), chunk=chunk, out=mean)
    del dose, sigma32
    mark("unet")
    indptr, indices, dose_v, sigma_v = compact(mean, sigma, truncation, to_host=to_host)
    mark("compaction")
    if timings is not None:
        marks[-1][1].synchronize()
        for (_, a), (name, b) in zip(marks, marks[1:]):
            timings[name] = timings.get(name, 0.0) + a.elapsed_time(b)
    deposited, escaped, unscored, emitted = view.books
    counts = np.asarray(view.counts)
    _, _, DijResult = _result_types()
    return DijResult(
        grid_shape=shape, n_beamlets=view.n_beamlets,
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
