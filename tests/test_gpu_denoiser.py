"""The denoiser's kernels against the float32 CPU oracle (torch conv3d + autograd).

Every convolution entry point (forward, data gradient through the flipped
weights, weight gradient), the pooling and joining kernels with their
gradients, and the whole U-Net's parameter gradient are compared with the
oracle on the same bf16-rounded operands.  Tolerances: the kernels accumulate
in fp32 like the oracle, so what separates them is the bf16 rounding of a
kernel's OUTPUT (relative 2^-8) and of intermediate activations in the full
network; the fp32 weight gradient differs only in summation order.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle.unet import OracleUNet, bf16, conv3d_reference
from pyradmc_b200 import _lib
from pyradmc_b200.denoiser import LEVELS, UNet3D, init_parameters, kpad_for, layout

pytestmark = pytest.mark.gpu

BF16_REL = 2.0 ** -8


def _dev(a, dtype):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0").to(dtype)


def _weights(rng, cin, cout):
    kpad = kpad_for(cin)
    w = np.zeros((cout, kpad), dtype=np.float32)
    w[:, :27 * cin] = bf16(rng.normal(0, np.sqrt(2.0 / (27 * cin)), (cout, 27 * cin)))
    return w, kpad


CONV_SHAPES = [
    # (n, d, h, w, cin, cout): ragged voxel counts, non-cubic grids, every cout tile
    (1, 8, 8, 8, 8, 16),
    (2, 6, 5, 7, 16, 8),
    (1, 4, 8, 6, 48, 16),
    (1, 8, 8, 8, 96, 32),
    (2, 4, 4, 4, 192, 64),
    (1, 4, 6, 4, 64, 48),
    (1, 4, 4, 4, 128, 96),
    (1, 2, 4, 4, 64, 128),
    (1, 2, 2, 4, 128, 192),
]


@pytest.mark.parametrize("shape", CONV_SHAPES)
def test_conv3d_forward_matches_oracle(gpu, shape):
    import torch

    n, d, h, w, cin, cout = shape
    rng = np.random.default_rng(sum(shape) * 31 + cin)
    x = bf16(rng.normal(size=(n, d, h, w, cin)))
    wt, kpad = _weights(rng, cin, cout)
    bias = rng.normal(size=cout).astype(np.float32)
    lib = _lib.load()
    dx, dw, db = _dev(x, torch.bfloat16), _dev(wt, torch.bfloat16), _dev(bias, torch.float32)
    for relu in (0, 1):
        y = torch.full((n, d, h, w, cout), float("nan"), dtype=torch.bfloat16, device=gpu)
        assert lib.pmd_conv3d(dx.data_ptr(), dw.data_ptr(), db.data_ptr(), y.data_ptr(), n, d, h, w,
                              cin, cout, kpad, relu, None) == 0
        got = y.float().cpu().numpy()
        ref = conv3d_reference(x, wt, bias, cin, cout, kpad, bool(relu))
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, ref, rtol=BF16_REL, atol=1e-5 * np.abs(ref).max())


WGRAD_SHAPES = [
    # every (cin, cout) of the network, partial tiles in d, h and w, one tile
    # (cin = 8 with its zero partner plane) up to several tiles per CTA, and
    # tap groups x channel groups for the wide layers
    (1, 8, 8, 8, 8, 16), (1, 3, 17, 9, 8, 16), (2, 6, 5, 7, 16, 32), (1, 4, 6, 4, 64, 64), (1, 4, 4, 4, 192, 64),
    (1, 4, 4, 8, 48, 16), (1, 2, 4, 4, 128, 128), (1, 3, 17, 9, 16, 16), (1, 2, 3, 9, 96, 32),
    (2, 16, 32, 24, 48, 16), (1, 32, 64, 64, 16, 16), (1, 8, 16, 16, 32, 32),
]


def _wgrad_plan(lib, shape):
    import ctypes

    info = (ctypes.c_int * 8)()
    return list(info) if lib.pmd_conv3d_wgrad_plan(*shape, info) == 0 else None


@pytest.mark.parametrize("shape", WGRAD_SHAPES)
def test_conv3d_weight_gradient_matches_oracle(gpu, shape):
    """The tensor-core weight gradient (default) and the mma.sync one
    (pmd_conv3d_impl(1)) against torch's fp32 conv3d_weight on the same bf16
    operands."""
    import torch
    from torch.nn.grad import conv3d_weight

    n, d, h, w, cin, cout = shape
    rng = np.random.default_rng(7 + cin + cout + d)
    x = bf16(rng.normal(size=(n, d, h, w, cin)))
    g = bf16(rng.normal(size=(n, d, h, w, cout)))
    kpad = kpad_for(cin)
    lib = _lib.load()
    assert _wgrad_plan(lib, shape) is not None  # the tensor-core kernel covers every layer
    dx, dg = _dev(x, torch.bfloat16), _dev(g, torch.bfloat16)
    xt = torch.from_numpy(x.transpose(0, 4, 1, 2, 3).copy())
    gt = torch.from_numpy(g.transpose(0, 4, 1, 2, 3).copy())
    ref = conv3d_weight(xt.double(), (cout, cin, 3, 3, 3), gt.double(), padding=1)
    ref_flat = np.zeros((cout, kpad), dtype=np.float64)
    ref_flat[:, :27 * cin] = ref.numpy().transpose(0, 2, 3, 4, 1).reshape(cout, -1)
    ref_b = g.astype(np.float64).reshape(-1, cout).sum(0)
    scale = np.abs(ref_flat).max()
    m = n * d * h * w
    got = {}
    previous = lib.pmd_conv3d_impl(-1)
    try:
        for impl in (0, 1):
            lib.pmd_conv3d_impl(impl)
            dw = torch.zeros((cout, kpad), dtype=torch.float32, device=gpu)
            db = torch.zeros(cout, dtype=torch.float32, device=gpu)
            assert lib.pmd_conv3d_wgrad(dx.data_ptr(), dg.data_ptr(), dw.data_ptr(), db.data_ptr(),
                                        n, d, h, w, cin, cout, kpad, None) == 0
            got[impl] = (dw.cpu().numpy(), db.cpu().numpy())
    finally:
        lib.pmd_conv3d_impl(previous)
    assert lib.pmd_conv3d_failures() == 0
    for impl, (gw, gb) in got.items():
        # fp32 sums of m products of bf16 values in an unfixed order
        np.testing.assert_allclose(gw, ref_flat, rtol=1e-4, atol=1e-6 * scale * max(1.0, m / 4096),
                                   err_msg=f"impl {impl}")
        np.testing.assert_allclose(gb, ref_b, rtol=1e-4, atol=1e-4 * np.abs(g).sum(0).max(),
                                   err_msg=f"impl {impl}")
        assert (gw[:, 27 * cin:] == 0).all()


@pytest.mark.parametrize("shape", [(1, 8, 8, 8, 16, 16), (2, 6, 5, 7, 48, 16), (1, 4, 6, 4, 96, 32),
                                   (1, 4, 4, 4, 192, 64), (1, 2, 4, 4, 64, 128),
                                   (1, 4, 4, 4, 128, 64), (1, 4, 4, 4, 32, 16)])
def test_conv3d_data_gradient_matches_oracle(gpu, shape):
    import torch
    from torch.nn.grad import conv3d_input

    n, d, h, w, cin, cout = shape
    rng = np.random.default_rng(11 + cin + cout)
    wt, kpad = _weights(rng, cin, cout)
    g = bf16(rng.normal(size=(n, d, h, w, cout)))
    kpad_d = kpad_for(cout)
    lib = _lib.load()
    dwt = _dev(wt, torch.bfloat16)
    wd = torch.zeros((cin, kpad_d), dtype=torch.bfloat16, device=gpu)
    assert lib.pmd_flip_weights(dwt.data_ptr(), wd.data_ptr(), cin, cout, kpad, kpad_d, None) == 0
    gx = torch.empty((n, d, h, w, cin), dtype=torch.bfloat16, device=gpu)
    dg = _dev(g, torch.bfloat16)
    assert lib.pmd_conv3d(dg.data_ptr(), wd.data_ptr(), None, gx.data_ptr(), n, d, h, w, cout, cin,
                          kpad_d, 0, None) == 0
    w5 = wt[:, :27 * cin].reshape(cout, 3, 3, 3, cin).transpose(0, 4, 1, 2, 3).copy()
    ref = conv3d_input((n, cin, d, h, w), torch.from_numpy(w5),
                       torch.from_numpy(g.transpose(0, 4, 1, 2, 3).copy()), padding=1)
    ref = ref.numpy().transpose(0, 2, 3, 4, 1)
    got = gx.float().cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=BF16_REL, atol=1e-5 * np.abs(ref).max())


def test_pool_upcat_and_their_gradients(gpu):
    import torch
    import torch.nn.functional as F

    rng = np.random.default_rng(3)
    n, d, h, w, c_up, c_skip = 2, 8, 4, 6, 16, 8
    lib = _lib.load()
    x = bf16(rng.normal(size=(n, d, h, w, c_skip)))
    dx = _dev(x, torch.bfloat16)
    y = torch.empty((n, d // 2, h // 2, w // 2, c_skip), dtype=torch.bfloat16, device=gpu)
    assert lib.pmd_avgpool(dx.data_ptr(), y.data_ptr(), n, d, h, w, c_skip, None) == 0
    ref = F.avg_pool3d(torch.from_numpy(x.transpose(0, 4, 1, 2, 3).copy()), 2).numpy().transpose(0, 2, 3, 4, 1)
    np.testing.assert_allclose(y.float().cpu().numpy(), ref, rtol=BF16_REL, atol=1e-6)

    gy = bf16(rng.normal(size=tuple(y.shape)))
    prior = bf16(rng.normal(size=x.shape))
    gx = _dev(prior, torch.bfloat16)
    assert lib.pmd_avgpool_grad(_dev(gy, torch.bfloat16).data_ptr(), gx.data_ptr(), n, d, h, w,
                                c_skip, 1, None) == 0
    up = np.repeat(np.repeat(np.repeat(gy, 2, 1), 2, 2), 2, 3) / 8.0
    np.testing.assert_allclose(gx.float().cpu().numpy(), prior + up, rtol=BF16_REL, atol=1e-6)

    upin = bf16(rng.normal(size=(n, d // 2, h // 2, w // 2, c_up)))
    dup = _dev(upin, torch.bfloat16)
    out = torch.empty((n, d, h, w, c_up + c_skip), dtype=torch.bfloat16, device=gpu)
    assert lib.pmd_upcat(dup.data_ptr(), dx.data_ptr(), out.data_ptr(), n, d, h, w, c_up, c_skip,
                         None) == 0
    ref = np.concatenate([np.repeat(np.repeat(np.repeat(upin, 2, 1), 2, 2), 2, 3), x], axis=-1)
    np.testing.assert_array_equal(out.float().cpu().numpy(), ref)

    gout = bf16(rng.normal(size=ref.shape))
    dgout = _dev(gout, torch.bfloat16)
    gup = torch.empty_like(dup)
    gskip = torch.empty_like(dx)
    assert lib.pmd_upcat_grad(dgout.data_ptr(), gup.data_ptr(), gskip.data_ptr(), n, d, h, w, c_up,
                              c_skip, 0, None) == 0
    ref_up = gout[..., :c_up].reshape(n, d // 2, 2, h // 2, 2, w // 2, 2, c_up).sum((2, 4, 6))
    np.testing.assert_allclose(gup.float().cpu().numpy(), ref_up, rtol=BF16_REL, atol=1e-5)
    np.testing.assert_array_equal(gskip.float().cpu().numpy(), gout[..., c_up:])


def _batch(rng, b, s):
    """A smooth positive dose-like field with noise, its clean version, a
    density and a loss weight; noisy and density are exact in bf16 (the
    kernels' input rounding)."""
    z, y, x = np.meshgrid(*(np.arange(s),) * 3, indexing="ij")
    clean = np.exp(-((x - s / 2) ** 2 + (y - s / 2) ** 2) / (0.1 * s * s)) * np.exp(-z / (2.0 * s))
    clean = np.ascontiguousarray(np.broadcast_to(clean, (b, s, s, s)), dtype=np.float32)
    noisy = bf16(clean * (1 + 0.3 * rng.normal(size=clean.shape)))
    density = bf16(1.0 + 0.2 * rng.random((b, s, s, s)))
    weight = rng.random((b, s, s, s)).astype(np.float32)
    return noisy, density, clean, weight


def test_unet_gradients_match_oracle(gpu):
    import torch

    rng = np.random.default_rng(5)
    params = init_parameters(seed=3)
    layers, head_w, head_b, _ = layout()
    params[head_w:head_w + LEVELS[0]] = rng.normal(0, 0.5, LEVELS[0])  # non-zero head: gradients flow
    params[head_b] = 0.01
    for l in layers:  # the kernels read bf16 convolution weights: give the oracle the same
        sl = slice(l.w_off, l.w_off + l.cout * l.kpad)
        params[sl] = bf16(params[sl])
    noisy, density, clean, weight = _batch(rng, 2, 16)
    sigma = bf16(0.3 * clean)  # the Monte Carlo sigma channel
    net = UNet3D(gpu, params=params, loss_lambda=0.5)
    loss, grad = net.gradients(_dev(noisy, torch.float32), _dev(density, torch.float32),
                               _dev(clean, torch.float32), _dev(weight, torch.float32),
                               _dev(sigma, torch.float32))
    torch.cuda.synchronize()
    got = grad.cpu().numpy()
    ref_loss, ref = OracleUNet(params).gradients(torch.from_numpy(noisy), torch.from_numpy(density),
                                                 torch.from_numpy(clean), torch.from_numpy(weight),
                                                 0.5, torch.from_numpy(sigma))
    assert abs(float(loss.item()) - ref_loss) <= 0.02 * ref_loss
    for l in layers:
        for off, size in ((l.w_off, l.cout * l.kpad), (l.b_off, l.cout)):
            a, b = got[off:off + size], ref[off:off + size]
            cos = float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b) + 1e-30))
            rel = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
            assert cos > 0.99 and rel < 0.15, (l.name, off == l.b_off, cos, rel)
    hw = slice(head_w, head_w + LEVELS[0])
    np.testing.assert_allclose(got[hw], ref[hw], rtol=0.05, atol=0.02 * np.abs(ref[hw]).max())


def test_zero_head_network_is_the_identity_and_training_reduces_the_loss(gpu):
    import torch

    rng = np.random.default_rng(9)
    noisy, density, clean, weight = _batch(rng, 2, 16)
    target = clean + 0.2  # an offset the network must learn on top of the denoising
    net = UNet3D(gpu, seed=1, lr=2e-3)
    p0 = net.parameters()
    args = [_dev(a, torch.float32) for a in (noisy, density, target, weight)]
    out = net.predict(args[0], args[1]).cpu().numpy()
    np.testing.assert_array_equal(out, noisy)  # zero head: prediction = input dose
    losses = [float(net.train_step(*args).item()) for _ in range(150)]
    assert np.isfinite(losses).all()
    assert np.mean(losses[-5:]) < 0.6 * losses[0], losses[::10]
    p = net.parameters()
    assert np.isfinite(p).all()
    for l in layout()[0]:
        w, w0 = (q[l.w_off:l.w_off + l.cout * l.kpad].reshape(l.cout, l.kpad) for q in (p, p0))
        assert (w[:, 27 * l.cin:] == 0).all(), l.name  # K padding stays zero through Adam
        assert np.abs(w - w0).max() > 1e-3, l.name     # every layer received gradients


UMMA_SHAPES = [
    # (n, d, h, w, cin, cout): partial tiles in every dimension, cin = 8 tap
    # pairing, one- and multi-pass weights, every N the network uses, and
    # enough tiles that every CTA runs several (pipelined buffers alternate)
    (2, 64, 64, 72, 48, 16),
    (1, 33, 40, 24, 16, 48),
    (1, 4, 16, 8, 8, 16),
    (1, 3, 20, 12, 16, 16),
    (2, 5, 17, 9, 48, 16),
    (1, 4, 16, 16, 16, 48),
    (1, 2, 18, 10, 32, 32),
    (1, 3, 16, 8, 32, 96),
    (1, 3, 18, 10, 96, 32),
    (1, 2, 16, 16, 64, 64),
    (1, 2, 8, 8, 64, 192),
    (1, 2, 8, 8, 64, 128),
    # beyond the single-buffered kernel: weights streamed in channel groups
    (1, 2, 16, 16, 192, 64),
    (2, 3, 8, 8, 128, 128),
]

SMEM_MAX = 232448


def _umma_single_pass(cin, cout):
    """Whether the single-buffered tensor-memory kernel stages every weight at
    once (its plan's shared-memory arithmetic)."""
    if cin > 96:
        return False
    cpt = cin // 8
    tz = 4 if cin <= 16 and cout <= 16 else (2 if cin <= 48 else 1)
    chunks = 27 * cpt + (1 if cpt == 1 else 0)
    return (tz + 2) * 180 * 16 * cpt + 256 + 16 + chunks * (cout * 16 + 8) <= SMEM_MAX


def _plan(lib, shape, impl):
    import ctypes

    info = (ctypes.c_int * 8)()
    previous = lib.pmd_conv3d_impl(impl)
    try:
        assert lib.pmd_conv3d_plan(*shape, info) == 0
    finally:
        lib.pmd_conv3d_impl(previous)
    return list(info)


@pytest.mark.parametrize("shape", UMMA_SHAPES)
def test_tensor_memory_convolution_matches_oracle(gpu, shape):
    """The tcgen05/TMEM kernels (each forced) against the oracle, and against
    the mma.sync kernel on the same operands."""
    import torch

    n, d, h, w, cin, cout = shape
    rng = np.random.default_rng(100 + sum(shape))
    x = bf16(rng.normal(size=(n, d, h, w, cin)))
    wt, kpad = _weights(rng, cin, cout)
    bias = rng.normal(size=cout).astype(np.float32)
    lib = _lib.load()
    dx, dw, db = _dev(x, torch.bfloat16), _dev(wt, torch.bfloat16), _dev(bias, torch.float32)
    ref = conv3d_reference(x, wt, bias, cin, cout, kpad, True)
    outs = {}
    previous = lib.pmd_conv3d_impl(-1)
    try:
        # warp-specialized, pipelined and single-buffered tensor memory, mma.sync
        for impl in (4, 3, 2, 1):
            lib.pmd_conv3d_impl(impl)
            y = torch.full((n, d, h, w, cout), float("nan"), dtype=torch.bfloat16, device=gpu)
            code = lib.pmd_conv3d(dx.data_ptr(), dw.data_ptr(), db.data_ptr(), y.data_ptr(), n, d, h,
                                  w, cin, cout, kpad, 1, None)
            if impl == 3 and code == -1:
                continue  # weights in several passes: no pipelined plan
            if impl == 2 and code == -1 and cin > 96:
                continue  # outside the single-buffered kernel
            assert code == 0, impl
            torch.cuda.synchronize()
            outs[impl] = y.float().cpu().numpy()
    finally:
        lib.pmd_conv3d_impl(previous)
    assert lib.pmd_conv3d_failures() == 0
    for impl, got in outs.items():
        assert np.isfinite(got).all(), impl
        np.testing.assert_allclose(got, ref, rtol=BF16_REL, atol=1e-5 * np.abs(ref).max(),
                                   err_msg=f"impl {impl}")
    # all accumulate the same products in fp32: at most a bf16 rounding step apart
    np.testing.assert_allclose(outs[4], outs[1], rtol=2 * BF16_REL, atol=1e-5 * np.abs(ref).max())
    if 2 in outs:
        np.testing.assert_allclose(outs[2], outs[1], rtol=2 * BF16_REL, atol=1e-5 * np.abs(ref).max())
    if 3 in outs:  # the same MMAs in the same order: identical
        np.testing.assert_array_equal(outs[3], outs[2])
    ws = _plan(lib, shape, 4)
    if ws[2] == 1 and ws[4] == 0 and 2 in outs and _umma_single_pass(cin, cout):
        # one channel group, resident weights: the same MMAs in the same order
        np.testing.assert_array_equal(outs[4], outs[2])


def test_tensor_memory_path_rejects_what_it_does_not_cover(gpu):
    lib = _lib.load()
    previous = lib.pmd_conv3d_impl(2)
    try:  # cin = 128 is outside the tensor-memory kernel: nothing launched
        assert lib.pmd_conv3d(None, None, None, None, 1, 2, 2, 2, 128, 128, kpad_for(128), 1,
                              None) == -1
    finally:
        lib.pmd_conv3d_impl(previous)


def _oriented_reference(src, shape, win, window):
    """numpy restatement of the oriented window map: (a, b, k) -> grid voxel."""
    wa, wb, wd = window
    out = np.zeros((len(win), wa, wb, wd), dtype=np.float32)
    where = np.full((len(win), wa, wb, wd), -1, dtype=np.int64)
    for n, (ox, oy, oz, orient, col, q1, q2) in enumerate(win):
        d, f = orient >> 1, orient & 1
        l1, l2 = [a for a in range(3) if a != d]
        o = (ox, oy, oz)
        for a in range(wa):
            for b in range(wb):
                for k in range(wd):
                    s1, s2 = (k * int(q1) + 32768) >> 16, (k * int(q2) + 32768) >> 16
                    g = [0, 0, 0]
                    g[l1], g[l2] = o[l1] + a + s1, o[l2] + b + s2
                    g[d] = o[d] + (wd - 1 - k if f else k)
                    if all(0 <= g[i] < shape[i] for i in range(3)):
                        flat = (g[0] * shape[1] + g[1]) * shape[2] + g[2]
                        out[n, a, b, k] = src[col, flat]
                        where[n, a, b, k] = col * int(np.prod(shape)) + flat
    return out, where


def test_oriented_window_gather_and_scatter(gpu):
    """Every orientation, shears of up to one voxel per plane either way,
    windows partly outside the grid, several windows per column: the CUDA
    gather against the numpy map, and the scatter writes max(x, 0) * scale into
    exactly the gathered voxels."""
    import torch

    from pyradmc_b200 import denoise_dij as D

    shape, window = (9, 7, 6), (4, 3, 5)
    rng = np.random.default_rng(7)
    src = rng.normal(size=(3, int(np.prod(shape)))).astype(np.float32)
    win = np.array([[ox, oy, oz, orient, col, q1, q2] for orient in range(6) for col in range(3)
                    for ox, oy, oz in [tuple(rng.integers(-3, 8, size=3))]
                    for q1, q2 in [tuple(rng.integers(-65536, 65537, size=2))]], dtype=np.int32)
    ref, where = _oriented_reference(src, shape, win, window)
    dsrc = torch.from_numpy(src).to(gpu)
    dwin = torch.from_numpy(win).to(gpu)
    got = D.gather_oriented(dsrc, shape, dwin, window).cpu().numpy()
    np.testing.assert_array_equal(got, ref)
    # scatter, one window per (orientation, column) pair at a time (windows of
    # one column must not overlap)
    for n in range(len(win)):
        dst = torch.full((3, int(np.prod(shape))), -7.0, dtype=torch.float64, device=gpu)
        data = torch.from_numpy(rng.normal(size=(1, *window)).astype(np.float32)).to(gpu)
        scale = torch.tensor([2.5], dtype=torch.float32, device=gpu)
        D.scatter_oriented(data, scale, shape, dwin[n:n + 1].contiguous(), dst)
        expect = np.full(3 * int(np.prod(shape)), -7.0)
        sel = where[n] >= 0
        expect[where[n][sel]] = np.maximum(data.cpu().numpy()[0][sel], 0.0) * 2.5
        np.testing.assert_allclose(dst.cpu().numpy().ravel(), expect, rtol=1e-7)


@pytest.mark.parametrize("shape", [(2, 5, 17, 9, 16, 16), (1, 8, 32, 24, 16, 16), (1, 3, 18, 10, 32, 32)])
def test_head_fused_into_the_last_convolution_is_bit_identical(gpu, shape):
    """pmd_conv3d_head (the 1x1x1 head in the warp-specialized kernel's
    epilogue) against pmd_conv3d then pmd_head: the same bf16 features and the
    same float32 sum in channel order, so equal bit for bit."""
    import torch

    n, d, h, w, cin, cout = shape
    rng = np.random.default_rng(7 + sum(shape))
    x = bf16(rng.normal(size=(n, d, h, w, cin)))
    wt, kpad = _weights(rng, cin, cout)
    bias = rng.normal(size=cout).astype(np.float32)
    hw = rng.normal(size=cout).astype(np.float32)
    hb = np.array([0.25], np.float32)
    m = n * d * h * w
    base = rng.normal(size=m).astype(np.float32)
    lib = _lib.load()
    dx, dw = _dev(x, torch.bfloat16), _dev(wt, torch.bfloat16)
    db, dhw, dhb, dbase = (_dev(a, torch.float32) for a in (bias, hw, hb, base))
    for with_base in (True, False):
        feat = torch.empty((m, cout), dtype=torch.bfloat16, device=gpu)
        two = torch.full((m,), float("nan"), dtype=torch.float32, device=gpu)
        one = torch.full((m,), float("nan"), dtype=torch.float32, device=gpu)
        bp = dbase.data_ptr() if with_base else None
        assert lib.pmd_conv3d(dx.data_ptr(), dw.data_ptr(), db.data_ptr(), feat.data_ptr(), n, d, h, w,
                              cin, cout, kpad, 1, None) == 0
        assert lib.pmd_head(feat.data_ptr(), dhw.data_ptr(), dhb.data_ptr(), bp, two.data_ptr(), m,
                            cout, None) == 0
        assert lib.pmd_conv3d_head(dx.data_ptr(), dw.data_ptr(), db.data_ptr(), dhw.data_ptr(),
                                   dhb.data_ptr(), bp, one.data_ptr(), n, d, h, w, cin, cout, kpad, 1,
                                   None) == 0
        torch.cuda.synchronize()
        a, b = one.cpu().numpy(), two.cpu().numpy()
        assert np.isfinite(a).all()
        np.testing.assert_array_equal(a, b)
    assert lib.pmd_conv3d_failures() == 0
    # outside the kernel (cin = 8 is not a warp-specialized shape): nothing launched
    assert lib.pmd_conv3d_head(dx.data_ptr(), dw.data_ptr(), db.data_ptr(), dhw.data_ptr(),
                               dhb.data_ptr(), None, one.data_ptr(), n, d, h, w, 4, cout, kpad, 1,
                               None) == -1


def test_predict_with_the_fused_head_equals_the_unfused_network(gpu):
    import torch

    rng = np.random.default_rng(12)
    params = init_parameters(seed=4)
    _, head_w, head_b, _ = layout()
    params[head_w:head_w + LEVELS[0]] = rng.normal(0, 0.5, LEVELS[0])
    params[head_b] = 0.01
    noisy, density, _, _ = _batch(rng, 2, 16)
    net = UNet3D(gpu, params=params)
    args = (_dev(noisy, torch.float32), _dev(density, torch.float32))
    fused = net.predict(*args).clone()
    launches = net.launches
    net.fuse_head = False
    plain = net.predict(*args).clone()
    assert net.launches - launches == launches + 1  # one more launch: the separate head
    np.testing.assert_array_equal(fused.cpu().numpy(), plain.cpu().numpy())
    assert not np.array_equal(plain.cpu().numpy(), noisy)  # the head contributes
