"""The denoiser's host side without a GPU: parameter layout, the oracle's
weight-layout conversions (pinned against a direct loop over the taps), argument
checks of the C-ABI that return before any launch, and the no-CPU-fallback rule."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle.unet import OracleUNet, conv3d_reference, conv_weight, weight_to_flat
from pyradmc_b200 import _lib
from pyradmc_b200.denoiser import (IN_CHANNELS, LEVELS, forward_flops_per_voxel, init_parameters,
                                   kpad_for, layout)
from tests.conftest import cuda_available


def test_layout_is_aligned_and_padded():
    layers, head_w, head_b, n = layout()
    assert [l.cout for l in layers] == [16, 16, 32, 32, 64, 64, 128, 128, 64, 64, 32, 32, 16, 16]
    assert layers[0].cin == IN_CHANNELS and layers[8].cin == LEVELS[3] + LEVELS[2]
    ends = 0
    for l in layers:
        assert l.kpad % 64 == 0 and l.kpad >= 27 * l.cin and l.kpad - 27 * l.cin < 64
        assert l.w_off % 64 == 0 and l.b_off % 64 == 0 and l.w_off >= ends
        ends = l.b_off + l.cout
    assert head_w % 64 == 0 and head_b > head_w and n > head_b
    p = init_parameters(0)
    assert p.shape == (n,) and p.dtype == np.float32
    for l in layers:
        w = p[l.w_off:l.w_off + l.cout * l.kpad].reshape(l.cout, l.kpad)
        assert (w[:, 27 * l.cin:] == 0).all() and w[:, :27 * l.cin].std() > 0
    assert (p[head_w:head_b + 1] == 0).all()
    assert kpad_for(8) == 256 and kpad_for(128) == 3456 and kpad_for(48) == 1344
    # 2*27*(8*16 + 16*16 + 48*16 + 16*16) at full resolution plus the coarser levels
    assert 130_000 < forward_flops_per_voxel() < 140_000


def test_oracle_convolution_follows_the_tap_order_of_the_kernels():
    rng = np.random.default_rng(1)
    n, d, h, w, cin, cout = 1, 3, 4, 5, 8, 2
    kpad = kpad_for(cin)
    x = rng.normal(size=(n, d, h, w, cin)).astype(np.float32)
    wt = np.zeros((cout, kpad), dtype=np.float32)
    wt[:, :27 * cin] = rng.normal(size=(cout, 27 * cin))
    ref = np.zeros((n, d, h, w, cout))
    for z in range(d):
        for y in range(h):
            for xx in range(w):
                for tap in range(27):
                    zz, yy, x3 = z + tap // 9 - 1, y + (tap // 3) % 3 - 1, xx + tap % 3 - 1
                    if 0 <= zz < d and 0 <= yy < h and 0 <= x3 < w:
                        ref[0, z, y, xx] += wt[:, tap * cin:(tap + 1) * cin] @ x[0, zz, yy, x3]
    got = conv3d_reference(x, wt, None, cin, cout, kpad, relu=False)
    np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-5)


def test_weight_conversions_round_trip():
    layers, *_ = layout()
    p = init_parameters(2)
    for l in layers[:3]:
        w = conv_weight(p, l)
        assert tuple(w.shape) == (l.cout, l.cin, 3, 3, 3)
        np.testing.assert_array_equal(weight_to_flat(w, l), p[l.w_off:l.w_off + l.cout * l.kpad])


def test_oracle_network_with_a_zero_head_is_the_identity():
    rng = np.random.default_rng(0)
    dose = torch.from_numpy(rng.random((1, 8, 8, 8)).astype(np.float32))
    rho = torch.ones_like(dose)
    out = OracleUNet(init_parameters(0)).forward(dose, rho)
    assert torch.equal(out, dose)


def test_abi_rejects_unsupported_shapes_before_launching():
    lib = _lib.load()
    assert lib.pmd_conv3d(None, None, None, None, 1, 8, 8, 8, 8, 24, 256, 1, None) == -1  # cout
    assert lib.pmd_conv3d(None, None, None, None, 1, 8, 8, 8, 12, 16, 384, 1, None) == -1  # cin
    assert lib.pmd_conv3d(None, None, None, None, 1, 8, 8, 8, 8, 16, 200, 1, None) == -1  # kpad
    assert lib.pmd_conv3d_wgrad(None, None, None, None, 1, 8, 8, 8, 8, 8, 256, None) == -1
    assert lib.pmd_head_grad(None, None, None, None, None, None, 10, 65, None) == -1
    assert lib.pmd_csc_to_dense(None, None, None, 70000, 1, None, None, None) == -1
    assert lib.pmd_avgpool(None, None, 1, 3, 4, 4, 8, None) == -1
    assert lib.pmd_adam(None, None, None, None, None, 10, 1e-3, 0.9, 0.999, 1e-8, 0, None) == -1


@pytest.mark.skipif(cuda_available(), reason="checks the no-device behaviour")
def test_network_refuses_to_run_without_a_cuda_device():
    from pyradmc_b200.denoiser import UNet3D

    with pytest.raises(RuntimeError, match="CUDA device only"):
        UNet3D("cuda:0")


def test_convolution_plans_of_the_network_layers():
    """pmd_conv3d_plan is host arithmetic: the default path's kernel and plan
    for every layer of a 16-window inference chunk (64 x 64 x 128 windows)."""
    import ctypes

    lib = _lib.load()
    level = {"enc0": 0, "enc1": 1, "enc2": 2, "mid_": 3, "dec2": 2, "dec1": 1, "dec0": 0}
    previous = lib.pmd_conv3d_impl(0)
    plans = {}
    try:
        for l in layout()[0]:
            f = 2 ** level[l.name[:4]]
            info = (ctypes.c_int * 8)()
            assert lib.pmd_conv3d_plan(16, 64 // f, 64 // f, 128 // f, l.cin, l.cout, info) == 0
            plans[l.name] = list(info)
        assert lib.pmd_conv3d_plan(1, 1, 1, 1, 12, 16, (ctypes.c_int * 8)()) == -1  # cin % 8
        assert lib.pmd_conv3d_plan(1, 1, 1, 1, 16, 16, None) == -1
    finally:
        lib.pmd_conv3d_impl(previous)
    assert plans.pop("enc0a")[0] == 2  # the 8-channel input layer: single-buffered kernel
    for name, (kernel, cg, groups, stages, streamed, tz, per_sm, smem) in plans.items():
        assert kernel == 4, name  # every other layer: warp-specialized
        assert 2 <= stages <= 4 and cg * groups * 8 == dict((l.name, l.cin) for l in layout()[0])[name]
        assert smem <= 232448 and per_sm in (1, 2) and tz in (1, 2, 4), name
        assert per_sm == 1 or 2 * (smem + 1024) <= 233472, name
    assert plans["dec0a"][1:7] == [2, 3, 3, 0, 2, 2]  # three resident groups, two blocks per SM
    assert plans["dec1a"][4] == 0  # 166 KB of weights stay resident
    assert all(plans[n][4] == 1 for n in ("enc2b", "mid_a", "mid_b", "dec2a", "dec2b"))


def _window_map(win, window, shape):
    """(grid index or -1) of every voxel of one oriented window: the map of
    pmd_gather_windows_oriented restated in numpy."""
    ox, oy, oz, orient, _, q1, q2 = (int(v) for v in win)
    d, f = orient >> 1, orient & 1
    l1, l2 = [a for a in range(3) if a != d]
    wa, wb, wd = window
    out = np.full((wa, wb, wd, 3), -1, dtype=np.int64)
    o = (ox, oy, oz)
    for k in range(wd):
        s1, s2 = (k * q1 + 32768) >> 16, (k * q2 + 32768) >> 16
        for a in range(wa):
            for b in range(wb):
                g = [0, 0, 0]
                g[l1], g[l2] = o[l1] + a + s1, o[l2] + b + s2
                g[d] = o[d] + (wd - 1 - k if f else k)
                if all(0 <= g[i] < shape[i] for i in range(3)):
                    out[a, b, k] = g
    return out


def test_oriented_windows_follow_each_beamlet():
    """Window planning (torch on the CPU): an oblique beamlet travelling
    towards -x and drifting in +y gets depth chunks along x from its entry side,
    sheared so that the beamlet stays within a voxel of the window's centre line
    at every depth; a +z beamlet gets the plain, unsheared window."""
    from pyradmc_b200 import denoise_dij as D

    shape = (40, 24, 16)
    dose = torch.zeros((2, *shape))
    beam = {}
    for x in range(40):
        t = 39 - x  # depth from the entry side (the beam enters at x = 39)
        y = int(round(4 + 0.4 * t))
        dose[0, x, y, 8] = 1.0 + 0.01 * t
        beam[(x, y, 8)] = t
    dose[1, 5, 7, :] = 1.0
    dirs = np.array([[-1.0, 0.4, 0.0], [0.0, 0.0, 1.0]])
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    assert D.orientation_codes(dirs).tolist() == [1, 4]
    window = (8, 8, 16)
    win = D.oriented_windows(dose.view(2, -1), shape, dirs, window).numpy()
    assert win.shape[1] == 7 and win[:, 4].tolist() == [0, 0, 0, 1]
    first = win[win[:, 4] == 0]
    assert (first[:, 3] == 1).all() and (first[:, 5] == round(0.4 * 65536)).all()
    assert (first[:, 6] == 0).all()
    assert first[:, 0].tolist() == [40 - 16, 40 - 32, 40 - 48]  # chunks from the entry side
    seen = 0
    for w in first:
        m = _window_map(w, window, shape)
        for a in range(8):
            for b in range(8):
                for k in range(16):
                    g = tuple(m[a, b, k])
                    if g in beam:  # the beamlet runs down the window's centre line
                        assert abs(a - 3.5) <= 1.5 and b == 8 - int(w[2]), (g, a, b, k)
                        seen += 1
    assert seen == 40  # every beamlet voxel lies in one window
    assert win[3].tolist() == [1, 3, 0, 4, 1, 0, 0]  # x 5 - 4, y 7 - 4, full depth, no shear
    one = D.oriented_windows(dose.view(2, -1), shape, dirs, window, starts=np.array([10, 0]))
    assert one.shape == (2, 7) and one[0, 0] == 40 - 26  # one window per column at that depth


def test_chunks_respect_the_32_bit_activation_limit():
    from pyradmc_b200.denoise_dij import chunk_windows

    # 64 x 64 x 128 windows: 48 channels x 524,288 voxels each -> at most 85 per pass
    assert chunk_windows(100, (64, 64, 128), 100) == 50  # two equal passes
    assert chunk_windows(100, (48, 48, 128), 100) == 100
    assert chunk_windows(7, (64, 64, 64), 100) == 7
    assert chunk_windows(250, (64, 64, 128), 100) == 84  # three passes of <= 85
    for n in (1, 33, 100, 257):
        c = chunk_windows(n, (64, 64, 128), 100)
        assert c * 64 * 64 * 128 * 48 < 2 ** 31 and c >= 1
