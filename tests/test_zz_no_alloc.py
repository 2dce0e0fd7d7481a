"""The allocation-free compaction entry point, ``pmc_dij_compact_static``.

It serves callers that cannot call cudaMalloc themselves or have the library do
it for them — all of their device memory comes from their own pool, or their
footprint is fixed at start-up — so it works on device buffers the caller
already owns and keeps its scratch in a static device array.  This test hands it
device buffers (allocated here by the test harness, as such a caller's pool
would), calls it through the C-ABI twice in a row on different inputs, and
checks every output against the allocating entry point ``pmc_truncate_dense`` on
the same data: the CSC must be identical, bit for bit, as the reduction tests
require.  Around the second call the device's free memory must not drop: the
entry point's defining property is that it allocates nothing.  The file sorts
last so that a stop at the first failure has already run every other test.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from pyradmc_b200 import _lib
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _allocating_reference(native, mean, sigma, truncation):
    n_cols, n_vox = mean.shape
    counts = np.zeros(n_cols, dtype=np.int64)
    nnz = C.c_int64()
    m = np.ascontiguousarray(mean)
    s = np.ascontiguousarray(sigma)
    native.check(native.lib.pmc_truncate_dense(native.handle, _lib.ptr(m, C.c_double),
                                               _lib.ptr(s, C.c_double), n_cols, n_vox, truncation,
                                               _lib.ptr(counts, C.c_int64), C.byref(nnz)))
    indptr = np.zeros(n_cols + 1, dtype=np.int64)
    idx = np.zeros(nnz.value, dtype=np.int64)
    dose = np.zeros(nnz.value)
    sig = np.zeros(nnz.value)
    native.check(native.lib.pmc_dij_fetch(native.handle, _lib.ptr(indptr, C.c_int64),
                                          _lib.ptr(idx, C.c_int64), _lib.ptr(dose, C.c_double),
                                          _lib.ptr(sig, C.c_double)))
    return counts, idx, dose, sig


def _static(lib, mean, sigma, truncation, capacity):
    import torch

    dev = torch.device("cuda:0")
    n_cols, n_vox = mean.shape
    d_mean = torch.from_numpy(np.ascontiguousarray(mean)).to(dev)
    d_sigma = torch.from_numpy(np.ascontiguousarray(sigma)).to(dev)
    d_counts = torch.full((n_cols,), -1, dtype=torch.int64, device=dev)
    d_idx = torch.full((capacity,), -1, dtype=torch.int64, device=dev)
    d_dose = torch.full((capacity,), -1.0, dtype=torch.float64, device=dev)
    d_sig = torch.full((capacity,), -1.0, dtype=torch.float64, device=dev)
    nnz = C.c_int64(-1)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    free_before = torch.cuda.mem_get_info(dev)[0]
    code = lib.pmc_dij_compact_static(
        C.c_void_p(d_mean.data_ptr()), C.c_void_p(d_sigma.data_ptr()), n_cols, n_vox,
        float(truncation), capacity, C.c_void_p(d_counts.data_ptr()),
        C.c_void_p(d_idx.data_ptr()), C.c_void_p(d_dose.data_ptr()), C.c_void_p(d_sig.data_ptr()),
        C.byref(nnz), C.c_void_p(stream.cuda_stream))
    assert code == _lib.PMC_OK, code
    free_after = torch.cuda.mem_get_info(dev)[0]  # the call has synchronized its stream
    k = nnz.value
    return (d_counts.cpu().numpy(), d_idx[:k].cpu().numpy(), d_dose[:k].cpu().numpy(),
            d_sig[:k].cpu().numpy(), k, free_before - free_after)


def _inputs():
    with np.load(GOLDEN / "reduction.npz") as z:
        golden = (np.ascontiguousarray(z["mean"]), np.ascontiguousarray(z["sigma"]))
    rng = np.random.default_rng(7)
    n_cols, n_vox = 9, 3 * 4096 + 17  # several tiles per column, a ragged last tile
    mean = np.where(rng.random((n_cols, n_vox)) < 0.3, rng.exponential(1.0, (n_cols, n_vox)), 0.0)
    mean[4] = 0.0  # an empty column
    sigma = rng.random((n_cols, n_vox)) * mean
    return [(golden[0], golden[1], 1.0e-3), (mean, sigma, 0.05)]


def test_static_compaction_matches_the_allocating_entry_point_twice_in_a_row(gpu):
    import pyradmc_b200 as P

    grid = P.VoxelGrid.uniform_water((2, 2, 2), (1.0, 1.0, 1.0))
    native = P.B200Engine(grid, P.AnalyticWaterTables())._native()
    lib = _lib.load()
    for call, (mean, sigma, trunc) in enumerate(_inputs()):
        counts, idx, dose, sig = _allocating_reference(native, mean, sigma, trunc)
        got_counts, got_idx, got_dose, got_sig, nnz, used = _static(lib, mean, sigma, trunc,
                                                                     capacity=mean.size)
        if call > 0:  # the first call may load the module (and its static array) lazily
            assert used <= 0, f"the allocation-free entry point took {used} bytes of device memory"
        assert nnz == idx.size
        np.testing.assert_array_equal(got_counts, counts)
        np.testing.assert_array_equal(got_idx, idx)
        np.testing.assert_array_equal(got_dose, dose)
        np.testing.assert_array_equal(got_sig, sig)


def test_static_compaction_rejects_what_it_cannot_hold(gpu):
    import torch

    lib = _lib.load()
    mean, sigma, trunc = _inputs()[1]
    _, idx, _, _, _, _ = _static(lib, mean, sigma, trunc, capacity=mean.size)
    d = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    d_mean = torch.from_numpy(mean).cuda()  # held: a freed temporary could be reused
    d_sigma = torch.from_numpy(sigma).cuda()
    torch.cuda.synchronize()
    nnz = C.c_int64(-1)
    small = lib.pmc_dij_compact_static(
        C.c_void_p(d_mean.data_ptr()), C.c_void_p(d_sigma.data_ptr()), mean.shape[0],
        mean.shape[1], trunc, 4, C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
        C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()), C.byref(nnz), None)
    assert small == _lib.PMC_ERR_CAPACITY and nnz.value == idx.size
    too_many = lib.pmc_dij_compact_static(C.c_void_p(d.data_ptr()), C.c_void_p(d.data_ptr()),
                                          5000, 1, 0.0, 0, C.c_void_p(d.data_ptr()), None, None,
                                          None, C.byref(nnz), None)
    assert too_many == _lib.PMC_ERR_INVALID
