"""The denoiser's final truncation + CSC (denoise_dij.compact, through the
allocation-free pmc_dij_compact_static) against a NumPy restatement of the
reference assembler's rule (scoring/dij.py:351-366: keep m > 0 and m >=
truncation x column maximum, rows ascending), including a call that needs more
room than the previous call of its shape reserved (the capacity retry)."""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _expected(mean, sigma, truncation):
    indptr, idx, dose, sig = [0], [], [], []
    for c in range(mean.shape[0]):
        m = mean[c]
        keep = np.flatnonzero((m > 0) & (m >= truncation * m.max()))
        idx.append(keep)
        dose.append(m[keep])
        sig.append(sigma[c][keep])
        indptr.append(indptr[-1] + keep.size)
    return np.array(indptr), np.concatenate(idx), np.concatenate(dose), np.concatenate(sig)


def test_compaction_matches_the_rule_and_grows_its_reservation(gpu):
    import torch

    from pyradmc_b200 import denoise_dij as D

    rng = np.random.default_rng(3)
    n_cols, vox = 6, 70_000
    for density in (0.001, 0.5):  # the second call needs ~500x the first's entries
        mean = rng.random((n_cols, vox)) * (rng.random((n_cols, vox)) < density)
        mean[:, :3] = 0.0
        sigma = 0.1 * mean
        got = D.compact(torch.from_numpy(mean).to(gpu), torch.from_numpy(sigma).to(gpu), 1e-3, to_host=True)
        ref = _expected(mean, sigma, 1e-3)
        for a, b in zip(got, ref, strict=True):
            np.testing.assert_array_equal(a, b)
