"""TEST INFRASTRUCTURE — the reference's statistical detection oracles.

Restated from pyRadMC's test suite (tests/conftest.py:109-196): the chi-squared
test over a region of interest, and its batched variant that calibrates the null
for batch-estimated sigmas with the Welch-Satterthwaite effective degrees of
freedom (each voxel's z^2 is F(1, nu); E[z^2] = nu / (nu - 2)).
"""

from __future__ import annotations

import numpy as np
from scipy import stats


def chi2_batched(a, sigma_a, n_a, b, sigma_b, n_b, mask=None) -> dict:
    """Statistics of the batched chi-squared comparison (no assertion)."""
    if min(n_a, n_b) < 6:
        raise ValueError("need at least 6 batches per side for a calibrated batched chi2")
    if mask is None:
        mask = np.ones(np.shape(a), dtype=bool)
    va = np.asarray(sigma_a)[mask] ** 2
    vb = np.asarray(sigma_b)[mask] ** 2
    if np.any(va + vb <= 0.0):
        raise ValueError("zero uncertainty in the compared region; score dose-squared")
    nu = (va + vb) ** 2 / (va**2 / (n_a - 1) + vb**2 / (n_b - 1))
    z_sq = (np.asarray(a)[mask] - np.asarray(b)[mask]) ** 2 / (va + vb)
    chi2 = float(np.sum(z_sq))
    mean = float(np.sum(nu / (nu - 2.0)))
    variance = float(np.sum(2.0 * nu**2 * (nu - 1.0) / ((nu - 2.0) ** 2 * (nu - 4.0))))
    z = (chi2 - mean) / np.sqrt(variance)
    return dict(chi2=chi2, null_mean=mean, null_sd=float(np.sqrt(variance)),
                p_value=float(stats.norm.sf(z)), n=int(np.count_nonzero(mask)),
                chi2_per_dof=chi2 / max(1, int(np.count_nonzero(mask))))


RECORDS: list[dict] = []  # every comparison made with a `case` name, for the parity report


def assert_chi2_consistent_batched(a, sigma_a, n_a, b, sigma_b, n_b, alpha=0.01, mask=None,
                                   case: str | None = None):
    r = chi2_batched(a, sigma_a, n_a, b, sigma_b, n_b, mask)
    if case is not None:
        RECORDS.append({"case": case, "chi2_per_dof": r["chi2_per_dof"], "p": r["p_value"],
                        "n_voxels": r["n"], "null_mean_per_dof": r["null_mean"] / max(1, r["n"]),
                        "passed": r["p_value"] > alpha})
    assert r["p_value"] > alpha, (
        f"chi2={r['chi2']:.1f} vs batched-null mean {r['null_mean']:.1f} (sd {r['null_sd']:.1f}) "
        f"on {r['n']} voxels, p={r['p_value']:.2e} < alpha={alpha}. "
        "The two estimates are not statistically consistent: suspect a bias, not noise."
    )
    return r


def high_dose_mask(ref_dose, ref_sigma, other_sigma, fraction=0.1, minimum=1):
    """High-dose region where both estimates carry a defined uncertainty."""
    mask = ref_dose > fraction * ref_dose.max()
    mask &= (ref_sigma > 0.0) & (other_sigma > 0.0)
    assert np.count_nonzero(mask) >= minimum, "mask too small to detect anything"
    return mask
