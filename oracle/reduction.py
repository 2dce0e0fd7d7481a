"""TEST INFRASTRUCTURE — numpy restatement of pyRadMC's batch scorer and Dij assembler.

``fold_finalize`` follows ``BatchedBeamletScorer.end_batch`` and ``finalize``
(pyradmc/scoring/dij.py:155-191) operation for operation; ``truncate`` follows
``DijAssembler.add_block`` + ``finalize`` (scoring/dij.py:351-434).  The inputs
are the int64 quanta maps a kernel backend scores (1e-9 MeV per quantum,
kernels.py:96), so a device reduction of the same maps must match bit for bit.
"""

from __future__ import annotations

import numpy as np

QUANTUM = 1.0e-9


def fold_finalize(quanta: np.ndarray, voxel_mass: np.ndarray, per_batch) -> tuple:
    """``quanta``: [n_batches][n_cols][n_vox] int64.  Returns (mean, sigma, total quanta).

    ``per_batch`` is one count for every column or one per column.
    """
    n_batches, n_cols, n_vox = quanta.shape
    nh = np.broadcast_to(np.asarray(per_batch, dtype=np.float64), (n_cols,))
    covered = voxel_mass > 0.0
    s1 = np.zeros((n_cols, n_vox))
    s2 = np.zeros((n_cols, n_vox))
    for b in range(n_batches):
        energy = quanta[b].astype(np.float64) * QUANTUM
        dose = np.divide(energy, voxel_mass[np.newaxis, :] * nh[:, np.newaxis],
                         out=np.zeros_like(energy), where=covered[np.newaxis, :])
        s1 += dose
        s2 += dose**2
    n = n_batches
    mean = s1 / n
    if n == 1:
        sigma = np.zeros_like(mean)
    else:
        variance = np.maximum(0.0, s2 / n - mean**2) * n / (n - 1)
        sigma = np.sqrt(variance / n)
    return mean, sigma, int(quanta.sum())


def truncate(mean: np.ndarray, sigma: np.ndarray, truncation: float) -> tuple:
    """Per-column relative truncation into CSC: (indptr, indices, dose, sigma)."""
    indices, dose, sig, counts = [], [], [], []
    for row_dose, row_sigma in zip(mean, sigma, strict=True):
        col_max = float(row_dose.max(initial=0.0))
        keep = row_dose >= truncation * col_max
        keep &= row_dose > 0.0
        idx = np.flatnonzero(keep)
        indices.append(idx.astype(np.int64))
        dose.append(row_dose[idx])
        sig.append(row_sigma[idx])
        counts.append(int(idx.size))
    indptr = np.zeros(len(counts) + 1, dtype=np.int64)
    np.cumsum(counts, out=indptr[1:])
    return indptr, np.concatenate(indices), np.concatenate(dose), np.concatenate(sig)
