"""Generate the golden fixtures from pyRadMC itself (its ReferenceEngine oracle).

Run in a checkout that has pyRadMC (the reference) available::

    HOME=<writable dir> python tests/golden/make_golden.py /path/to/pyRadMC

It writes, next to this file:

``ref_<case>.npz``
    ``ReferenceEngine.run`` / ``run_dij`` outputs for every case of ``cases.py``
    (dose, sigma, energy books), the statistical oracle of the B200 parity tests.
``reduction.npz``
    Seeded int64 quanta maps and the exact outputs of pyRadMC's own host scorers
    on them — ``BatchedBeamletScorer.end_batch``/``finalize`` (scoring/dij.py:
    155-191) and ``DijAssembler.add_block``/``finalize`` (:351-434) — the
    bit-exact pin of the device fold, finalize, truncation and compaction.
``philox_kat.npz``
    Nothing from pyRadMC: the Philox4x32-10 known-answer vectors are checked in
    ``tests/test_oracle.py`` directly.

pyRadMC's GS table cache lives under ``$HOME/.cache/pyradmc``; point ``HOME`` at
a scratch directory.
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

from cases import CASES, layered_density  # noqa: E402


def build_case(name: str):
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.grid import VoxelGrid
    from pyradmc.geometry.source import (
        BeamletGridSource,
        ParallelBeamSource,
        PencilBeamSource,
        SpectralBeamletSource,
        SpectralBeamSource,
    )
    from pyradmc.geometry.spectrum import ali_rogers_mv

    case = CASES[name]
    g = case["grid"]
    grid = VoxelGrid.uniform_water(g["shape"], g["spacing"])
    if "layers" in g:
        density = layered_density(g["shape"], g["spacing"], (0.0, 0.0, 0.0), g["layers"])
        grid = VoxelGrid(shape=g["shape"], spacing=g["spacing"], density=density,
                         material=grid.material)
    s = case["source"]
    kind = s["kind"]
    if kind == "parallel":
        source = ParallelBeamSource(s["energy"], s["z"], s["x_range"], s["y_range"])
    elif kind == "pencil":
        source = PencilBeamSource(s["energy"], s["position"], s["direction"])
    elif kind == "spectral":
        source = SpectralBeamSource(ali_rogers_mv("varian-6mv", e_min=0.1), s["focal_point"],
                                    s["center"], s["width_u"], s["width_v"])
    elif kind == "lattice":
        source = BeamletGridSource(s["energy"], s["z"], s["x_range"], s["y_range"], s["n_x"],
                                   s["n_y"])
    elif kind == "spectral_beamlets":
        source = SpectralBeamletSource(ali_rogers_mv("varian-6mv", e_min=0.1), s["focal_point"],
                                       s["centers"], s["width_u"], s["width_v"])
    else:
        raise ValueError(kind)
    xs = AnalyticCrossSections(geometry_densities=grid.max_density_by_material())
    return grid, xs, source, case["run"]


def run_case(name: str) -> None:
    from pyradmc.backends.ref.engine import ReferenceEngine
    from pyradmc.rng.host import HostRNG

    grid, xs, source, run = build_case(name)
    engine = ReferenceEngine(grid=grid, cross_sections=xs, rng=HostRNG())
    t0 = time.perf_counter()
    if "n_histories_per_beamlet" in run:
        res = engine.run_dij(source, **run)
        dense = np.stack([res.column_dense(j).reshape(-1) for j in range(res.n_beamlets)])
        sig = np.stack([res.sigma_dense(j).reshape(-1) for j in range(res.n_beamlets)])
        out = dict(dose=dense, dose_sigma=sig, n_batches=res.n_batches,
                   indptr=res.indptr, indices=res.indices, csc_dose=res.dose)
    else:
        res = engine.run(source, **run)
        out = dict(dose=res.dose, dose_sigma=res.dose_sigma, n_batches=res.n_batches,
                   n_histories=res.n_histories)
    elapsed = time.perf_counter() - t0
    np.savez_compressed(
        HERE / f"ref_{name}.npz",
        energy_emitted=res.energy_emitted,
        energy_deposited=res.energy_deposited,
        energy_escaped=res.energy_escaped,
        energy_unscored=res.energy_unscored,
        seconds=elapsed,
        **out,
    )
    print(f"{name}: {elapsed:.1f} s", flush=True)


def make_reduction() -> None:
    """Pin the device reduction against pyRadMC's own scorer and assembler."""
    from pyradmc.geometry.grid import VoxelGrid
    from pyradmc.scoring.dij import BatchedBeamletScorer, DijAssembler

    rng = np.random.default_rng(20260801)
    shape = (6, 7, 9)
    n_vox = int(np.prod(shape))
    n_cols, n_batches, per_batch = 3, 5, 40
    density = rng.uniform(0.2, 1.9, size=shape)
    grid = VoxelGrid(shape=shape, spacing=(0.3, 0.25, 0.5), density=density,
                     material=np.zeros(shape, dtype=np.int32))
    # Sparse integer quanta maps (~10 % occupied), one per batch.
    quanta = np.zeros((n_batches, n_cols, n_vox), dtype=np.int64)
    occupied = rng.random(quanta.shape) < 0.1
    quanta[occupied] = rng.integers(1, 10**12, size=int(occupied.sum()))
    quanta[:, 2, :] = 0  # an all-empty column
    quanta[:, 1, 5] = 10**15  # one dominant entry: most of column 1 falls below truncation
    scorer = BatchedBeamletScorer(grid, n_batches, n_cols)
    for b in range(n_batches):
        scorer.deposit_block(quanta[b].astype(np.float64) * 1.0e-9)
        scorer.end_batch(per_batch)
    block = scorer.finalize()
    outputs = {}
    for trunc in (0.0, 1.0e-3, 0.2):
        asm = DijAssembler(grid_shape=shape, n_beamlets=n_cols, n_histories_per_beamlet=per_batch * n_batches,
                           n_batches=n_batches, truncation=trunc)
        asm.add_block(0, block.dose, block.sigma)
        dij = asm.finalize(0.0, 0.0, 0.0)
        tag = f"{trunc:g}"
        outputs[f"indptr_{tag}"] = dij.indptr
        outputs[f"indices_{tag}"] = dij.indices
        outputs[f"dose_{tag}"] = dij.dose
        outputs[f"sigma_{tag}"] = dij.sigma
    np.savez_compressed(
        HERE / "reduction.npz",
        quanta=quanta,
        voxel_mass=(grid.density * grid.voxel_volume).reshape(-1),
        per_batch=per_batch,
        mean=block.dose,
        sigma=block.sigma,
        **outputs,
    )
    print("reduction written", flush=True)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit("usage: python tests/golden/make_golden.py /path/to/pyRadMC [case ...]")
    sys.path.insert(0, sys.argv[1])
    names = sys.argv[2:] or ["reduction", *CASES]
    for name in names:
        if name == "reduction":
            make_reduction()
        else:
            run_case(name)
