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
``ref_ct_beamlets_<count>.npz``
    ``ReferenceEngine.run_dij`` on the scaled-down CT-like Dij (``CT_CASE``),
    once per per-beamlet count of ``CT_CASE["counts"]``.
``philox_kat.npz``
    Nothing from pyRadMC: the Philox4x32-10 known-answer vectors are checked in
    ``tests/test_oracle.py`` directly.

Cases with ``shards`` (and the CT case) run as one process per statistical
batch: shard ``k`` is a one-batch ``ReferenceEngine`` run with seed
``seed * 100 + k``, and the shards' batch means are combined with the
reference scorer's own formulas (``scoring/dose.py:169-207``: mean of the batch
means, sigma from their sample variance).  That is exactly the estimate a
single multi-batch run would give if its batch ``k`` drew those streams; it
only spreads the single-threaded reference over the host's cores.

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

from cases import (  # noqa: E402
    CASES,
    COLLIMATION,
    CT_CASE,
    layered_density,
    layered_material,
    make_scoring,
    make_source,
)

REFERENCE: str | None = None  # path of the pyRadMC checkout, set by __main__ and the workers


def _reference_sources():
    from types import SimpleNamespace

    import pyradmc.geometry.source as S
    from pyradmc.geometry.collimation import TransmissionMaskBeamletSource, TransmissionMaskSource
    from pyradmc.geometry.spectrum import ali_rogers_mv

    return SimpleNamespace(
        PencilBeamSource=S.PencilBeamSource, ParallelBeamSource=S.ParallelBeamSource,
        SpectralBeamSource=S.SpectralBeamSource, BeamletGridSource=S.BeamletGridSource,
        SpectralBeamletSource=S.SpectralBeamletSource,
        CompositeBeamletSource=S.CompositeBeamletSource,
        TransmissionMaskSource=TransmissionMaskSource,
        TransmissionMaskBeamletSource=TransmissionMaskBeamletSource,
        PhaseSpaceSource=_reference_phsp,
        spectrum=lambda: ali_rogers_mv("varian-6mv", e_min=0.1),
        collimated=_reference_collimated)


def _reference_stack():
    from pyradmc.geometry.collimation import MLC, BeamFrame, BeamLimitingStack, JawPair

    c = COLLIMATION
    return BeamLimitingStack(frame=BeamFrame(origin=c["focal"]), devices=(JawPair(**c["jaw"]), MLC(**c["mlc"])))


def _reference_collimated(inner, beamlets: bool):
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.collimation import CollimatedBeamletSource, CollimatedSource

    cls = CollimatedBeamletSource if beamlets else CollimatedSource
    return cls(inner, _reference_stack(), AnalyticCrossSections())


def make_collimation() -> None:
    """tests/golden/collimation.npz: the COLLIMATION stack flattened
    (BeamLimitingStack.flatten) and the transmission table that pyRadMC's
    CollimatedSource builds for the 6 MV spectrum (_StackTransmission,
    geometry/collimation.py:945-969), so the tests need no reference code."""
    from pyradmc.geometry.source import SpectralBeamSource
    from pyradmc.geometry.spectrum import ali_rogers_mv

    inner = SpectralBeamSource(ali_rogers_mv("varian-6mv", e_min=0.1), COLLIMATION["focal"], (4.0, 4.0, 0.0),
                               6.0, 6.0)
    src = _reference_collimated(inner, False)
    model = src._model
    stack = _reference_stack()
    c = stack.flatten()
    out = {f"stack_{n}": np.asarray(getattr(c, n)) for n in c.__dataclass_fields__}
    out["stack_materials"] = np.asarray(stack.materials)
    out["stack_densities"] = np.asarray(stack.densities)
    out["log_energy"] = np.asarray(model._log_energies)
    out["log_total"] = np.asarray(model._log_mu) + np.log(np.asarray(model._densities))[:, None]
    np.savez_compressed(HERE / "collimation.npz", **out)
    print("collimation written", flush=True)


def _reference_phsp(path):
    import warnings

    from pyradmc.geometry.phasespace import PhaseSpaceSource

    warnings.filterwarnings("ignore", message=".*latent variance")  # oversampling is intended
    return PhaseSpaceSource(path)


def make_phsp_file() -> None:
    """tests/golden/phsp_beam.IAEAheader/.IAEAphsp: 20,000 seeded records, a
    divergent 6 x 6 cm field at z = -0.5 cm from a focal spot 100 cm above
    the phantom centre: 90 % photons of the 6 MV spectrum, 8 % electrons and
    2 % positrons of 0.5-3 MeV, weights U(0.5, 1.5)."""
    sys.path.insert(0, str(HERE.parents[1]))
    from pyradmc.geometry.spectrum import ali_rogers_mv

    from pyradmc_b200.phasespace import write_iaea

    rng = np.random.default_rng(20260901)
    n = 20_000
    kind = rng.choice([1, 2, 3], size=n, p=[0.90, 0.08, 0.02]).astype(np.int32)
    spectrum = ali_rogers_mv("varian-6mv", e_min=0.1)
    u = rng.random((n, 2))
    energy = spectrum.sample_energies(u[:, 0], u[:, 1])
    energy = np.where(kind == 1, energy, rng.uniform(0.5, 3.0, size=n))
    x = rng.uniform(1.0, 7.0, size=n)
    y = rng.uniform(1.0, 7.0, size=n)
    z = np.full(n, -0.5)
    d = np.stack([x - 4.0, y - 4.0, z + 100.0], axis=1)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    write_iaea(HERE / "phsp_beam", dict(particle_type=kind, energy=energy, x=x, y=y, z=z, ux=d[:, 0],
                                        uy=d[:, 1], uz=d[:, 2], weight=rng.uniform(0.5, 1.5, size=n)))
    print("phsp_beam written", flush=True)


def build_case(name: str):
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.grid import VoxelGrid

    case = CASES[name]
    g = case["grid"]
    grid = VoxelGrid.uniform_water(g["shape"], g["spacing"])
    if "layers" in g:
        density = layered_density(g["shape"], g["spacing"], (0.0, 0.0, 0.0), g["layers"])
        material = grid.material
        if "material_layers" in g:
            material = layered_material(g["shape"], g["spacing"], (0.0, 0.0, 0.0), g["material_layers"])
        grid = VoxelGrid(shape=g["shape"], spacing=g["spacing"], density=density, material=material)
    source = make_source(case["source"], _reference_sources())
    if case.get("cross_sections") == "water_bone":
        xs = water_and_bone(grid.max_density_by_material())
    else:
        xs = AnalyticCrossSections(geometry_densities=grid.max_density_by_material())
    run = dict(case["run"])
    if "scoring" in case:
        from types import SimpleNamespace

        from pyradmc.scoring.cylinder import CylindricalScoringGrid, geometric_edges

        run["scoring_grid"] = make_scoring(case, grid, SimpleNamespace(
            CylindricalScoringGrid=CylindricalScoringGrid, geometric_edges=geometric_edges))
    return grid, xs, source, run


def water_and_bone(geometry_densities):
    """pyRadMC's analytic source with the first five materials of its registry
    addressable (water ... cortical bone): Compton, stopping powers, Moller and
    scattering power follow each material's composition; the photoelectric,
    pair and radiative fits stay water's.  A synthetic multi-material source for
    the dose-to-water parity case."""
    from pyradmc.data.analytic import AnalyticCrossSections

    class WaterAndBone(AnalyticCrossSections):
        @property
        def n_materials(self) -> int:
            return 5

        @property
        def provenance(self) -> str:
            return "analytic closed-form, registry materials 0-4 (synthetic multi-material test source)"

    return WaterAndBone(geometry_densities=geometry_densities)


def make_bone_pack() -> None:
    """tests/golden/pack_water_bone.npz: the water_and_bone tables at 6 MeV and
    the GS grid of water + cortical bone."""
    sys.path.insert(0, str(HERE.parents[1]))
    from pyradmc_b200.model import save_pack

    from cases import BONE_MATERIAL

    xs = water_and_bone(((0, 1.0), (BONE_MATERIAL, 1.85)))
    save_pack(xs, HERE / "pack_water_bone.npz", ecut=0.2, pcut=0.05, e_max=6.0 * (1 + 1e-6),
              materials=[0, BONE_MATERIAL])
    print("pack_water_bone written", flush=True)


def _combine_batches(batch_means: np.ndarray):
    """Mean and sigma of equal-weight batch means (scoring/dose.py:188-207)."""
    n = batch_means.shape[0]
    s1 = batch_means.sum(axis=0)
    s2 = (batch_means**2).sum(axis=0)
    mean = s1 / n
    variance = np.maximum(0.0, s2 / n - mean**2) * n / (n - 1)
    return mean, np.sqrt(variance / n)


def _init_worker(reference: str) -> None:
    global REFERENCE
    REFERENCE = reference
    sys.path.insert(0, reference)


def _forward_shard(task):
    name, k = task
    from pyradmc.backends.ref.engine import ReferenceEngine
    from pyradmc.rng.host import HostRNG

    grid, xs, source, run = build_case(name)
    shards = CASES[name]["shards"]
    run = dict(run)
    run["n_histories"] //= shards
    run["n_batches"] = 1
    run["seed"] = run["seed"] * 100 + k
    res = ReferenceEngine(grid=grid, cross_sections=xs, rng=HostRNG()).run(source, **run)
    books = (res.energy_emitted, res.energy_deposited, res.energy_escaped, res.energy_unscored)
    return res.dose.reshape(-1), books


def _ct_build():
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.grid import VoxelGrid
    from pyradmc.geometry.source import SpectralBeamletSource
    from pyradmc.geometry.spectrum import ali_rogers_mv

    sys.path.insert(0, str(HERE.parents[1]))
    from pyradmc_b200 import phantoms

    g = CT_CASE["grid"]
    mirror = phantoms.ellipsoid_phantom(shape=g["shape"], spacing=g["spacing"], seed=g["ellipsoid_seed"])
    grid = VoxelGrid(shape=g["shape"], spacing=g["spacing"], density=mirror.density,
                     material=np.zeros(g["shape"], dtype=np.int32))
    f = CT_CASE["fan"]
    fan = phantoms.beamlet_fan(mirror, n_x=f["n_x"], n_y=f["n_y"], pitch=f["pitch"], width=f["width"],
                               sad=f["sad"])
    source = SpectralBeamletSource(ali_rogers_mv("varian-6mv", e_min=0.1), fan.focal_point,
                                   fan.centers, fan.width_u, fan.width_v)
    xs = AnalyticCrossSections(geometry_densities=grid.max_density_by_material())
    return grid, xs, source


def _ct_shard(task):
    count, k = task
    from pyradmc.backends.ref.engine import ReferenceEngine
    from pyradmc.rng.host import HostRNG

    grid, xs, source = _ct_build()
    run = dict(CT_CASE["run"])
    n_batches = run.pop("n_batches")
    seed = run.pop("seed") * 100 + k
    res = ReferenceEngine(grid=grid, cross_sections=xs, rng=HostRNG()).run_dij(
        source, n_histories_per_beamlet=count // n_batches, n_batches=1, seed=seed, **run)
    dense = np.stack([res.column_dense(j).reshape(-1) for j in range(res.n_beamlets)])
    books = (res.energy_emitted, res.energy_deposited, res.energy_escaped, res.energy_unscored)
    return dense, books


def _pool(n_tasks: int):
    import multiprocessing
    import os
    from concurrent.futures import ProcessPoolExecutor

    for var in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[var] = "1"  # one core per shard
    return ProcessPoolExecutor(max_workers=min(n_tasks, os.cpu_count() or 1),
                               mp_context=multiprocessing.get_context("spawn"),
                               initializer=_init_worker, initargs=(REFERENCE,))


def _warm_gs_cache(name: str) -> None:
    """Build the eager GS node window once before the workers start: the
    reference otherwise extends its on-disk grid lazily, node by node, in every
    worker at once."""
    from pyradmc.data.goudsmit_saunderson import build_gs_grid, gs_window_from_tables

    grid, xs, source, _ = build_case(name)
    materials = sorted({int(m) for m in np.unique(grid.material)})
    for e_max in (source.max_energy, 6.0):
        tables = xs.build_tables(ecut=0.2, pcut=0.05, e_max=e_max * (1 + 1e-6))
        build_gs_grid(*gs_window_from_tables(tables, materials))


def run_sharded(name: str) -> None:
    shards = CASES[name]["shards"]
    _warm_gs_cache(name)
    t0 = time.perf_counter()
    with _pool(shards) as pool:
        parts = list(pool.map(_forward_shard, [(name, k) for k in range(shards)]))
    elapsed = time.perf_counter() - t0
    grid, _, _, run_kw = build_case(name)
    scoring = run_kw.get("scoring_grid")
    grid_shape = tuple(scoring.shape) if scoring is not None else tuple(grid.shape)
    mean, sigma = _combine_batches(np.stack([p[0] for p in parts]))
    books = np.sum([p[1] for p in parts], axis=0)
    run = CASES[name]["run"]
    np.savez_compressed(
        HERE / f"ref_{name}.npz",
        energy_emitted=books[0], energy_deposited=books[1], energy_escaped=books[2],
        energy_unscored=books[3], seconds=elapsed,
        dose=mean.reshape(grid_shape), dose_sigma=sigma.reshape(grid_shape),
        n_batches=shards, n_histories=run["n_histories"], shard_seeds=run["seed"] * 100 + np.arange(shards),
    )
    print(f"{name}: {elapsed:.1f} s over {shards} shards", flush=True)


def run_ct() -> None:
    n_batches = CT_CASE["run"]["n_batches"]
    _warm_gs_cache("dij_spectral")
    for count in CT_CASE["counts"]:
        t0 = time.perf_counter()
        with _pool(n_batches) as pool:
            parts = list(pool.map(_ct_shard, [(count, k) for k in range(n_batches)]))
        elapsed = time.perf_counter() - t0
        batch = np.stack([p[0] for p in parts])  # [batch][column][voxel]
        mean, sigma = _combine_batches(batch)
        books = np.sum([p[1] for p in parts], axis=0)
        np.savez_compressed(
            HERE / f"ref_ct_beamlets_{count}.npz",
            energy_emitted=books[0], energy_deposited=books[1], energy_escaped=books[2],
            energy_unscored=books[3], seconds=elapsed, dose=mean, dose_sigma=sigma,
            n_batches=n_batches, n_histories_per_beamlet=count,
            shard_seeds=CT_CASE["run"]["seed"] * 100 + np.arange(n_batches),
        )
        print(f"ct_beamlets {count}: {elapsed:.1f} s over {n_batches} shards", flush=True)


def run_case(name: str) -> None:
    if "shards" in CASES[name]:
        run_sharded(name)
        return
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
    REFERENCE = sys.argv[1]
    sys.path.insert(0, REFERENCE)
    names = sys.argv[2:] or ["reduction", "bone_pack", "phsp_file", "collimation", *CASES, "ct_beamlets"]
    for name in names:
        if name == "reduction":
            make_reduction()
        elif name == "bone_pack":
            make_bone_pack()
        elif name == "phsp_file":
            make_phsp_file()
        elif name == "collimation":
            make_collimation()
        elif name == "ct_beamlets":
            run_ct()
        else:
            run_case(name)
