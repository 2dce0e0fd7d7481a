"""Shared fixtures: markers, the case builder, and the GPU-availability gate.

``@pytest.mark.gpu`` tests need a CUDA device and the built sm_100a library;
everything else runs on a CPU-only host (oracle, host logic, ABI exports,
multi-process gloo tests).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT), str(GOLDEN)):
    if p not in sys.path:
        sys.path.insert(0, p)

from cases import (  # noqa: E402
    CASES,
    CT_CASE,
    SEED,
    layered_density,
    layered_material,
    make_scoring,
    make_source,
)


def pytest_sessionfinish(session, exitstatus):
    """Write every named chi-squared comparison of the session ({case,
    chi2_per_dof, p, n_voxels}) to $PMC_PARITY_REPORT, default
    .parity/chi2.json at the repository root."""
    import json
    import os

    from oracle import stats

    if not stats.RECORDS:
        return
    path = Path(os.environ.get("PMC_PARITY_REPORT", ROOT / ".parity" / "chi2.json"))
    path.parent.mkdir(parents=True, exist_ok=True)
    path.write_text(json.dumps(stats.RECORDS, indent=1))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: longer statistical runs")


def cuda_available() -> bool:
    try:
        from pyradmc_b200 import _lib

        return _lib.load().pmc_device_count() > 0
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not cuda_available():
        pytest.fail("no CUDA device visible to the B200 library: the gpu tests need a B200")
    return "cuda:0"


def collimated(inner, beamlets: bool):
    """`inner` seen through the collimated cases' stack, with the stack and
    transmission table pyRadMC built (tests/golden/collimation.npz)."""
    import pyradmc_b200 as P
    from pyradmc_b200.presolve import CompiledHeadStack

    with np.load(GOLDEN / "collimation.npz") as z:
        f = {k: z[k] for k in z.files}
    names = [n for n in CompiledHeadStack.__dataclass_fields__ if n not in ("materials", "densities", "_keep")]
    stack = CompiledHeadStack(**{n: f[f"stack_{n}"] for n in names},
                              materials=tuple(int(m) for m in f["stack_materials"]),
                              densities=tuple(float(d) for d in f["stack_densities"]))
    cls = P.CollimatedBeamletSource if beamlets else P.CollimatedSource
    return cls.from_tables(inner, stack, f["log_energy"], f["log_total"])


def build_case(name: str):
    """(grid, cross_sections, source, run kwargs) of a golden case, on this package's types."""
    import pyradmc_b200 as P

    case = CASES[name]
    g = case["grid"]
    grid = P.VoxelGrid.uniform_water(g["shape"], g["spacing"])
    if "layers" in g:
        material = grid.material
        if "material_layers" in g:
            material = layered_material(g["shape"], g["spacing"], (0, 0, 0), g["material_layers"])
        grid = P.VoxelGrid(shape=g["shape"], spacing=g["spacing"],
                           density=layered_density(g["shape"], g["spacing"], (0, 0, 0), g["layers"]),
                           material=material)
    from types import SimpleNamespace

    from pyradmc_b200.phasespace import PhaseSpaceSource

    ns = SimpleNamespace(**{name: getattr(P, name) for name in (
        "PencilBeamSource", "ParallelBeamSource", "SpectralBeamSource", "BeamletGridSource",
        "SpectralBeamletSource", "CompositeBeamletSource", "TransmissionMaskSource",
        "TransmissionMaskBeamletSource")},
        spectrum=P.ali_rogers_varian_6mv,
        PhaseSpaceSource=PhaseSpaceSource, collimated=collimated)
    src = make_source(case["source"], ns)
    if case.get("cross_sections") == "water_bone":
        xs = P.PackedCrossSections(GOLDEN / "pack_water_bone.npz")
    else:
        xs = P.AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    run = dict(case["run"])
    if "scoring" in case:
        run["scoring_grid"] = make_scoring(case, grid, P)
    return grid, xs, src, run


def build_ct_case():
    """(grid, cross_sections, source) of the scaled-down CT-like Dij case."""
    import pyradmc_b200 as P
    from pyradmc_b200 import phantoms

    g = CT_CASE["grid"]
    grid = phantoms.ellipsoid_phantom(shape=g["shape"], spacing=g["spacing"], seed=g["ellipsoid_seed"])
    f = CT_CASE["fan"]
    src = phantoms.beamlet_fan(grid, n_x=f["n_x"], n_y=f["n_y"], pitch=f["pitch"], width=f["width"],
                               sad=f["sad"])
    xs = P.AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, src


def load_ref(name: str) -> dict:
    with np.load(GOLDEN / f"ref_{name}.npz") as z:
        return {k: z[k] for k in z.files}


__all__ = ["CASES", "CT_CASE", "GOLDEN", "ROOT", "SEED", "build_case", "build_ct_case",
           "cuda_available", "load_ref"]
