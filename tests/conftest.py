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

from cases import CASES, SEED, layered_density  # noqa: E402


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


def build_case(name: str):
    """(grid, cross_sections, source, run kwargs) of a golden case, on this package's types."""
    import pyradmc_b200 as P

    case = CASES[name]
    g = case["grid"]
    grid = P.VoxelGrid.uniform_water(g["shape"], g["spacing"])
    if "layers" in g:
        grid = P.VoxelGrid(shape=g["shape"], spacing=g["spacing"],
                           density=layered_density(g["shape"], g["spacing"], (0, 0, 0), g["layers"]),
                           material=grid.material)
    s = case["source"]
    kind = s["kind"]
    if kind == "parallel":
        src = P.ParallelBeamSource(s["energy"], s["z"], s["x_range"], s["y_range"])
    elif kind == "pencil":
        src = P.PencilBeamSource(s["energy"], s["position"], s["direction"])
    elif kind == "spectral":
        src = P.SpectralBeamSource(P.ali_rogers_varian_6mv(), s["focal_point"], s["center"],
                                   s["width_u"], s["width_v"])
    elif kind == "lattice":
        src = P.BeamletGridSource(s["energy"], s["z"], s["x_range"], s["y_range"], s["n_x"], s["n_y"])
    else:
        src = P.SpectralBeamletSource(P.ali_rogers_varian_6mv(), s["focal_point"], s["centers"],
                                      s["width_u"], s["width_v"])
    xs = P.AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, src, dict(case["run"])


def load_ref(name: str) -> dict:
    with np.load(GOLDEN / f"ref_{name}.npz") as z:
        return {k: z[k] for k in z.files}


__all__ = ["CASES", "GOLDEN", "ROOT", "SEED", "build_case", "cuda_available", "load_ref"]
