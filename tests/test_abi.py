"""The drop-in boundary on a CPU-only host: the C-ABI library builds, loads and
exports every entry point ``include/pyradmc_b200.h`` declares, its ctypes
mirrors have the C layout, and the engine fails loudly (never falls back to a
CPU path) when no CUDA device is present."""

from __future__ import annotations

import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from pyradmc_b200 import _lib
from tests.conftest import ROOT, cuda_available

HEADER = ROOT / "include" / "pyradmc_b200.h"
DENOISE_HEADER = ROOT / "include" / "pyradmc_b200_denoise.h"
PRESOLVE_HEADER = ROOT / "include" / "pyradmc_b200_presolve.h"


def declared_symbols() -> set[str]:
    text = HEADER.read_text() + DENOISE_HEADER.read_text() + PRESOLVE_HEADER.read_text()
    return set(re.findall(r"\b(pm[cd]_[a-z0-9_]+)\s*\(", text)) - {"pmc_progress_fn"}


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = declared_symbols()
    assert declared, "no declarations parsed from the header"
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing, f"symbols declared but not exported: {missing}"
    assert declared <= set(_lib.SIGNATURES), "ctypes signatures missing for some symbols"
    out = subprocess.run(["nm", "-D", "--defined-only", str(_lib.library_path())],
                         capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (pm[cd]_\w+)", out))
    assert declared <= exported
    assert any(name.startswith("pmd_") for name in declared)


def test_abi_version():
    assert _lib.load().pmc_abi_version() == 2


def test_ctypes_structs_match_the_c_layout(tmp_path):
    structs = {
        "pmc_tables_desc": _lib.TablesDesc,
        "pmc_scoring_desc": _lib.ScoringDesc,
        "pmc_source_desc": _lib.SourceDesc,
        "pmc_beamlet_desc": _lib.BeamletDesc,
        "pmc_beamlet_rec": _lib.BeamletRec,
        "pmc_run_params": _lib.RunParams,
        "pmc_books": _lib.Books,
        "pmc_counters": _lib.Counters,
        "pmc_head_stack": _lib.HeadStack,
        "pmc_head_mu": _lib.HeadMu,
        "pmc_head_params": _lib.HeadParams,
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"',
             f'#include "{PRESOLVE_HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for field, _ in py._fields_:
            lines.append(f'printf("{cname}.{field} %zu\\n", offsetof({cname}, {field}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                       check=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for field, _ in py._fields_:
            assert int(got[f"{cname}.{field}"]) == getattr(py, field).offset, f"{cname}.{field}"


def test_null_engine_arguments_are_rejected_without_a_device():
    lib = _lib.load()
    assert lib.pmc_create(None, 0) == _lib.PMC_ERR_INVALID
    assert lib.pmc_upload_tables(None, None) == _lib.PMC_ERR_INVALID
    assert lib.pmc_run_forward(None, None, None, None, None, None) == _lib.PMC_ERR_INVALID
    assert lib.pmc_last_error(None) == b"no engine"


@pytest.mark.skipif(cuda_available(), reason="checks the no-device behaviour")
def test_engine_refuses_to_run_without_a_cuda_device():
    import pyradmc_b200 as P

    grid = P.VoxelGrid.uniform_water((4, 4, 4), (1.0, 1.0, 1.0))
    engine = P.B200Engine(grid, P.AnalyticWaterTables())
    src = P.PencilBeamSource(6.0, (2.0, 2.0, -1.0), (0.0, 0.0, 1.0))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        engine.run(src, n_histories=10, n_batches=2, seed=1)
    with pytest.raises(ValueError, match="CUDA devices only"):
        P.B200Engine(grid, P.AnalyticWaterTables(), device="cpu").run(src, n_histories=10,
                                                                       n_batches=2, seed=1)


def test_pack_tables_match_the_reference_arrays():
    """The packed tables round-trip the reference's CrossSectionTables fields."""
    import pyradmc_b200 as P

    xs = P.AnalyticWaterTables(geometry_densities=((0, 1.85),))
    t = xs.build_tables(ecut=0.2, pcut=0.05, e_max=6.0 * (1 + 1e-6))
    base = P.AnalyticWaterTables().build_tables(ecut=0.2, pcut=0.05, e_max=6.0 * (1 + 1e-6))
    assert t.n_points == 2048 and t.mu_compton.shape == (1, 2048)
    assert np.allclose(t.majorant, 1.85 * base.majorant, rtol=1e-15, atol=0)
    with pytest.raises(ValueError, match="no water table pack"):
        xs.build_tables(ecut=0.2, pcut=0.05, e_max=7.0)
    with pytest.raises(ValueError, match="water only"):
        P.AnalyticWaterTables(geometry_densities=((1, 1.0),))
