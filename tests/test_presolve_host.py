"""The head pre-solve's host side (no GPU): the fixture, the descriptors built
from pyRadMC's own objects, and the argument checks of resolve_presolve
(geometry/head.py:340-370)."""

from __future__ import annotations

import os
import sys
from pathlib import Path

import numpy as np
import pytest

from pyradmc_b200 import presolve as PS
from tests.golden import presolve_case as case

GOLDEN = Path(__file__).resolve().parent / "golden" / "presolve_golden.npz"
SOURCE = os.environ.get("PYRADMC_SOURCE", "/root/reference")  # the pyRadMC checkout, when present


def golden():
    return np.load(GOLDEN)


def compiled(g, tag: str) -> PS.CompiledHeadStack:
    names = [f for f in PS.CompiledHeadStack.__dataclass_fields__ if f not in ("materials", "densities", "_keep")]
    return PS.CompiledHeadStack(**{n: g[f"{tag}_{n}"] for n in names},
                                materials=tuple(int(m) for m in g[f"{tag}_materials"]),
                                densities=tuple(float(d) for d in g[f"{tag}_densities"]))


def test_fixture_holds_every_case():
    g = golden()
    for tag in ("att", "fc", "air"):
        t = g[f"{tag}_totals"]
        assert t[0] > 0 and t[1] > 0 and t[5] > 0
    assert g["att_totals"][4] == 0 and g["fc_totals"][4] == 0 and g["air_totals"][4] > 0
    assert g["mu_log_total"].shape == (3, 512)
    s = compiled(g, "s1")
    assert s.n_devices == 2 and s.exit_z == case.MLC["z_bottom"]


def test_descriptor_arrays_reach_the_c_struct():
    s = compiled(golden(), "s2")
    c = s.to_c()
    assert c.n_devices == 3 and c.n_leaf_edges == 5 and c.n_tips == 4
    assert c.kind[2] == 1 and c.jaw_focused[0] == 1 and c.mlc_focused_sides[2] == 1
    assert c.rotation[8] == 1.0 and c.origin[2] == case.FOCAL[2]


def test_argument_checks():
    s = compiled(golden(), "s1")
    with pytest.raises(ValueError, match="mode"):
        PS.resolve_presolve(s, None, 60.0, "fast")
    with pytest.raises(ValueError, match="above the stack exit"):
        PS.resolve_presolve(s, None, 49.0, "auto")
    with pytest.raises(ValueError, match="inside the stack"):
        PS.resolve_presolve(s, PS.AirColumn(45.0, 90.0), 95.0, "auto")
    with pytest.raises(ValueError, match="above the air column end"):
        PS.resolve_presolve(s, PS.AirColumn(51.0, 95.0), 90.0, "auto")
    with pytest.raises(ValueError, match="requires a stack"):
        PS.resolve_presolve(None, None, 60.0, "auto")
    assert PS.resolve_presolve(s, None, 60.0, "auto") == "first_compton"
    assert PS.resolve_presolve(s, None, 60.0, "attenuation") == "attenuation"
    with pytest.raises(ValueError):
        PS.AirColumn(0.0, 10.0)
    with pytest.raises(ValueError):
        PS.AirColumn(10.0, 20.0, density=0.0)


@pytest.mark.skipif(not os.path.isdir(os.path.join(SOURCE, "pyradmc")), reason="pyRadMC is not available here")
def test_descriptors_from_pyradmc_objects_equal_the_fixture():
    if SOURCE not in sys.path:
        sys.path.insert(0, SOURCE)
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.collimation import MLC, BeamFrame, BeamLimitingStack, JawPair

    g = golden()
    stack = BeamLimitingStack(frame=BeamFrame(origin=case.FOCAL), devices=(JawPair(**case.JAW), MLC(**case.MLC)))
    got = PS.CompiledHeadStack.from_stack(stack)
    ref = compiled(g, "s1")
    for name in PS.CompiledHeadStack.__dataclass_fields__:
        if name != "_keep":
            np.testing.assert_array_equal(np.asarray(getattr(got, name)), np.asarray(getattr(ref, name)), name)
    pairs = (*zip(stack.materials, stack.densities, strict=True), (case.AIR["material"], case.AIR["density"]))
    mu = PS.HeadMuTables.build(AnalyticCrossSections(), pairs, 0.010, case.FanSource.max_energy, 512)
    np.testing.assert_allclose(mu.log_energy, g["mu_log_energy"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(mu.log_total, g["mu_log_total"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(mu.log_compton, g["mu_log_compton"], rtol=0, atol=1e-12)
