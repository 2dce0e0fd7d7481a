"""The head pre-solve on the GPU against pyRadMC's host pre-solve
(geometry/head.py:373-575) through the committed fixture
(tests/golden/make_presolve_golden.py), with the checks and tolerances of the
reference's own device test (tests/physics/test_warp_presolve.py:95-165):

* chord lengths through jaws (straight and focused, both axes) and MLCs
  (straight and focused sides, rounded tips, open and closed pairs) equal the
  reference's float64 lengths to float32 precision;
* attenuation mode is deterministic geometry: the same kept count and, to
  2e-3, the same summed weight and weight-energy;
* first-Compton mode (with and without the air column) draws from this
  backend's own streams: totals within 0.5 %, the mean energy within 0.2 %,
  the contaminant electrons within 2 %, and the energy spectra of both kinds
  consistent bin by bin;
* the output is a deterministic function of the seed, and the engine
  transports it as a phase-space source.
"""

from __future__ import annotations

import numpy as np
import pytest

from pyradmc_b200 import presolve as PS
from tests.golden import presolve_case as case
from tests.test_presolve_host import compiled, golden

pytestmark = pytest.mark.gpu


def _mu(g):
    return PS.HeadMuTables(g["mu_log_energy"], g["mu_log_total"], g["mu_log_compton"])


def _run(g, gpu, mode, air=False, seed=case.SEED, **kw):
    return PS.presolve_head_device(
        case.FanSource(), n_histories=case.N, seed=seed,
        exit_z=case.AIR_EXIT_Z if air else case.EXIT_Z, stack=compiled(g, "s1"),
        air=PS.AirColumn(**case.AIR) if air else None, mode=mode, device=gpu,
        mu_tables=_mu(g), **kw)


def _totals(ps):
    c = ps.columns()
    w = c["weight"].astype(np.float64)
    e = c["energy"].astype(np.float64)
    k = c["particle_type"]
    return np.array([len(ps), w.sum(), (w * e).sum(), np.count_nonzero(k == 1), np.count_nonzero(k == 2),
                     (w * e).sum() / w.sum()])


@pytest.mark.parametrize("tag", ["s1", "s2"])
def test_chord_lengths_equal_the_reference(gpu, tag):
    g = golden()
    s = compiled(g, tag)
    for name, fwd in (("len_full", False), ("len_fwd", True)):
        got = PS.stack_path_lengths(s, g[f"{tag}_ray_p"], g[f"{tag}_ray_d"], from_origin=fwd).astype(np.float64)
        ref = g[f"{tag}_{name}"]
        inf = ~np.isfinite(ref)
        assert np.array_equal(~np.isfinite(got), inf), name
        fin = ~inf
        assert (ref[fin] > 0).mean() > 0.1, "the rays must actually cross the devices"
        # float32 geometry over ~100 cm lever arms
        np.testing.assert_allclose(got[fin], ref[fin], rtol=1e-4, atol=2e-3, err_msg=f"{tag} {name}")


def test_attenuation_mode_matches_the_host_to_float32(gpu):
    g = golden()
    got = _totals(_run(g, gpu, "attenuation"))
    host = g["att_totals"]
    assert got[0] == host[0] and got[4] == 0
    np.testing.assert_allclose(got[1], host[1], rtol=2e-3)
    np.testing.assert_allclose(got[2], host[2], rtol=2e-3)


def test_first_compton_totals_match_the_host_statistically(gpu):
    g = golden()
    ps = _run(g, gpu, "first_compton")
    got, host = _totals(ps), g["fc_totals"]
    assert got[4] == 0  # no air, no contaminant electrons
    np.testing.assert_allclose(got[0], host[0], rtol=5e-3)
    np.testing.assert_allclose(got[1], host[1], rtol=5e-3)
    np.testing.assert_allclose(got[2], host[2], rtol=5e-3)
    np.testing.assert_allclose(got[5], host[5], rtol=2e-3)
    _spectra_agree(ps, g, "fc", kinds=((1, "photon"),))


def test_air_column_adds_contaminant_electrons_matching_the_host(gpu):
    g = golden()
    ps, dropped = _run(g, gpu, "first_compton", air=True, return_dropped=True)
    got, host = _totals(ps), g["air_totals"]
    assert got[4] > 0
    np.testing.assert_allclose(got[4], host[4], rtol=2e-2)
    np.testing.assert_allclose(got[1], host[1], rtol=5e-3)
    np.testing.assert_allclose(got[2], host[2], rtol=5e-3)
    assert dropped >= 0.0
    _spectra_agree(ps, g, "air", kinds=((1, "photon"), (2, "electron")))


def _spectra_agree(ps, g, tag, kinds):
    c = ps.columns()
    bins = np.linspace(0.0, 6.0, 25)
    for k, name in kinds:
        m = c["particle_type"] == k
        w = c["weight"][m].astype(np.float64)
        e = c["energy"][m].astype(np.float64)
        a, a2 = np.histogram(e, bins=bins, weights=w)[0], np.histogram(e, bins=bins, weights=w * w)[0]
        b, b2 = g[f"{tag}_{name}_hist"], g[f"{tag}_{name}_hist2"]
        use = (a2 + b2) > 0
        z = (a[use] - b[use]) / np.sqrt(a2[use] + b2[use])
        # the transmitted backbone is common to both runs, so these z-scores are
        # conservative; a systematic error shows as a large one
        assert np.abs(z).max() < 5.0, (name, z)


def test_output_is_a_function_of_the_seed_and_the_engine_transports_it(gpu):
    from pyradmc_b200 import B200Engine
    from pyradmc_b200.model import AnalyticWaterTables, VoxelGrid

    g = golden()
    a = _run(g, gpu, "first_compton", air=True)
    b = _run(g, gpu, "first_compton", air=True)
    for name in ("particle_type", "energy", "x", "y", "z", "ux", "uy", "uz", "weight"):
        np.testing.assert_array_equal(a.columns()[name], b.columns()[name])
    c = _run(g, gpu, "first_compton", air=True, seed=case.SEED + 1)
    assert not np.array_equal(a.columns()["energy"], c.columns()["energy"])
    # the phase space on a water block below the exit plane
    grid = VoxelGrid.uniform_water((16, 16, 16), (1.0, 1.0, 1.0), origin=(0.0, 0.0, -4.5))  # exit plane: z = -5
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    res = B200Engine(grid, xs, device=gpu).run(a, n_histories=40_000, n_batches=4, seed=case.SEED)
    assert res.dose.max() > 0
    balance = res.energy_deposited + res.energy_escaped + res.energy_unscored
    assert balance == pytest.approx(res.energy_emitted, rel=1e-4)


def test_device_phase_space_is_transported_in_place_with_the_same_dose(gpu):
    """return_device_source keeps the population on the GPU; the engine reads it
    in place (PMC_SRC_PHASESPACE_DEVICE) and scores exactly the dose of the
    same phase space copied to the host and uploaded again."""
    from pyradmc_b200 import B200Engine
    from pyradmc_b200.model import AnalyticWaterTables, VoxelGrid

    g = golden()
    host = _run(g, gpu, "first_compton", air=True)
    dev = _run(g, gpu, "first_compton", air=True, return_device_source=True)
    assert len(dev) == len(host)
    for name in ("particle_type", "energy", "weight"):
        np.testing.assert_allclose(dev.columns()[name], host.columns()[name], rtol=1e-6, atol=0)
    grid = VoxelGrid.uniform_water((16, 16, 16), (1.0, 1.0, 1.0), origin=(0.0, 0.0, -4.5))
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    engine = B200Engine(grid, xs, device=gpu)
    a = engine.run(host, n_histories=40_000, n_batches=4, seed=case.SEED)
    b = engine.run(dev, n_histories=40_000, n_batches=4, seed=case.SEED)
    np.testing.assert_array_equal(a.dose, b.dose)
    np.testing.assert_array_equal(a.dose_sigma, b.dose_sigma)
    assert a.energy_emitted == b.energy_emitted
