"""Host-side contract of ``B200Engine`` that needs no GPU: argument validation
with the reference's exception types and messages (engine.py:512-550,
:1070-1091), before any device is touched."""

from __future__ import annotations

import pytest

import pyradmc_b200 as P


@pytest.fixture
def engine():
    grid = P.VoxelGrid.uniform_water((4, 4, 4), (1.0, 1.0, 1.0))
    return P.B200Engine(grid, P.AnalyticWaterTables())


SRC = P.PencilBeamSource(6.0, (2.0, 2.0, -1.0), (0.0, 0.0, 1.0))
LAT = P.BeamletGridSource(6.0, -1.0, (0.0, 4.0), (0.0, 4.0), 2, 2)


@pytest.mark.parametrize(
    "kwargs,match",
    [
        (dict(n_histories=0, n_batches=1), "at least one history"),
        (dict(n_histories=10, n_batches=3), "not divisible"),
        (dict(n_histories=10, n_batches=2, concurrent_batches=0), "at least one lane"),
        (dict(n_histories=10, n_batches=2, primary_kind="neutron"), "unknown primary_kind"),
        (dict(n_histories=10, n_batches=2, scoring_mode="dose"), "unknown scoring_mode"),
        (dict(n_histories=10, n_batches=2, scoring_mode="dose_to_water", transport_electrons=False),
         "requires electron transport"),
        (dict(n_histories=10, n_batches=2, msc_model="moliere"), "unknown msc_model"),
        (dict(n_histories=10, n_batches=2, deposit_resolution_cm=0.0), "must be positive"),
    ],
)
def test_run_validation(engine, kwargs, match):
    with pytest.raises(ValueError, match=match):
        engine.run(SRC, seed=1, **kwargs)


@pytest.mark.parametrize(
    "kwargs,match",
    [
        (dict(n_histories_per_beamlet=0, n_batches=1), "at least one history per beamlet"),
        (dict(n_histories_per_beamlet=10, n_batches=3), "not divisible"),
        (dict(n_histories_per_beamlet=[10, 20, 30], n_batches=2), "per-beamlet history counts"),
        (dict(n_histories_per_beamlet=[10, 20, 30, 31], n_batches=2), "not divisible"),
        (dict(n_histories_per_beamlet=10, n_batches=2, beamlet_group_size=0), "positive beamlet group"),
        (dict(n_histories_per_beamlet=10, n_batches=2, truncation=-1.0), "negative truncation"),
        (dict(n_histories_per_beamlet=10, n_batches=2, devices=[]), "at least one device"),
    ],
)
def test_run_dij_validation(engine, kwargs, match):
    with pytest.raises(ValueError, match=match):
        engine.run_dij(LAT, seed=1, **kwargs)


def test_unsupported_source_is_refused(engine):
    class Odd:
        max_energy = 1.0

    with pytest.raises(ValueError, match="unsupported source type"):
        engine.run(Odd(), n_histories=4, n_batches=2, seed=1)


def test_lattice_bounds_interpolate_edges():
    lat = P.BeamletGridSource(6.0, -1.0, (2.0, 14.0), (2.0, 14.0), 3, 2)
    assert lat.beamlet_bounds(0) == (2.0, 6.0, 2.0, 8.0)
    assert lat.beamlet_bounds(5) == (10.0, 14.0, 8.0, 14.0)
    assert lat.n_beamlets == 6


def test_spectrum_mirror_matches_the_packed_reference_cdf():
    import numpy as np

    from pyradmc_b200.model import DATA

    spec = P.ali_rogers_varian_6mv()
    with np.load(DATA / "spectrum_varian_6mv.npz") as z:
        assert np.array_equal(spec.cdf, z["cdf"])
    assert spec.max_energy == pytest.approx(5.76)
    assert 1.4 < spec.mean_energy < 1.8
