"""Beamlet sources beyond the two built-in generators, through the C-ABI (CUDA
device needed).

* A concatenation of beamlet sources (a multi-beam plan as one Dij) gives, for
  correlated sampling, exactly the columns of the separate runs: the stream key
  of a history is its within-beamlet index, whatever column it lands in.
* A per-beamlet mixture (CompositeBeamletSource, geometry/source.py:239-277)
  is pinned against pyRadMC's ReferenceEngine in test_gpu_transport.py
  (``dij_composite``); here its mean is checked against the weighted sum of its
  components' Dijs.
* The host pre-sampling route (BeamletSource.sample_beamlet_batch, the Warp
  engine's ``_generate_group_presampled``, engine.py:3224-3335) transports the
  same primaries as the in-kernel fan, statistically.
"""

from __future__ import annotations

import numpy as np
import pytest

import pyradmc_b200 as P
from oracle import stats
from tests.conftest import GOLDEN, SEED, build_case

pytestmark = pytest.mark.gpu


def _water(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)):
    grid = P.VoxelGrid.uniform_water(shape, spacing)
    return grid, P.AnalyticWaterTables(geometry_densities=grid.max_density_by_material())


def _fan(focal, centers, u=(1.0, 0.0, 0.0), v=(0.0, 1.0, 0.0), width=1.5):
    return P.SpectralBeamletSource(P.ali_rogers_varian_6mv(), focal, centers, width, width, u, v)


class PresampledFan:
    """A beamlet source the engine cannot generate in-kernel: it only offers
    vectorized host sampling (the fan of _DivergentFan.sample_through_batch,
    geometry/source.py:508-549, with its own PCG64 stream)."""

    def __init__(self, fan):
        self.fan = fan
        self.n_beamlets = fan.n_beamlets
        self.max_energy = fan.max_energy

    def sample_beamlet_batch(self, seed, history_offset, n, beamlet):
        bitgen = np.random.PCG64(seed)
        bitgen.advance(4 * history_offset)
        u = np.random.Generator(bitgen).random((n, 4))
        sp = self.fan.spectrum
        k = np.minimum(np.searchsorted(sp.cdf, u[:, 0], side="left"), sp.cdf.size - 1)
        energy = sp.edges[k] + (sp.edges[k + 1] - sp.edges[k]) * u[:, 1]
        du = (u[:, 2] - 0.5) * self.fan.width_u
        dv = (u[:, 3] - 0.5) * self.fan.width_v
        focal = np.asarray(self.fan.focal_point)
        target = (np.asarray(self.fan.centers[beamlet]) + du[:, None] * np.asarray(self.fan.u_axis)
                  + dv[:, None] * np.asarray(self.fan.v_axis))
        d = target - focal
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        f32 = np.float32
        return {"particle_type": np.ones(n, np.int32), "energy": energy.astype(f32),
                "x": np.full(n, focal[0], f32), "y": np.full(n, focal[1], f32),
                "z": np.full(n, focal[2], f32), "ux": d[:, 0].astype(f32),
                "uy": d[:, 1].astype(f32), "uz": d[:, 2].astype(f32),
                "weight": np.ones(n, f32)}


def test_concatenated_beams_are_the_separate_dijs_bit_for_bit(gpu):
    grid, xs = _water()
    beam_z = _fan((4.0, 4.0, -100.0), [(3.0, 3.0, 0.0), (5.0, 5.0, 0.0)])
    beam_x = _fan((-100.0, 4.0, 4.0), [(4.0, 3.0, 3.0), (4.0, 5.0, 5.0), (4.0, 4.0, 4.0)],
                  u=(0.0, 1.0, 0.0), v=(0.0, 0.0, 1.0))
    # every part at the fans' top energy: the tables' log-energy nodes depend on
    # the call's maximum energy, so only then are the runs' physics tables equal
    lattice = P.BeamletGridSource(beam_z.max_energy, -1.0, (1.0, 7.0), (1.0, 7.0), 2, 1)
    plan = P.ConcatenatedBeamletSource([beam_z, beam_x, lattice])
    assert plan.max_energy == lattice.max_energy == beam_x.max_energy
    kw = dict(n_batches=4, seed=SEED, truncation=1e-3)
    engine = P.B200Engine(grid, xs)
    whole = engine.run_dij(plan, n_histories_per_beamlet=[4000, 8000, 4000, 4000, 8000, 4000, 4000], **kw)
    parts = [engine.run_dij(beam_z, n_histories_per_beamlet=[4000, 8000], **kw),
             engine.run_dij(beam_x, n_histories_per_beamlet=[4000, 4000, 8000], **kw),
             engine.run_dij(lattice, n_histories_per_beamlet=4000, **kw)]
    j = 0
    for part in parts:
        for k in range(part.n_beamlets):
            np.testing.assert_array_equal(whole.column_dense(j), part.column_dense(k))
            np.testing.assert_array_equal(whole.sigma_dense(j), part.sigma_dense(k))
            j += 1
    assert j == whole.n_beamlets == 7


def test_composite_mean_is_the_weighted_sum_of_its_components(gpu):
    grid, xs, src, run = build_case("dij_composite")
    engine = P.B200Engine(grid, xs)
    run["n_histories_per_beamlet"] = 16_000
    mix = engine.run_dij(src, correlated=False, **run)
    comps = [engine.run_dij(c, correlated=False, seed=run["seed"] + 1 + i,
                            **{k: v for k, v in run.items() if k != "seed"})
             for i, c in enumerate(src._sources)]
    w = np.diff(np.concatenate([[0.0], src._cdf]))
    for j in range(mix.n_beamlets):
        a = mix.column_dense(j).reshape(-1)
        sa = mix.sigma_dense(j).reshape(-1)
        b = sum(wk * c.column_dense(j).reshape(-1) for wk, c in zip(w, comps, strict=True))
        sb = np.sqrt(sum((wk * c.sigma_dense(j).reshape(-1)) ** 2 for wk, c in zip(w, comps, strict=True)))
        mask = stats.high_dose_mask(a, sa, sb, minimum=50)
        stats.assert_chi2_consistent_batched(a, sa, mix.n_batches, b, sb, mix.n_batches, mask=mask,
                                             case=f"composite = weighted components, column {j}")


def test_presampled_route_matches_the_in_kernel_fan(gpu):
    grid, xs = _water()
    fan = _fan((4.0, 4.0, -100.0), [(3.0, 3.0, 0.0), (5.0, 4.0, 0.0)])
    engine = P.B200Engine(grid, xs)
    kw = dict(n_histories_per_beamlet=[40_000, 80_000], n_batches=8, truncation=0.0)
    inner = engine.run_dij(fan, seed=SEED, **kw)
    host = engine.run_dij(PresampledFan(fan), seed=SEED + 5, **kw)
    for j in range(2):
        a, sa = inner.column_dense(j).reshape(-1), inner.sigma_dense(j).reshape(-1)
        b, sb = host.column_dense(j).reshape(-1), host.sigma_dense(j).reshape(-1)
        mask = stats.high_dose_mask(a, sa, sb, minimum=50)
        stats.assert_chi2_consistent_batched(a, sa, 8, b, sb, 8, mask=mask,
                                             case=f"presampled fan column {j}")
    # emitted energy is booked per uploaded primary; the ledger closes
    assert host.energy_emitted == pytest.approx(inner.energy_emitted, rel=0.01)
    balance = host.energy_deposited + host.energy_escaped + host.energy_unscored
    assert balance == pytest.approx(host.energy_emitted, rel=1e-4)


def test_a_failing_host_sampler_raises_its_own_exception(gpu):
    grid, xs = _water((8, 8, 8))

    class Broken(PresampledFan):
        def sample_beamlet_batch(self, *args):
            raise KeyError("no such beamlet file")

    with pytest.raises(KeyError, match="no such beamlet file"):
        P.B200Engine(grid, xs).run_dij(Broken(_fan((2.0, 2.0, -100.0), [(2.0, 2.0, 0.0)])),
                                       n_histories_per_beamlet=100, n_batches=2, seed=SEED)


class _HostSampled:
    """The phase space seen only through ``sample_batch``: the host
    pre-sampling route pyRadMC's Warp engine takes (engine.py:2833-2877)."""

    def __init__(self, inner):
        self.inner = inner
        self.max_energy = inner.max_energy

    def sample_batch(self, seed, history_offset, n):
        return self.inner.sample_batch(seed, history_offset, n)


def test_resident_phase_space_matches_host_sampling_and_closes_the_ledger(gpu):
    grid, xs, src, run = build_case("phasespace")
    # 10 % of the records are 0.5-3 MeV electrons and positrons that stop within
    # a few voxels of the entrance: at the fixture's 80k histories a surface
    # voxel sees a handful of them per batch, too few for normal batch means.
    # Both routes run here, so the comparison takes 10x the histories.
    run.update(n_histories=800_000, n_batches=20)
    engine = P.B200Engine(grid, xs)
    resident = engine.run(src, **run)
    host = engine.run(_HostSampled(src), **run)
    mask = stats.high_dose_mask(resident.dose, resident.dose_sigma, host.dose_sigma, minimum=200)
    stats.assert_chi2_consistent_batched(resident.dose, resident.dose_sigma, run["n_batches"],
                                         host.dose, host.dose_sigma, run["n_batches"], mask=mask,
                                         case="phase space: resident vs host-sampled")
    for r in (resident, host):  # weights and kinds (positron rest mass) threaded end to end
        balance = r.energy_deposited + r.energy_escaped + r.energy_unscored
        assert balance == pytest.approx(r.energy_emitted, rel=1e-4)
    assert resident.energy_emitted == pytest.approx(host.energy_emitted, rel=0.02)


def test_resident_phase_space_is_bit_inert_to_scheduling(gpu):
    grid, xs, src, run = build_case("phasespace")
    run["n_histories"] = 20_000
    a = P.B200Engine(grid, xs).run(src, **run)
    b = P.B200Engine(grid, xs, chunk_size=999, use_graph=False, tail_steps=5).run(src, **run)
    np.testing.assert_array_equal(a.dose, b.dose)
    np.testing.assert_array_equal(a.dose_sigma, b.dose_sigma)
    assert a.energy_emitted == b.energy_emitted


def _masked(fan, mask, width=4.0, **kw):
    axes = dict(u_axis=(0.0, 1.0, 0.0), v_axis=(1.0, 0.0, 0.0))
    axes.update(kw)
    return P.TransmissionMaskSource(fan, mask=mask, plane_center=(4.0, 4.0, -50.0), width_u=width,
                                    width_v=width, **axes)


def test_an_open_mask_is_bit_inert_and_a_closed_one_emits_nothing(gpu):
    """The spectral fan through a transmission mask (the Warp engine's
    generate_spectral_masked_beam, kernels.py:2137-2244).  An all-ones mask
    whose rectangle holds the whole fan leaves every primary at weight exactly
    1 (the incremental bilinear form is exact on a plateau), so the run is the
    unmasked fan's bit for bit; an all-zeros mask, or a rectangle the fan
    misses, emits nothing; a constant mask c books c times the emitted
    energy.  The masked dose itself is pinned against pyRadMC's
    ReferenceEngine in test_gpu_transport.py (``spectral_masked``)."""
    grid, xs = _water()
    engine = P.B200Engine(grid, xs)
    fan = P.SpectralBeamSource(P.ali_rogers_varian_6mv(), (4.0, 4.0, -100.0), (4.0, 4.0, 0.0), 6.0, 6.0)
    kw = dict(n_histories=40_000, n_batches=8, seed=SEED)
    plain = engine.run(fan, **kw)
    # the fan is 3 cm wide at the plane: a 4 cm rectangle holds all of it
    opened = engine.run(_masked(fan, np.ones((7, 3))), **kw)
    np.testing.assert_array_equal(opened.dose, plain.dose)
    np.testing.assert_array_equal(opened.dose_sigma, plain.dose_sigma)
    assert opened.energy_emitted == plain.energy_emitted
    assert opened.energy_deposited == plain.energy_deposited
    for closed in (_masked(fan, np.zeros((2, 2))),
                   P.TransmissionMaskSource(fan, mask=np.ones((2, 2)), plane_center=(20.0, 4.0, -50.0),
                                            width_u=4.0, width_v=4.0)):
        res = engine.run(closed, **kw)
        assert not res.dose.any() and res.energy_emitted == 0.0 and res.energy_deposited == 0.0
    half = engine.run(_masked(fan, np.full((3, 4), 0.5)), **kw)
    assert half.energy_emitted == pytest.approx(0.5 * plain.energy_emitted, rel=1e-8)


def test_the_native_path_rejects_a_bad_mask(gpu):
    """The C-ABI checks the mask as _MaskTransmission.__init__ does
    (geometry/collimation.py:1013-1023), whatever object the caller hands in:
    PMC_ERR_INVALID, a ValueError."""
    grid, xs = _water()
    engine = P.B200Engine(grid, xs)
    fan = P.SpectralBeamSource(P.ali_rogers_varian_6mv(), (4.0, 4.0, -100.0), (4.0, 4.0, 0.0), 6.0, 6.0)

    class TransmissionMaskSource:  # duck-typed, unchecked on the host
        inner = fan
        max_energy = fan.max_energy
        plane_center = (4.0, 4.0, -50.0)
        width_u = width_v = 4.0
        u_axis, v_axis = (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)

        def __init__(self, mask, **kw):
            self.mask = mask
            self.__dict__.update(kw)

    kw = dict(n_histories=1000, n_batches=1, seed=SEED)
    for bad, match in ((TransmissionMaskSource(np.full((2, 2), 1.5)), "within 0..1"),
                       (TransmissionMaskSource(np.full((2, 2), np.nan)), "within 0..1"),
                       (TransmissionMaskSource(np.ones((2, 2)), width_u=0.0), "widths"),
                       (TransmissionMaskSource(np.ones((2, 2)), v_axis=(0.6, 0.8, 0.0)), "orthogonal")):
        with pytest.raises(ValueError, match=match):
            engine.run(bad, **kw)


def _open_stack():
    """One jaw pair whose edges stand far outside every beam: zero chords."""
    from pyradmc_b200.presolve import CompiledHeadStack

    z = np.load(GOLDEN / "collimation.npz")
    stack = CompiledHeadStack(
        origin=z["stack_origin"], rotation=z["stack_rotation"], kind=np.array([0]), z_top=np.array([40.0]),
        z_bottom=np.array([45.0]), jaw_axis=np.array([0]), jaw_edge_neg=np.array([-1000.0]),
        jaw_edge_pos=np.array([1000.0]), jaw_focused=np.array([0]), mlc_tip_radius=np.zeros(1),
        mlc_focused_sides=np.zeros(1, dtype=np.int32), mlc_n_pairs=np.zeros(1, dtype=np.int32),
        mlc_edges_off=np.zeros(1, dtype=np.int32), mlc_tips_off=np.zeros(1, dtype=np.int32),
        leaf_edges_v=np.zeros(0), tips_neg=np.zeros(0), tips_pos=np.zeros(0), materials=(0,),
        densities=(3.0,))
    return stack, z["log_energy"], z["log_total"][:1]


def test_an_open_stack_is_bit_inert_and_a_closed_stack_attenuates(gpu):
    """Collimated sources (CollimatedSource / CollimatedBeamletSource,
    geometry/collimation.py:1154-1204) weight each in-kernel primary by the
    stack's transmission.  A stack no ray crosses transmits exactly 1, so the
    forward run and the Dij are the plain sources' bit for bit; the cases'
    stack (a jaw and a three-pair MLC of 3 g/cc water) books less emitted
    energy than the open fan and no more than it.  The collimated dose itself
    is pinned against pyRadMC's ReferenceEngine in test_gpu_transport.py
    (``collimated_spectral``, ``dij_collimated``)."""
    from tests.conftest import collimated

    grid, xs = _water()
    engine = P.B200Engine(grid, xs)
    fan = P.SpectralBeamSource(P.ali_rogers_varian_6mv(), (4.0, 4.0, -100.0), (4.0, 4.0, 0.0), 6.0, 6.0)
    stack, log_e, log_total = _open_stack()
    kw = dict(n_histories=40_000, n_batches=8, seed=SEED)
    plain = engine.run(fan, **kw)
    opened = engine.run(P.CollimatedSource.from_tables(fan, stack, log_e, log_total), **kw)
    np.testing.assert_array_equal(opened.dose, plain.dose)
    assert opened.energy_emitted == plain.energy_emitted
    closed = engine.run(collimated(fan, False), **kw)
    assert 0.2 * plain.energy_emitted < closed.energy_emitted < 0.95 * plain.energy_emitted

    beams = _fan((4.0, 4.0, -100.0), ((3.0, 3.0, 0.0), (5.0, 3.0, 0.0), (3.0, 5.0, 0.0)), width=2.0)
    dkw = dict(n_histories_per_beamlet=4000, n_batches=4, seed=SEED, truncation=0.0)
    a = engine.run_dij(beams, **dkw)
    b = engine.run_dij(P.CollimatedBeamletSource.from_tables(beams, stack, log_e, log_total), **dkw)
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.dose, b.dose)
    np.testing.assert_array_equal(a.sigma, b.sigma)
    lattice = P.BeamletGridSource(6.0, -1.0, (2.0, 6.0), (2.0, 6.0), 2, 2)
    c = engine.run_dij(lattice, **dkw)
    d = engine.run_dij(P.CollimatedBeamletSource.from_tables(lattice, stack, log_e, log_total), **dkw)
    np.testing.assert_array_equal(c.dose, d.dose)


def test_open_masks_are_bit_inert_on_every_in_kernel_source(gpu):
    """A mask of ones whose rectangle holds every ray weights nothing: a masked
    parallel field and masked beamlets (TransmissionMaskBeamletSource,
    geometry/collimation.py:1264) are the plain sources' runs bit for bit.  The
    masked Dij itself is pinned against pyRadMC's ReferenceEngine in
    test_gpu_transport.py (``dij_masked``)."""
    grid, xs = _water()
    engine = P.B200Engine(grid, xs)
    field = P.ParallelBeamSource(6.0, -1.0, (1.0, 7.0), (1.0, 7.0))
    kw = dict(n_histories=20_000, n_batches=4, seed=SEED)
    plain = engine.run(field, **kw)
    masked = engine.run(P.TransmissionMaskSource(field, mask=np.ones((3, 3)), plane_center=(4.0, 4.0, -50.0),
                                                 width_u=20.0, width_v=20.0), **kw)
    np.testing.assert_array_equal(masked.dose, plain.dose)
    assert masked.energy_emitted == pytest.approx(plain.energy_emitted, rel=1e-12)
    beams = _fan((4.0, 4.0, -100.0), ((3.0, 3.0, 0.0), (5.0, 3.0, 0.0), (3.0, 5.0, 0.0)), width=2.0)
    dkw = dict(n_histories_per_beamlet=4000, n_batches=4, seed=SEED, truncation=0.0)
    a = engine.run_dij(beams, **dkw)
    b = engine.run_dij(P.TransmissionMaskBeamletSource(beams, mask=np.ones((2, 5)),
                                                       plane_center=(4.0, 4.0, -50.0), width_u=4.0,
                                                       width_v=4.0), **dkw)
    np.testing.assert_array_equal(a.indptr, b.indptr)
    np.testing.assert_array_equal(a.dose, b.dose)
    np.testing.assert_array_equal(a.sigma, b.sigma)
