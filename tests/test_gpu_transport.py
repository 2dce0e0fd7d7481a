"""B200 transport against the reference, through the C-ABI (CUDA device needed).

Mirrors the reference's own backend parity suite
(tests/integration/test_warp_backend.py, tests/dij/test_dij_warp.py):

* statistical equivalence with pyRadMC's ``ReferenceEngine`` on every golden
  case — the batched chi-squared detection oracle over the high-dose region;
* bit reproducibility within the device and bit-inertness of every scheduling
  knob (chunk size, block shape, graph vs host-driven drain, group size);
* the exact identities: a 1x1 lattice is the open field bit for bit, the energy
  ledger closes, uneven per-beamlet counts reproduce the equal-count columns;
* the device reduction equals pyRadMC's scorer and assembler bit for bit;
* failure paths: majorant violation, queue overflow and the step cap come back
  as RuntimeError from kernels that stop themselves (no fault, no hang).
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import pyradmc_b200 as P
from oracle import stats
from pyradmc_b200 import _lib
from tests.conftest import CASES, CT_CASE, GOLDEN, SEED, build_case, build_ct_case, load_ref

pytestmark = pytest.mark.gpu

ENERGY_BALANCE_RTOL = 1.0e-4  # float32 transport + 1e-9 MeV quanta (test_warp_backend.py:35)

FORWARD = [n for n, c in CASES.items() if "n_histories" in c["run"]]
DIJ = [n for n, c in CASES.items() if "n_histories_per_beamlet" in c["run"]]


def _engine(name, **kw):
    grid, xs, src, run = build_case(name)
    return P.B200Engine(grid, xs, **kw), src, run


@pytest.mark.parametrize("name", FORWARD)
def test_dose_matches_reference_engine(gpu, name):
    engine, src, run = _engine(name)
    mult = 2 if name == "readme_pencil" else 8
    run["n_histories"] *= mult
    result = engine.run(src, **run)
    ref = load_ref(name)
    mask = stats.high_dose_mask(ref["dose"], ref["dose_sigma"], result.dose_sigma,
                                fraction=CASES[name].get("chi2_fraction", 0.1), minimum=50)
    stats.assert_chi2_consistent_batched(ref["dose"], ref["dose_sigma"], int(ref["n_batches"]),
                                         result.dose, result.dose_sigma, result.n_batches, mask=mask,
                                         case=name)


@pytest.mark.parametrize("name", DIJ)
def test_dij_columns_match_reference_engine(gpu, name):
    engine, src, run = _engine(name)
    run["n_histories_per_beamlet"] *= 8
    dij = engine.run_dij(src, **run)
    ref = load_ref(name)
    for j in range(dij.n_beamlets):
        a, sa = ref["dose"][j], ref["dose_sigma"][j]
        b, sb = dij.column_dense(j).reshape(-1), dij.sigma_dense(j).reshape(-1)
        mask = stats.high_dose_mask(a, sa, sb, minimum=50)
        stats.assert_chi2_consistent_batched(a, sa, int(ref["n_batches"]), b, sb, dij.n_batches,
                                             mask=mask, case=f"{name} column {j}")


def test_dose_to_water_weights_the_bone_deposits_by_the_stopping_power_ratio(gpu):
    """The same histories scored both ways (scoring draws no random numbers):
    water voxels away from the bone get identical doses, bone voxels get the
    medium dose times the water/bone restricted stopping-power ratio at the
    depositing electron's energy (scoring/dose_to_water.py:67-84), a ratio
    bounded by the table's values from ECUT up."""
    grid, xs, src, run = build_case("dtw_bone")
    engine = P.B200Engine(grid, xs)
    run.pop("scoring_mode")
    w = engine.run(src, scoring_mode="dose_to_water", **run)
    m = engine.run(src, scoring_mode="dose_to_medium", **run)
    bone = np.asarray(grid.material) != 0
    near = bone.copy()
    near[:, :, 1:] |= bone[:, :, :-1]
    near[:, :, :-1] |= bone[:, :, 1:]
    np.testing.assert_array_equal(w.dose[~near], m.dose[~near])
    tab = xs.build_tables(0.2, 0.05, 6.0 * (1 + 1e-6))
    s = np.asarray(tab.stopping_restricted)
    e = np.exp(tab.electron_log_e_min + np.arange(tab.n_points) / tab.electron_inv_dlog)
    spr = (s[0] / s[4])[e >= 0.2]
    hit = bone & (m.dose > 0.05 * m.dose.max())
    ratio = w.dose[hit] / m.dose[hit]
    assert spr.min() * (1 - 1e-6) <= ratio.min() and ratio.max() <= spr.max() * (1 + 1e-6)
    assert ratio.mean() > 1.02  # water stops electrons better than cortical bone per gram
    assert w.energy_deposited == m.energy_deposited  # the ledger books physical energy


def test_ct_phantom_with_uneven_counts_matches_reference_engine(gpu):
    """The benchmark's Dij at reduced size: a 40^3 CT-like phantom (seeded
    ellipsoids of density 0.2-1.9 g/cc), 5 mm 6 MV spectral beamlets, uneven
    per-column counts.  pyRadMC's run_dij takes one count for all columns, so
    each column is compared with the reference run at its own count."""
    grid, xs, src = build_ct_case()
    lo, hi = CT_CASE["counts"]
    counts = [lo, hi, lo, hi]
    n_batches = CT_CASE["run"]["n_batches"]
    engine = P.B200Engine(grid, xs)
    dij = engine.run_dij(src, n_histories_per_beamlet=[4 * c for c in counts], n_batches=n_batches,
                         seed=SEED + 1, truncation=0.0)
    refs = {c: load_ref(f"ct_beamlets_{c}") for c in (lo, hi)}
    for j, c in enumerate(counts):
        ref = refs[c]
        a, sa = ref["dose"][j], ref["dose_sigma"][j]
        b, sb = dij.column_dense(j).reshape(-1), dij.sigma_dense(j).reshape(-1)
        for fraction in (0.1, 0.01):  # the beamlet core, then the penumbra and low-dose tail
            mask = stats.high_dose_mask(a, sa, sb, fraction=fraction, minimum=50)
            stats.assert_chi2_consistent_batched(
                a, sa, int(ref["n_batches"]), b, sb, dij.n_batches, mask=mask,
                case=f"ct_beamlets column {j} ({c} histories, >= {fraction:g} of max)")


def _same(a, b):
    assert np.array_equal(a.dose, b.dose)
    assert np.array_equal(a.dose_sigma, b.dose_sigma)
    assert a.energy_deposited == b.energy_deposited
    assert a.energy_escaped == b.energy_escaped
    assert a.energy_unscored == b.energy_unscored


def test_bit_reproducible_within_device(gpu):
    engine, src, run = _engine("full_slab")
    _same(engine.run(src, **run), engine.run(src, **run))


@pytest.mark.parametrize("knobs", [
    dict(use_graph=False),
    dict(chunk_size=300),
    dict(chunk_size=5000, block_size=128),
    dict(blocks_per_sm=1, block_size=64),
    dict(queue_factor=64, chunk_size=1000),
    dict(tail_steps=1),  # every particle parked after one step once its round runs dry
    dict(tail_steps=-1),  # never parked
    dict(smem_tables=False),
    dict(smem_tables=True, tail_steps=7, use_graph=False),
])
def test_scheduling_knobs_are_bit_inert(gpu, knobs):
    base, src, run = _engine("full_slab")
    other, _, _ = _engine("full_slab", **knobs)
    _same(base.run(src, **run), other.run(src, **run))


def test_spectral_and_electron_routes_are_bit_inert(gpu):
    for name in ("slab_spectral", "electron_beam"):
        a, src, run = _engine(name)
        b, _, _ = _engine(name, chunk_size=777, use_graph=False, tail_steps=3, smem_tables=False)
        _same(a.run(src, **run), b.run(src, **run))


def test_ct_dij_is_bit_inert_to_parking_and_table_placement(gpu):
    grid, xs, src = build_ct_case()
    kw = dict(n_histories_per_beamlet=[20_000, 60_000, 20_000, 60_000], n_batches=10, seed=SEED,
              truncation=1e-3)
    a = P.B200Engine(grid, xs).run_dij(src, **kw)
    b = P.B200Engine(grid, xs, tail_steps=2, smem_tables=False, chunk_size=4096).run_dij(src, **kw)
    for f in ("indptr", "indices", "dose", "sigma"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert a.energy_deposited == b.energy_deposited and a.energy_escaped == b.energy_escaped


@pytest.mark.parametrize("transport_electrons", [False, True])
def test_energy_ledger_closes(gpu, transport_electrons):
    engine, src, run = _engine("full_slab")
    run["transport_electrons"] = transport_electrons
    r = engine.run(src, **run)
    balance = r.energy_deposited + r.energy_escaped + r.energy_unscored
    assert balance == pytest.approx(r.energy_emitted, rel=ENERGY_BALANCE_RTOL)
    mass = (engine.grid.density * engine.grid.voxel_volume)
    assert (r.dose * mass).sum() * r.n_histories == pytest.approx(r.energy_deposited, rel=1e-9)


def test_sigma_is_scored(gpu):
    engine, src, run = _engine("full_slab")
    r = engine.run(src, **run)
    high = r.dose > 0.5 * r.dose.max()
    assert np.all(r.dose_sigma[high] > 0.0)


def test_single_beamlet_is_the_open_field_bitwise(gpu):
    grid, xs, _, _ = build_case("dij_lattice")
    engine = P.B200Engine(grid, xs)
    lattice = P.BeamletGridSource(6.0, -1.0, (2.0, 14.0), (2.0, 14.0), 1, 1)
    field = P.ParallelBeamSource(6.0, -1.0, (2.0, 14.0), (2.0, 14.0))
    dij = engine.run_dij(lattice, n_histories_per_beamlet=2000, n_batches=4, seed=SEED,
                         truncation=0.0)
    run = engine.run(field, n_histories=2000, n_batches=4, seed=SEED)
    np.testing.assert_array_equal(dij.column_dense(0), run.dose)
    np.testing.assert_array_equal(dij.sigma_dense(0), run.dose_sigma)
    assert dij.energy_deposited == run.energy_deposited
    assert dij.energy_escaped == run.energy_escaped
    assert dij.energy_emitted == run.energy_emitted


@pytest.mark.parametrize("group", [1, 3])
def test_beamlet_group_size_is_bit_inert(gpu, group):
    engine, src, run = _engine("dij_lattice")
    run["truncation"] = 1e-3
    a = engine.run_dij(src, beamlet_group_size=4, **run)
    b = engine.run_dij(src, beamlet_group_size=group, **run)
    for f in ("indptr", "indices", "dose", "sigma"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
    assert a.energy_deposited == b.energy_deposited and a.energy_escaped == b.energy_escaped


def test_released_device_memory_is_rebuilt_bit_for_bit(gpu):
    """release_device_memory frees the engine's buffers; the next call uploads
    and allocates again (on the stream the caller set) and gives the same Dij,
    also when the second upload reuses the freed sizes."""
    import torch

    engine, src, run = _engine("dij_lattice")
    run["truncation"] = 1e-3
    stream = torch.cuda.Stream(device=gpu)
    engine.use_stream(stream.cuda_stream)
    a = engine.run_dij(src, **run)
    engine.release_device_memory()
    b = engine.run_dij(src, **run)
    engine.drop_uploads()  # same sizes again: the buffers are reused, not reallocated
    c = engine.run_dij(src, **run)
    for f in ("indptr", "indices", "dose", "sigma"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f))
        np.testing.assert_array_equal(getattr(a, f), getattr(c, f))
    assert engine._streams[engine.device] == stream.cuda_stream  # re-applied to the new engine


def test_uneven_counts_reproduce_equal_count_columns(gpu):
    """Correlated keys are the within-beamlet index r, so a column depends only
    on its own count: uneven counts give, column by column, the equal-count Dij."""
    engine, src, run = _engine("dij_lattice")
    counts = [800, 1600, 2400, 800]
    run.pop("n_histories_per_beamlet")
    uneven = engine.run_dij(src, n_histories_per_beamlet=counts, **run)
    for j, n in enumerate(counts):
        equal = engine.run_dij(src, n_histories_per_beamlet=n, **run)
        np.testing.assert_array_equal(uneven.column_dense(j), equal.column_dense(j))
        np.testing.assert_array_equal(uneven.sigma_dense(j), equal.sigma_dense(j))


def test_independent_mapping_with_uneven_counts_uses_global_offsets(gpu):
    engine, src, run = _engine("dij_lattice")
    run.pop("n_histories_per_beamlet")
    run["correlated"] = False
    a = engine.run_dij(src, n_histories_per_beamlet=[800, 800, 800, 800], **run)
    b = engine.run_dij(src, n_histories_per_beamlet=800, **run)
    np.testing.assert_array_equal(a.dose, b.dose)


def test_fluence_sum_reproduces_the_open_field(gpu):
    """Mean of untruncated independent columns is an open-field estimate
    (tests/dij/test_dij_ref.py:71-127), compared by batched chi-squared."""
    grid, xs, _, _ = build_case("dij_lattice")
    engine = P.B200Engine(grid, xs)
    lattice = P.BeamletGridSource(6.0, -1.0, (2.0, 14.0), (2.0, 14.0), 2, 2)
    field = P.ParallelBeamSource(6.0, -1.0, (2.0, 14.0), (2.0, 14.0))
    dij = engine.run_dij(lattice, n_histories_per_beamlet=8000, n_batches=8, seed=SEED,
                         transport_electrons=False, truncation=0.0, correlated=False)
    run = engine.run(field, n_histories=32000, n_batches=8, seed=SEED + 1,
                     transport_electrons=False)
    n = dij.n_beamlets
    dose_sum = dij.dose_for_weights(np.full(n, 1.0 / n))
    var = sum(dij.sigma_dense(j) ** 2 for j in range(n))
    sigma_sum = np.sqrt(var) / n
    mask = stats.high_dose_mask(run.dose, run.dose_sigma, sigma_sum, minimum=200)
    stats.assert_chi2_consistent_batched(dose_sum, sigma_sum, dij.n_batches, run.dose,
                                         run.dose_sigma, run.n_batches, mask=mask)


def test_truncation_keeps_entries_at_or_above_the_column_threshold(gpu):
    engine, src, run = _engine("dij_lattice")
    run["truncation"] = 0.05
    dij = engine.run_dij(src, **run)
    run["truncation"] = 0.0
    full = engine.run_dij(src, **run)
    for j in range(dij.n_beamlets):
        col = full.column_dense(j).reshape(-1)
        keep = np.flatnonzero((col >= 0.05 * col.max()) & (col > 0))
        lo, hi = dij.indptr[j], dij.indptr[j + 1]
        np.testing.assert_array_equal(dij.indices[lo:hi], keep)
        np.testing.assert_array_equal(dij.dose[lo:hi], col[keep])


# ---- the device reduction, bit for bit ------------------------------------------------
@pytest.fixture(scope="module")
def native(gpu):
    grid = P.VoxelGrid.uniform_water((2, 2, 2), (1.0, 1.0, 1.0))
    engine = P.B200Engine(grid, P.AnalyticWaterTables())
    return engine._native()


def test_device_fold_and_finalize_match_the_reference_scorer(native):
    with np.load(GOLDEN / "reduction.npz") as z:
        red = {k: z[k] for k in z.files}
    q = np.ascontiguousarray(red["quanta"])
    nb, nc, nv = q.shape
    mass = np.ascontiguousarray(red["voxel_mass"])
    per = np.full(nc, float(red["per_batch"]))
    mean = np.zeros(nc * nv)
    sigma = np.zeros(nc * nv)
    total = C.c_int64()
    native.check(native.lib.pmc_reduce_dense(native.handle, _lib.ptr(q, C.c_int64), nb, nc, nv,
                                             _lib.ptr(mass, C.c_double), _lib.ptr(per, C.c_double),
                                             _lib.ptr(mean, C.c_double), _lib.ptr(sigma, C.c_double),
                                             C.byref(total)))
    assert np.array_equal(mean.reshape(nc, nv), red["mean"])
    assert np.array_equal(sigma.reshape(nc, nv), red["sigma"])
    assert total.value == int(q.sum())


@pytest.mark.parametrize("trunc", ["0", "0.001", "0.2"])
def test_device_truncation_matches_the_reference_assembler(native, trunc):
    with np.load(GOLDEN / "reduction.npz") as z:
        red = {k: z[k] for k in z.files}
    mean = np.ascontiguousarray(red["mean"])
    sigma = np.ascontiguousarray(red["sigma"])
    nc, nv = mean.shape
    counts = np.zeros(nc, dtype=np.int64)
    nnz = C.c_int64()
    native.check(native.lib.pmc_truncate_dense(native.handle, _lib.ptr(mean, C.c_double),
                                               _lib.ptr(sigma, C.c_double), nc, nv, float(trunc),
                                               _lib.ptr(counts, C.c_int64), C.byref(nnz)))
    indptr = np.zeros(nc + 1, dtype=np.int64)
    idx = np.zeros(nnz.value, dtype=np.int64)
    dose = np.zeros(nnz.value)
    sig = np.zeros(nnz.value)
    native.check(native.lib.pmc_dij_fetch(native.handle, _lib.ptr(indptr, C.c_int64),
                                          _lib.ptr(idx, C.c_int64), _lib.ptr(dose, C.c_double),
                                          _lib.ptr(sig, C.c_double)))
    np.testing.assert_array_equal(indptr, red[f"indptr_{trunc}"])
    np.testing.assert_array_equal(idx, red[f"indices_{trunc}"])
    np.testing.assert_array_equal(dose, red[f"dose_{trunc}"])
    np.testing.assert_array_equal(sig, red[f"sigma_{trunc}"])


# ---- failure paths: the device stops itself, the host raises -------------------------------
def test_majorant_violation_raises(gpu):
    grid = P.VoxelGrid(shape=(4, 4, 8), spacing=(1.0, 1.0, 1.0),
                       density=np.full((4, 4, 8), 1.85), material=np.zeros((4, 4, 8), np.int32))
    engine = P.B200Engine(grid, P.AnalyticWaterTables(((0, 1.0),)))  # declares rho 1.0 only
    with pytest.raises(RuntimeError, match="majorant"):
        engine.run(P.PencilBeamSource(6.0, (2.0, 2.0, -1.0), (0, 0, 1)), n_histories=2000,
                   n_batches=2, seed=SEED)


def test_queue_overflow_raises_instead_of_dropping(gpu):
    grid, xs, src, run = build_case("readme_pencil")
    engine = P.B200Engine(grid, xs, chunk_size=1, queue_factor=1)
    run["n_histories"] = 2000
    with pytest.raises(RuntimeError, match="queue overflow"):
        engine.run(src, **run)


def test_step_cap_stops_the_kernel_and_raises(gpu):
    grid, xs, src, run = build_case("readme_pencil")
    engine = P.B200Engine(grid, xs, max_steps=2)
    run["n_histories"] = 1000
    with pytest.raises(RuntimeError, match="step cap"):
        engine.run(src, **run)
    # the context stays usable afterwards
    ok = P.B200Engine(grid, xs).run(src, **run)
    assert ok.energy_deposited > 0


def test_progress_ticks_once_per_batch(gpu):
    engine, src, run = _engine("full_slab")
    events = []
    engine.run(src, progress=events.append, **run)
    assert len(events) == run["n_batches"]
    assert events[-1].histories_done == events[-1].histories_total == run["n_histories"]


def test_native_library_is_the_in_tree_build(gpu):
    import os

    maps = open(f"/proc/{os.getpid()}/maps").read()
    assert str(_lib.library_path()) in maps
