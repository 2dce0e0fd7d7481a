"""The oracle itself, pinned before it is trusted (CPU only).

* Philox4x32-10 against the published known-answer vectors (Random123 KAT file,
  Salmon et al. SC'11) — the generator the oracle and the device share.
* The numpy reduction against pyRadMC's own ``BatchedBeamletScorer`` /
  ``DijAssembler`` outputs on seeded quanta maps (tests/golden/reduction.npz),
  bit for bit.
* The C transport against pyRadMC ``ReferenceEngine`` runs on every golden case
  by the reference's batched chi-squared oracle, plus its own scheduling
  invariances (thread count) and the exact energy ledger.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import reduction, stats
from tests.conftest import CASES, GOLDEN, build_case, load_ref

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("counter,key,expected", KAT)
def test_philox_known_answers(counter, key, expected):
    assert tuple(int(v) for v in oracle.philox(counter, key)) == expected


@pytest.fixture(scope="module")
def red():
    with np.load(GOLDEN / "reduction.npz") as z:
        return {k: z[k] for k in z.files}


def test_fold_finalize_is_bit_exact_against_the_reference_scorer(red):
    mean, sigma, total = reduction.fold_finalize(red["quanta"], red["voxel_mass"], int(red["per_batch"]))
    assert np.array_equal(mean, red["mean"])
    assert np.array_equal(sigma, red["sigma"])
    assert total == int(red["quanta"].sum())


@pytest.mark.parametrize("trunc", ["0", "0.001", "0.2"])
def test_truncation_is_bit_exact_against_the_reference_assembler(red, trunc):
    indptr, indices, dose, sigma = reduction.truncate(red["mean"], red["sigma"], float(trunc))
    assert np.array_equal(indptr, red[f"indptr_{trunc}"])
    assert np.array_equal(indices, red[f"indices_{trunc}"])
    assert np.array_equal(dose, red[f"dose_{trunc}"])
    assert np.array_equal(sigma, red[f"sigma_{trunc}"])


def _oracle_case(name, mult, seed_offset=1, n_threads=None):
    grid, xs, src, run = build_case(name)
    tab = xs.build_tables(0.2, 0.05, src.max_energy * (1 + 1e-6))
    gs = xs.gs_grid_for(tab, [0])
    dij = "n_histories_per_beamlet" in run
    counts = ([run["n_histories_per_beamlet"] * mult] * src.n_beamlets if dij
              else [run["n_histories"] * mult])
    mean, sigma, books = oracle.run(
        grid, tab, gs, src, counts=counts, n_batches=run["n_batches"], seed=run["seed"] + seed_offset,
        forward=not dij, transport_electrons=run.get("transport_electrons", True),
        msc_model=run.get("msc_model", "gs"), primary_kind=run.get("primary_kind", "photon"),
        n_threads=n_threads)
    return grid, src, run, counts, mean, sigma, books


# The C oracle restates the built-in generators on the analytic water source
# and the voxel scoring grid only; mixtures, phase spaces, collimated sources,
# the packed multi-material source and cylindrical scoring are pinned on the
# GPU against the reference fixtures directly.
ORACLE_CASES = [n for n, c in CASES.items()
                if c["source"]["kind"] not in ("composite", "phasespace", "collimated", "collimated_beamlets",
                                         "masked_beamlets")
                and "cross_sections" not in c
                and "scoring" not in c]


@pytest.mark.parametrize("name", ORACLE_CASES)
def test_oracle_transport_matches_reference_engine(name):
    mult = 1 if name == "readme_pencil" else 4
    _, _, run, counts, mean, sigma, _ = _oracle_case(name, mult)
    ref = load_ref(name)
    rd = ref["dose"].reshape(len(counts), -1)
    rs = ref["dose_sigma"].reshape(len(counts), -1)
    for j in range(len(counts)):
        mask = stats.high_dose_mask(rd[j], rs[j], sigma[j], minimum=50)
        stats.assert_chi2_consistent_batched(rd[j], rs[j], int(ref["n_batches"]), mean[j], sigma[j],
                                             run["n_batches"], mask=mask)


def test_oracle_energy_ledger_is_exact():
    grid, src, run, counts, mean, sigma, books = _oracle_case("full_slab", 1)
    emitted = counts[0] * src.max_energy
    assert books["deposited"] + books["escaped"] == pytest.approx(emitted, rel=1e-9)
    mass = (grid.density * grid.voxel_volume).reshape(-1)
    assert (mean[0] * mass).sum() * counts[0] == pytest.approx(books["deposited"], rel=1e-9)


def test_oracle_is_thread_count_invariant():
    a = _oracle_case("full_slab", 1, n_threads=1)
    b = _oracle_case("full_slab", 1, n_threads=5)
    assert np.array_equal(a[4], b[4])
    assert np.array_equal(a[5], b[5])
    assert a[6] == b[6]
