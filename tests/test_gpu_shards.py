"""Column shards on the device: every rank's ``run_dij_shard`` (here all ranks
in one process, one after the other) merges into exactly the Dij that one
``run_dij`` computes: the same CSC bit for bit."""

from __future__ import annotations

import numpy as np
import pytest

from pyradmc_b200.engine import merge_shards
from tests.conftest import build_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("world", [2, 3])
def test_shards_merge_into_the_whole_dij(gpu, world):
    import pyradmc_b200 as P

    grid, xs, src, kw = build_case("dij_spectral")
    engine = P.B200Engine(grid, xs, device=gpu)
    counts = np.array([480, 960, 240, 720], dtype=np.int64)
    whole = engine.run_dij(src, counts, kw["n_batches"], kw["seed"], truncation=0.0)
    parts = [engine.run_dij_shard(src, counts, kw["n_batches"], kw["seed"], rank=r, world=world,
                                  truncation=0.0) for r in range(world)]
    merged = merge_shards(parts)
    for name in ("indptr", "indices", "dose", "sigma"):
        np.testing.assert_array_equal(getattr(merged, name), getattr(whole, name))
    assert merged.n_beamlets == whole.n_beamlets
    np.testing.assert_allclose(merged.energy_deposited, whole.energy_deposited, rtol=1e-12)
