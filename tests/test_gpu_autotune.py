"""The autotuner on the device: it probes real launch shapes of the engine,
confirms on every probe that the Dij does not change by one bit, and the tuned
engine's full Dij equals the default engine's."""

from __future__ import annotations

import numpy as np
import pytest

from pyradmc_b200 import autotune as T
from tests.conftest import build_case

pytestmark = pytest.mark.gpu


def test_tuned_engine_is_bit_identical_to_the_default(gpu, tmp_path):
    import pyradmc_b200 as P

    grid, xs, src, kw = build_case("dij_spectral")
    engine = P.B200Engine(grid, xs, device=gpu)
    counts = np.full(src.n_beamlets, 2000, dtype=np.int64)
    shapes = [T.LaunchShape(128, None, 50_000), T.LaunchShape(256, 2, 400_000),
              T.LaunchShape(192, None, 1_000_000)]
    tuned, report = T.tune(engine, src, counts, 10, 7, fraction=0.5, repeats=1, shapes=shapes,
                           cache=tmp_path / "tune.json")
    assert not report["cached"] and len(report["timings"]) == 3
    assert T.LaunchShape(tuned.block_size, tuned.blocks_per_sm, tuned.chunk_size) in shapes
    a = engine.run_dij(src, counts, 10, 7)
    b = tuned.run_dij(src, counts, 10, 7)
    assert T.digest(a) == T.digest(b)
    again, report2 = T.tune(engine, src, counts, 10, 7, cache=tmp_path / "tune.json")
    assert report2["cached"] and again.block_size == tuned.block_size
