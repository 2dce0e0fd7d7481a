"""The launch-shape autotuner's host logic without a GPU: the search space, the
cache, the choice of the fastest candidate, and the refusal of a launch shape
that changes the Dij (the transport must be scheduling-inert)."""

from __future__ import annotations

import dataclasses
from types import SimpleNamespace

import numpy as np
import pytest

from pyradmc_b200 import autotune as T


@dataclasses.dataclass(frozen=True)
class FakeEngine:
    grid: object
    device: str = "cuda:0"
    chunk_size: int | None = None
    block_size: int | None = None
    blocks_per_sm: int | None = None
    tail_steps: int | None = None
    smem_tables: bool | None = None

    def drop_uploads(self):
        pass


def _dij(seed=0):
    rng = np.random.default_rng(seed)
    return SimpleNamespace(indptr=np.array([0, 3]), indices=np.array([1, 4, 9]),
                           dose=rng.random(3), sigma=rng.random(3))


def _fake_timer(calls):
    def timer(engine, source, counts, n_batches, seed):
        calls.append((engine.block_size, engine.blocks_per_sm, engine.chunk_size, int(counts.sum())))
        bs = engine.block_size or 256
        chunk = engine.chunk_size or 16 * 148 * 3 * bs
        t = abs(bs - 192) + (0 if engine.blocks_per_sm is None else 5)
        t += abs(chunk - 16 * 148 * 3 * bs) / 1e6
        t += 0.0 if engine.tail_steps == 256 else 0.5   # the second stage's favourite
        t += 0.0 if engine.smem_tables is None else 0.25
        return 1.0 + t, _dij()
    return timer


def test_search_space_covers_every_knob():
    shapes = T.candidates(148)
    assert len(shapes) == 1 + len(T.BLOCK_SIZES) * len(T.BLOCKS_PER_SM) * len(T.CHUNK_PER_THREAD)
    assert shapes[0] == T.LaunchShape(None, None, None)  # the engine's default competes too
    assert {s.block_size for s in shapes[1:]} == set(T.BLOCK_SIZES)
    assert all(s.chunk_size * 16 < 2 ** 31 for s in shapes[1:])  # queue index range at factor 16


def test_probe_counts_are_positive_batch_multiples():
    c = T.probe_counts([10, 1000, 123456], 0.1, 10)
    assert (c % 10 == 0).all() and (c >= 10).all() and c[2] == 12350


def test_tuner_picks_the_fastest_shape_and_caches_it(tmp_path):
    cache = tmp_path / "tune.json"
    engine = FakeEngine(grid=SimpleNamespace(shape=(128, 128, 128)))
    source = SimpleNamespace(n_beamlets=100)
    calls = []
    tuned, report = T.tune(engine, source, np.full(100, 200_000), 10, 1, cache=cache,
                           timer=_fake_timer(calls), sm_count=148, device_name="B200")
    assert (tuned.block_size, tuned.blocks_per_sm) == (192, None)
    assert tuned.chunk_size == 16 * 148 * 3 * 192
    assert (tuned.tail_steps, tuned.smem_tables) == (256, None)  # refined on the best geometry
    stage2 = T.refinements(T.LaunchShape(192, None, 16 * 148 * 3 * 192))
    assert len(stage2) == len(T.TAIL_STEPS) * len(T.SMEM_TABLES)  # the best itself is among them
    assert not report["cached"]
    assert len(report["timings"]) == len(T.candidates(148)) + len(stage2) - 1
    assert report["timings"][0]["block_size"] is None  # the default was timed
    assert all(c[3] == 100 * 20_000 for c in calls)  # probes run a tenth of the histories
    again, report2 = T.tune(engine, source, np.full(100, 200_000), 10, 1, cache=cache,
                            timer=_fake_timer([]), sm_count=148, device_name="B200")
    assert report2["cached"] and again == tuned
    other = T.cache_key("B200", (64, 64, 64), source, 2e7, True)
    assert other != report["key"]  # another grid
    assert other == T.cache_key("B200", (64, 64, 64), source, 3e7, True)  # the same decade


def test_tuner_refuses_a_shape_that_changes_the_dij(tmp_path):
    engine = FakeEngine(grid=SimpleNamespace(shape=(8, 8, 8)))

    def timer(e, source, counts, n_batches, seed):
        return 1.0, _dij(seed=1 if e.block_size == 192 else 0)

    with pytest.raises(RuntimeError, match="scheduling-inert"):
        T.tune(engine, SimpleNamespace(n_beamlets=1), [100], 10, 1, cache=None, timer=timer,
               sm_count=148, device_name="B200")
