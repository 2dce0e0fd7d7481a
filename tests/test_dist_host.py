"""The multi-GPU host path on CPU: two gloo ranks (world size 2).

Each rank takes its column range of a Dij from ``column_shards`` (no data-path
collective: beamlets keep their global history numbers), the shards meet on
rank 0 with one gather and ``merge_shards`` rebuilds the whole Dij exactly; the
bench's timing reductions (max over ranks, sums) and its weak-scaling
throughput run over the same process group.  The device work itself is
replaced by a deterministic synthetic CSC per column, which is what a rank's
``run_dij_shard`` returns in kind.
"""

from __future__ import annotations

import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest

from pyradmc_b200.engine import column_shards, merge_shards


def _full_dij(counts, n_vox=50, seed=3):
    """A synthetic Dij whose column j depends only on j (as the engine's does on
    the column's global histories)."""
    cols = []
    for j, c in enumerate(counts):
        rng = np.random.default_rng(seed + j)
        idx = np.sort(rng.choice(n_vox, size=1 + j % 7, replace=False)).astype(np.int64)
        cols.append((idx, rng.random(idx.size) * c, rng.random(idx.size)))
    return cols


def _as_result(cols, lo, hi, counts):
    part = cols[lo:hi]
    indptr = np.zeros(len(part) + 1, dtype=np.int64)
    np.cumsum([p[0].size for p in part], out=indptr[1:])
    cat = lambda k, dt: (np.concatenate([p[k] for p in part]) if part  # noqa: E731
                         else np.zeros(0, dtype=dt))
    return SimpleNamespace(grid_shape=(5, 5, 2), n_beamlets=hi - lo,
                           n_histories_per_beamlet=int(max(counts[lo:hi], default=0)),
                           n_batches=10, truncation=0.0, indptr=indptr,
                           indices=cat(0, np.int64), dose=cat(1, float), sigma=cat(2, float),
                           energy_emitted=float(sum(counts[lo:hi])), energy_deposited=1.0 * (hi - lo),
                           energy_escaped=0.5 * (hi - lo), energy_unscored=0.0, correlated=True,
                           scoring_mode="dose_to_medium", provenance=None)


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench

        counts = [10_000, 200_000, 30_000, 1_000_000, 50_000, 70_000, 10_000]
        spans = column_shards(counts, world)
        lo, hi = spans[rank]
        cols = _full_dij(counts)
        mine = (_as_result(cols, lo, hi, counts), (lo, hi))
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        bench.barrier(world)
        mx = bench.all_max(world, [float(rank + 1), 10.0 - rank])
        sm = bench.all_sum(world, [float(rank + 1)])
        if rank == 0:
            merged = merge_shards(gathered)
            whole = _as_result(cols, 0, len(counts), counts)
            ok = (np.array_equal(merged.indptr, whole.indptr)
                  and np.array_equal(merged.indices, whole.indices)
                  and np.array_equal(merged.dose, whole.dose)
                  and np.array_equal(merged.sigma, whole.sigma)
                  and merged.n_beamlets == len(counts)
                  and merged.energy_emitted == float(sum(counts))
                  and mx == [float(world), 10.0] and sm == [float(world * (world + 1) // 2)]
                  and bench.job_value(world * 1000, 4, 2000.0) == world * 2000.0)
            with open(os.path.join(out_dir, "ok"), "w") as f:
                f.write("1" if ok else f"0 {mx} {sm}")
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_shard_gather_and_merge_the_dij(tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    assert (tmp_path / "ok").read_text() == "1"


def test_column_shards_tile_the_columns_with_balanced_histories():
    rng = np.random.default_rng(0)
    counts = (10 ** rng.uniform(4, 6, 100)).astype(np.int64)
    for world in (1, 2, 3, 4, 8):
        spans = column_shards(counts, world)
        assert spans[0][0] == 0 and spans[-1][1] == 100 and len(spans) == world
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        loads = [counts[a:b].sum() for a, b in spans]
        assert max(loads) <= counts.sum() / world + counts.max()
    assert column_shards([5, 5], 4)[1] == (1, 1)  # more ranks than columns: empty shards
    with pytest.raises(ValueError):
        merge_shards([(_as_result(_full_dij([1, 2, 3]), 0, 1, [1, 2, 3]), (0, 1)),
                      (_as_result(_full_dij([1, 2, 3]), 2, 3, [1, 2, 3]), (2, 3))])
