"""Autotuner for the persistent transport launch: block size, resident blocks
per SM, the primaries admitted per transport round, how long a particle may
outlive its round's input before it is parked for the next round, and whether
the table rows are staged in shared memory.

The reference sizes its launches with fixed heuristics
(``pyradmc/backends/warp/engine.py:175-255`` for the history chunk,
``kernels.py:1032-1091`` for the compaction chunk); here the shape of the
persistent photon/electron kernels is chosen by measurement.  Every candidate
runs a short probe of the caller's own workload (the same beamlets at a
fraction of the histories) and the fastest wins.  Because histories draw from
streams keyed on ``(seed, history)`` and deposits are integers, the launch shape
cannot change the Dij by one bit; the tuner checks exactly that on every probe
and raises if two candidates disagree.

Results are cached per (device name, grid shape, source kind, beamlet count,
history decade, electron transport) in a JSON file, so a workload is tuned
once per machine.
"""

from __future__ import annotations

import dataclasses
import hashlib
import json
import math
import os
import threading
from dataclasses import dataclass
from pathlib import Path

import numpy as np

DEFAULT_CACHE = Path(os.environ.get("PYRADMC_B200_TUNE_CACHE",
                                    Path.home() / ".cache" / "pyradmc_b200" / "autotune.json"))
BLOCK_SIZES = (128, 192, 256)
BLOCKS_PER_SM = (None, 2, 3, 4)    # None: as many as the occupancy calculator allows;
                                   # 3 and 4 also pick the kernels' register budget
CHUNK_PER_THREAD = (8, 16, 32)     # admitted primaries per resident transport thread
ASSUMED_BLOCKS_PER_SM = 3          # resident estimate for sizing the chunk candidates
TAIL_STEPS = (None, 24, 256, 2048, -1)  # None: the library default; -1: never park
SMEM_TABLES = (None, False)        # None: the library's choice (staged when they fit)

_lock = threading.Lock()


@dataclass(frozen=True)
class LaunchShape:
    """None fields leave the engine's default (256 threads, occupancy-limited
    residency, 16 primaries per resident thread, the library's parking
    threshold and table placement)."""

    block_size: int | None
    blocks_per_sm: int | None
    chunk_size: int | None
    tail_steps: int | None = None
    smem_tables: bool | None = None

    def as_dict(self) -> dict:
        return dataclasses.asdict(self)


def candidates(sm_count: int) -> list[LaunchShape]:
    """The first search stage on a device with `sm_count` SMs (the launch
    geometry); the engine's default shape comes first, so tuning never picks a
    slower one."""
    out = [LaunchShape(None, None, None)]
    for bs in BLOCK_SIZES:
        for per_sm in BLOCKS_PER_SM:
            for m in CHUNK_PER_THREAD:
                resident = sm_count * (per_sm or ASSUMED_BLOCKS_PER_SM) * bs
                out.append(LaunchShape(bs, per_sm, int(m * resident)))
    return out


def refinements(best: LaunchShape) -> list[LaunchShape]:
    """The second stage: the parking threshold and the table placement on top
    of the best geometry (the best itself first)."""
    out = [best]
    for tail in TAIL_STEPS:
        for smem in SMEM_TABLES:
            shape = dataclasses.replace(best, tail_steps=tail, smem_tables=smem)
            if shape not in out:
                out.append(shape)
    return out


def cache_key(device_name: str, grid_shape, source, n_histories: int, transport_electrons: bool) -> str:
    decade = int(math.floor(math.log10(max(int(n_histories), 1))))
    n_beamlets = int(getattr(source, "n_beamlets", 1))
    return "|".join([device_name, "x".join(str(int(v)) for v in grid_shape), type(source).__name__,
                     str(n_beamlets), f"1e{decade}", "e" if transport_electrons else "kerma"])


def load_cache(path: Path = DEFAULT_CACHE) -> dict:
    try:
        return json.loads(Path(path).read_text())
    except (OSError, ValueError):
        return {}


def store_cache(key: str, shape: LaunchShape, path: Path = DEFAULT_CACHE) -> None:
    path = Path(path)
    with _lock:
        data = load_cache(path)
        data[key] = shape.as_dict()
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        tmp.replace(path)


def probe_counts(counts, fraction: float, n_batches: int) -> np.ndarray:
    """Per-beamlet probe counts: `fraction` of each, a positive multiple of n_batches."""
    c = np.asarray(counts, dtype=np.int64)
    return np.maximum(n_batches, np.round(c * fraction / n_batches).astype(np.int64) * n_batches)


def digest(dij) -> str:
    h = hashlib.sha256()
    for a in (dij.indptr, dij.indices, dij.dose, dij.sigma):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def tune(engine, source, counts, n_batches: int, seed: int, *, fraction: float = 0.1,
         repeats: int = 2, shapes: list[LaunchShape] | None = None, cache: Path | None = DEFAULT_CACHE,
         timer=None, transport_electrons: bool = True, sm_count: int | None = None,
         device_name: str | None = None):
    """(tuned engine, report): the engine with the fastest launch shape for a
    Dij of `counts` histories per beamlet on `source`.

    ``timer(engine, source, counts, n_batches, seed) -> (seconds, dij)`` times
    one probe (default: the transport and reduction time the engine's device
    events measured).  A cached shape is used without probing.  `sm_count` and
    `device_name` default to the engine's device.
    """
    if sm_count is None or device_name is None:
        import torch

        props = torch.cuda.get_device_properties(torch.device(engine.device))
        sm_count = sm_count or props.multi_processor_count
        device_name = device_name or props.name
    sms = int(sm_count)
    key = cache_key(device_name, engine.grid.shape, source, int(np.sum(counts)), transport_electrons)
    if cache is not None:
        hit = load_cache(cache).get(key)
        if hit is not None:
            shape = LaunchShape(**hit)
            return dataclasses.replace(engine, **shape.as_dict()), {"key": key, "cached": True,
                                                                    "shape": shape.as_dict()}
    timer = timer or _transport_seconds
    probe = probe_counts(counts, fraction, n_batches)
    report = {"key": key, "cached": False, "probe_histories": int(probe.sum()), "timings": []}
    best, best_t, reference = None, math.inf, None
    timed: dict = {}
    stages = [shapes] if shapes else [candidates(sms), None]
    for stage in stages:
        for shape in (stage if stage is not None else refinements(best)):
            if shape in timed:
                continue
            trial = dataclasses.replace(engine, **shape.as_dict())
            times = []
            for _ in range(repeats):
                seconds, dij = timer(trial, source, probe, n_batches, seed)
                times.append(seconds)
                d = digest(dij)
                if reference is None:
                    reference = d
                elif d != reference:
                    raise RuntimeError(f"launch shape {shape} changed the Dij: the transport is "
                                       "not scheduling-inert")
            t = float(np.median(times))
            timed[shape] = t
            report["timings"].append({**shape.as_dict(), "seconds": t})
            if t < best_t:
                best, best_t = shape, t
            trial.drop_uploads()
    report["shape"] = best.as_dict()
    if cache is not None:
        store_cache(key, best, cache)
    return dataclasses.replace(engine, **best.as_dict()), report


def _transport_seconds(engine, source, counts, n_batches, seed):
    dij = engine.run_dij(source, counts, n_batches, seed)
    c = engine.last_counters()
    return (c["transport_ms"] + c["reduce_ms"]) / 1e3, dij
