"""Benchmark: histories/s of a 100-beamlet 6 MV Dij on a 128^3 CT-like phantom.

Workload (the batched-Dij configuration the headline metric is quoted on):
a 128^3 phantom at 2.5 mm (water plus 6-12 seeded random ellipsoids of density
U(0.2, 1.9)), a 10x10 lattice of 5x5 mm beamlets of the Ali-Rogers Varian 6 MV
spectrum at SAD 100 cm, per-beamlet history counts log-uniform in 1e4-1e6
(seeded; ~2e7 histories in total), 10 batches, full electron transport with
Goudsmit-Saunderson multiple scattering, truncation 1e-3.  One step is one whole
Dij: transport, fold, finalize, truncation and CSC assembly.

``python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference]``
prints one JSON line.  ``value`` is histories/s over the device-resident step
(``run_dij_device``: transport to CSC, the CSC left in HBM; CUDA events on the
stream the engine runs on, max over ranks); ``e2e`` is the
same metric through ``B200Engine.run_dij`` from host data, with the grid, table
and GS uploads and the CSC readback inside the timed region.  Under torchrun the
N ranks compute one Dij of N x 100 columns (the benchmark fan N times over, each
copy with its own history keys), each rank its history-balanced share of the
columns (``column_shards`` / ``run_dij_shard``): weak scaling through the
product's own sharding, no data-path collective; the books and timings meet in
all-reduces outside the timed region.

``--impl reference`` times the CPU oracle (the C restatement of the reference's
transport, all host threads) on bounded samples of the same workload.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "histories/s and s per 100-beamlet Dij at 2% sigma: plain MC vs MC+denoiser"
N_BATCHES = 10
SEED = 20260726


WORKLOAD = "dij100"


def workload(rank: int = 0):
    """The benchmark Dij; ``--workload dij10`` is the reduced case the ncu
    captures use (the same phantom, one row of 10 beamlets, 1e5 histories each)."""
    from pyradmc_b200 import phantoms
    from pyradmc_b200.model import AnalyticWaterTables

    grid = phantoms.ellipsoid_phantom(seed=SEED)
    if WORKLOAD == "dij10":
        source = phantoms.beamlet_fan(grid, n_x=10, n_y=1)
        counts = np.full(source.n_beamlets, 100_000, dtype=np.int64)
    else:
        source = phantoms.beamlet_fan(grid)
        counts = phantoms.log_uniform_counts(source.n_beamlets, n_batches=N_BATCHES, seed=SEED)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, source, counts


def config_dict(counts, l2_note):
    return {
        "workload": ("dij_128cube_100beamlets_6MV" if WORKLOAD == "dij100"
                     else "dij_128cube_10beamlets_6MV_profile"),
        "phantom": "128^3 at 2.5 mm, water + seeded ellipsoids rho U(0.2,1.9)",
        "beamlets": int(len(counts)),
        "beamlet_mm": 5,
        "spectrum": "Ali-Rogers varian-6mv, e_min 0.1 MeV",
        "histories_per_dij": int(np.sum(counts)),
        "histories_per_beamlet": "log-uniform 1e4-1e6",
        "n_batches": N_BATCHES,
        "msc": "gs",
        "truncation": 1e-3,
        "l2": l2_note,
    }


# ---- clocks -----------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples during the timed region (every 50 ms); entering waits
    (at most 5 s) for the first sample, so sampling is live when timing starts."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int) -> None:
        self.index = index
        self.proc = None
        self.lines: list[str] = []
        self._t = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except OSError:
            self.proc = None
            return self
        t0 = time.monotonic()
        while not self.lines and self.proc.poll() is None and time.monotonic() - t0 < 5.0:
            time.sleep(0.01)
        self.lines.clear()  # samples from before the timed region
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self._t is not None:
            self._t.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9], strict=True):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---- distributed plumbing ---------------------------------------------------------------
def dist_setup(n_gpus: int):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device(f"cuda:{local}"))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _reduce(world, values, op):
    if world == 1:
        return list(values)
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op))
    return t.tolist()


def all_max(world, values):
    return _reduce(world, values, "MAX")


def all_sum(world, values):
    return _reduce(world, values, "SUM")


def job_value(histories_all_ranks: int, steps: int, max_total_ms: float) -> float:
    """Whole-job histories/s: the histories every rank ran per step, summed
    over ranks, over `steps` steps that take as long as the slowest rank."""
    return histories_all_ranks * steps / (max_total_ms / 1e3)


# ---- the CPU baseline -----------------------------------------------------------------
def _oracle_sample(grid, xs, source, counts, per_col, seed):
    """Time the C oracle on `per_col` histories of every beamlet (one batch)."""
    import oracle

    tab = xs.build_tables(0.2, 0.05, source.max_energy * (1 + 1e-6))
    gs = xs.gs_grid_for(tab, [0])
    t0 = time.perf_counter()
    oracle.run(grid, tab, gs, source, counts=list(counts), n_batches=1, seed=seed, forward=False,
               n_threads=oracle.max_threads(), max_histories=per_col)
    return time.perf_counter() - t0, int(np.sum(np.minimum(counts, per_col)))


def calibrate_sample(grid, xs, source, counts, target_seconds):
    """Grow the per-beamlet sample until one run takes ~target_seconds (or covers
    the whole workload), so the oracle's fixed costs do not dominate the rate."""
    per_col = 100
    elapsed, done = _oracle_sample(grid, xs, source, counts, per_col, SEED)
    while elapsed < 0.7 * target_seconds and per_col < int(np.max(counts)):
        per_col = int(per_col * min(8.0, max(1.5, target_seconds / max(elapsed, 1e-3))))
        elapsed, done = _oracle_sample(grid, xs, source, counts, per_col, SEED)
    return per_col, elapsed, done


def cpu_baseline(grid, xs, source, counts, target_seconds=15.0):
    """The C oracle on all host cores, on a bounded sample of the same Dij."""
    import oracle

    per_col, elapsed, done = calibrate_sample(grid, xs, source, counts, target_seconds)
    return {
        "value": done / elapsed,
        "unit": "histories/s",
        "cores": oracle.max_threads(),
        "kind": "port",
        "sample": f"{per_col} histories of each of the {len(counts)} beamlets ({done} histories, "
                  f"{elapsed:.1f} s), same phantom/spectrum/physics, one batch",
    }


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    grid, xs, source, counts = workload()
    import oracle

    threads = oracle.max_threads()
    # the first warm-up step sizes the per-step sample (~10 s of CPU work)
    per_col, _, _ = calibrate_sample(grid, xs, source, counts, 10.0)
    times, done = [], 0
    for step in range(max(0, args.warmup - 1) + args.steps):
        elapsed, done = _oracle_sample(grid, xs, source, counts, per_col, SEED + step)
        if step >= max(0, args.warmup - 1):
            times.append(elapsed)
    total = sum(times)
    value = done * len(times) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "histories/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(counts, "n/a (CPU)"),
        "cpu_baseline": {"value": value, "unit": "histories/s", "cores": threads, "kind": "port",
                         "sample": f"{per_col} histories of each beamlet per step ({done})"},
        "e2e": {"value": value, "unit": "histories/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ---- the B200 arm ---------------------------------------------------------------------
def algorithmic_bytes(c: dict) -> float:
    """Transport bytes by event: 13 B per Woodcock flight (voxel 5 + majorant 8),
    +32 B per real interaction (4 channel lookups), 77 B per electron substep
    (voxel 5 + 7 lookups x 8 + GS 16), 16 B per int64 deposit, 48 B per queue
    push and 48 B per pop."""
    pops = c["queue_pushes"]
    return (13.0 * c["photon_flights"] + 32.0 * c["photon_interactions"]
            + 77.0 * c["electron_substeps"] + 16.0 * c["deposits"]
            + 48.0 * c["queue_pushes"] + 48.0 * pops)


DENOISER_WEIGHTS = ROOT / "pyradmc_b200" / "data" / "denoiser_unet.npz"
# the network trained on coplanar gantry beams (oblique beamlets, 3 mm voxels)
PLAN_DENOISER_WEIGHTS = ROOT / "pyradmc_b200" / "data" / "denoiser_unet_coplanar.npz"
REF_HISTORIES = 8_000_000     # per beamlet: the high-statistics judge of the denoiser's error
LADDER = (1 / 4, 1 / 3, 0.4, 1 / 2, 2 / 3, 1.0, 1.5, 2.0, 3.0, 4.0, 6.0, 8.0)  # scales tried


def denoiser_leg(args, engine, source, counts, stream, device, plain_s_per_dij):
    """s per Dij at 2 % for MC + denoiser on the benchmark Dij, at two error
    thresholds: the metric's own (voxels >= 50 % of the column maximum, the
    per-beamlet sigma of examples/noise_bias_study.py:130-144) and the stricter
    >= 10 % region that takes in the penumbra.

    Untimed: a REF_HISTORIES-per-beamlet reference, then the history scales of
    LADDER (ascending; times the benchmark's per-beamlet counts) until the
    denoised columns reach a sigma-equivalent error <= 2 % on both regions;
    every rung reports error and signed bias at 50, 10 and 1 % of the maximum
    for both methods.  Plain Monte Carlo at 2 % on a region is its measured s
    per Dij at the benchmark counts times (its error there / 2 %)^2 (1/sqrt(N)).
    Every rung is denoised with windows DEN_LATERALS voxels across; for each
    window a region's candidate is the lowest rung where it reaches 2 %.
    Timed (CUDA events on the engine's stream): ``run_dij_denoised`` at each
    candidate's scale and window, from transport to the CSC in HBM
    (device-resident, like ``value``); the fastest candidate is the region's
    time."""
    import torch

    from pyradmc_b200 import _lib
    from pyradmc_b200 import denoise_dij as D
    from pyradmc_b200.denoiser import UNet3D, forward_flops_per_voxel, kpad_for

    if not DENOISER_WEIGHTS.exists():
        return {"unavailable": f"no trained weights at {DENOISER_WEIGHTS.relative_to(ROOT)}"}
    torch.cuda.empty_cache()  # the engine allocates outside torch's cache
    net = UNet3D.load(DENOISER_WEIGHTS, device=device)
    shape = tuple(engine.grid.shape)
    windows = {lat: D.inference_window(shape, lat) for lat in DEN_LATERALS}
    window = windows[DEN_LATERALS[0]]
    rho = torch.from_numpy(np.ascontiguousarray(engine.grid.density, dtype=np.float32).ravel()).to(device)
    ref = engine.run_dij_device(source, REF_HISTORIES, N_BATCHES, SEED + 977, truncation=0.0)
    ref_dose, _, ref_sigma = D.dense_columns(ref, device, with_sigma=True)
    # plain Monte Carlo's error at the benchmark counts, on each region
    view = engine.run_dij_device(source, counts, N_BATCHES, SEED + 31, truncation=0.0)
    dose, _, _ = D.dense_columns(view, device)
    plain_at_counts = D.error_report(dose, ref_dose, ref_sigma)
    del dose
    ladder, candidates = [], {}
    for g in LADDER:
        c = np.maximum(N_BATCHES, np.round(counts * g / N_BATCHES).astype(np.int64) * N_BATCHES)
        view = engine.run_dij_device(source, c, N_BATCHES, SEED + 31, truncation=0.0)
        dose, colmax, sg = D.dense_columns(view, device, with_sigma=True)
        by_window = {}
        for lat, win in windows.items():
            den = D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg, window=win,
                                  directions=D.beam_directions(source), spacing=engine.grid.spacing)
            by_window[lat] = D.error_report(den, ref_dose, ref_sigma)
            del den
        rung = {"scale": g, "histories": int(c.sum()),
                "denoised": by_window[DEN_LATERALS[0]],
                "denoised_by_lateral": {str(k): v for k, v in by_window.items()},
                "plain": D.error_report(dose, ref_dose, ref_sigma)}
        ladder.append(rung)
        del dose, sg
        for t in ("0.5", "0.1"):
            # each window's lowest rung that reaches 2 % (timed below; the faster wins)
            for lat in DEN_LATERALS:
                if (t, lat) not in candidates and by_window[lat][t]["sigma_eq"] <= 0.02:
                    candidates[(t, lat)] = (g, c)
        if len(candidates) == 2 * len(DEN_LATERALS):
            break
    del ref_dose, ref_sigma
    if not any(t == "0.5" for t, _ in candidates):
        return {"reached_2pct": False, "ladder": ladder,
                "reference_histories_per_beamlet": REF_HISTORIES}

    def timed(c, lateral, **extra):
        kw = dict(n_histories_per_beamlet=c, n_batches=N_BATCHES, seed=SEED, lateral=lateral, **extra)
        for _ in range(max(1, args.warmup)):
            D.run_dij_denoised(engine, net, source, truncation=1e-3, to_host=False, **kw)
        times, launches0 = [], net.launches
        torch.cuda.synchronize()
        dij = None
        for _ in range(args.steps):
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            dij = D.run_dij_denoised(engine, net, source, truncation=1e-3, to_host=False, **kw)
            end.record(stream)
            end.synchronize()
            times.append(start.elapsed_time(end) / 1e3)
        return float(np.median(times)), (net.launches - launches0) / args.steps, dij

    regions, chosen = {}, {}
    for t in ("0.5", "0.1"):
        # every window's candidate, in one group and in DEN_GROUP-column groups
        # whose denoising overlaps the next group's transport (the same Dij bit
        # for bit); the fastest is the method's time
        best, cand_s = None, {}
        for lat in DEN_LATERALS:
            if (t, lat) not in candidates:
                continue
            g, c = candidates[(t, lat)]
            s_seq, unet_launches, dij = timed(c, lat)
            s_pipe, _, _ = timed(c, lat, group_columns=DEN_GROUP, overlap=True)
            cand_s[lat] = min(s_seq, s_pipe)
            if best is None or min(s_seq, s_pipe) < best[0]:
                best = (min(s_seq, s_pipe), g, c, lat, s_seq, s_pipe, unet_launches, dij)
        if best is None:
            continue
        s_den, g, c, lat, s_seq, s_pipe, unet_launches, dij = best
        chosen[t] = (g, c, lat)
        plain_err = plain_at_counts[t]["sigma_eq"]
        plain_s = plain_s_per_dij * (plain_err / 0.02) ** 2
        rung = next(r for r in ladder if r["scale"] == g)
        regions[t] = {"history_scale": g, "histories_per_dij": int(c.sum()),
                      "s_per_dij_at_2pct": s_den, "plain_sigma_eq_at_benchmark_counts": plain_err,
                      "plain_s_per_dij_at_2pct": plain_s, "speedup_vs_plain": plain_s / s_den,
                      "lateral": lat, "denoised": rung["denoised_by_lateral"][str(lat)],
                      "plain_same_histories": rung["plain"],
                      "unet_launches_per_dij": unet_launches, "nnz": int(dij.indptr[-1]),
                      "s_one_group": s_seq, "s_pipelined": s_pipe,
                      "pipelined_group_columns": DEN_GROUP,
                      "candidates": {str(w): {"history_scale": candidates[(t, w)][0], "s_per_dij": cand_s[w]}
                                     for w in cand_s}}
    head = regions["0.5"]
    g, c, lat = chosen["0.5"]
    stages: dict = {}
    D.run_dij_denoised(engine, net, source, c, N_BATCHES, SEED, truncation=1e-3, to_host=False,
                       lateral=lat, timings=stages)

    # the dominant convolution (decoder level 0, 48 -> 16 channels, default path)
    lib = _lib.load()
    b, (wx, wy, wz) = 16, window
    x = torch.randn((b, wx, wy, wz, 48), device=device).to(torch.bfloat16)
    wt = (0.05 * torch.randn((16, kpad_for(48)), device=device)).to(torch.bfloat16)
    y = torch.empty((b, wx, wy, wz, 16), device=device, dtype=torch.bfloat16)
    conv = lambda: lib.pmd_conv3d(x.data_ptr(), wt.data_ptr(), None, y.data_ptr(), b, wx, wy, wz,  # noqa: E731
                                  48, 16, kpad_for(48), 1, stream.cuda_stream)
    for _ in range(3):
        conv()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        conv()
    e1.record(stream)
    e1.synchronize()
    conv_s = e0.elapsed_time(e1) / 10 / 1e3
    conv_tflops = 2.0 * b * wx * wy * wz * 27 * 48 * 16 / conv_s / 1e12
    unet_vox = len(counts) * int(np.prod(windows[lat]))  # the timed method's windows
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(peaks_path.read_text()) if peaks_path.exists() else {}
    bf16_peak = float(peaks.get("bf16_tflops", 1590.0))
    return {
        "reached_2pct": True,
        "s_per_dij_at_2pct": head["s_per_dij_at_2pct"],
        "plain_s_per_dij_at_2pct": head["plain_s_per_dij_at_2pct"],
        "speedup_vs_plain": head["speedup_vs_plain"],
        "history_scale": head["history_scale"],
        "histories_per_dij": head["histories_per_dij"],
        "threshold": "metric: voxels >= 50 % of the column maximum",
        "regions": regions,
        "plain_at_benchmark_counts": plain_at_counts,
        "plain_2pct": "extrapolated from the measured error at the benchmark counts (1/sqrt(N))",
        "sigma": "per-entry sigma of the denoised Dij is the input Monte Carlo sigma",
        "reference_histories_per_beamlet": REF_HISTORIES,
        "ladder": ladder,
        "window": list(windows[lat]),
        "windows_tried": {str(k): list(v) for k, v in windows.items()},
        "stage_ms": stages,
        "unet_forward_flops_per_dij": forward_flops_per_voxel() * unet_vox,
        "roofline": {"bound": "tensor", "kernel": "conv3d_ws_kernel (decoder level 0, 48->16)",
                     "achieved": conv_tflops, "peak": bf16_peak, "unit": "TFLOP/s",
                     "frac": conv_tflops / bf16_peak,
                     "peak_source": "measured" if "bf16_tflops" in peaks else "fallback",
                     "shape_cap": "M 128 x N 16 x K 16 MMAs read 4.5 KB of shared memory per "
                                  "65,536 FLOP: ~0.25 of the bf16 peak at most",
                     "source": "profiles/conv3d_ws_dec0a_ncu.md"},
    }


# ---- the full-plan workload ----------------------------------------------------------
PLAN_SHAPE = (256, 256, 128)
PLAN_SPACING = 0.3
PLAN_HELD_OUT = 50
PLAN_REF_HISTORIES = 8_000_000  # per held-out beamlet


def plan_workload():
    """A 256 x 256 x 128 phantom at 3 mm (water plus seeded ellipsoids of
    density U(0.2, 1.9), semi-axes scaled with the box from the 128^3 case's
    1-4 cm), 7 coplanar equi-spaced beams x 20 x 20 beamlets of 5 mm of the
    6 MV spectrum at SAD 100 cm = 2,800 columns, and 50 held-out columns
    spread evenly over the plan."""
    from pyradmc_b200 import model, phantoms
    from pyradmc_b200.model import AnalyticWaterTables

    scale = PLAN_SHAPE[0] * PLAN_SPACING / (128 * 0.25)
    grid = phantoms.ellipsoid_phantom(shape=PLAN_SHAPE, spacing=(PLAN_SPACING,) * 3, seed=SEED,
                                      semi_axis_range=(1.0 * scale, 4.0 * scale))
    plan, angles = phantoms.coplanar_plan(grid)
    held = np.linspace(0, plan.n_beamlets - 1, PLAN_HELD_OUT).round().astype(int)
    parts = []
    for j in held:
        k, i = plan.part_of(int(j))
        beam = plan.sources[k]
        parts.append(model.SpectralBeamletSource(beam.spectrum, beam.focal_point, [beam.centers[i]],
                                                 beam.width_u, beam.width_v, beam.u_axis, beam.v_axis))
    held_source = model.ConcatenatedBeamletSource(parts)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, plan, angles, held, held_source


def plan_leg(args, device, stream):
    """s per plan at 2 % sigma-equivalent error, plain Monte Carlo.

    Untimed: a PLAN_REF_HISTORIES-per-beamlet reference of the 50 held-out
    columns (independent streams), then a pilot at 1e5 histories per beamlet
    that sets the count N at which the held-out columns reach 2 % (1/sqrt(N)).
    Timed (CUDA events, device-resident like ``value``): the whole 2,800-column
    Dij at N, transport to CSC in HBM through grouped dense maps.  The held-out
    columns at N (bit-identical to the plan's own: correlated keys) confirm the
    error reached."""
    import torch

    from pyradmc_b200 import B200Engine
    from pyradmc_b200 import denoise_dij as D

    grid, xs, plan, angles, held, held_source = plan_workload()
    engine = B200Engine(grid, xs, device=device)
    engine.use_stream(stream.cuda_stream)
    ref = engine.run_dij_device(held_source, PLAN_REF_HISTORIES, N_BATCHES, SEED + 977, truncation=0.0)
    ref_dose, _, ref_sigma = D.dense_columns(ref, device, with_sigma=True)

    def held_error(n_per):
        view = engine.run_dij_device(held_source, n_per, N_BATCHES, SEED, truncation=0.0)
        dose, _, _ = D.dense_columns(view, device)
        err = D.sigma_equivalent_error(dose, ref_dose, ref_sigma)
        del dose
        return float(np.nanmean(err))

    pilot_n = 100_000
    pilot = held_error(pilot_n)
    n_2pct = int(np.ceil(pilot_n * (pilot / 0.02) ** 2 / N_BATCHES)) * N_BATCHES
    engine.run_dij_device(plan, n_2pct, N_BATCHES, SEED, truncation=1e-3)  # warm-up: same workload
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    view = engine.run_dij_device(plan, n_2pct, N_BATCHES, SEED, truncation=1e-3)
    e1.record(stream)
    e1.synchronize()
    seconds = e0.elapsed_time(e1) / 1e3
    c = engine.last_counters()
    nnz = int(view.nnz)
    reached = held_error(n_2pct)
    den = None
    if not args.no_denoiser:
        del view
        engine.release_device_memory()  # the plain plan's maps and CSC: room for dense columns
        torch.cuda.empty_cache()
        den = plan_denoiser(engine, plan, held_source, ref_dose, ref_sigma, n_2pct, seconds, device,
                            stream)
    del ref_dose, ref_sigma
    torch.cuda.empty_cache()
    return {
        "workload": "plan_256x256x128_3mm_7beams_2800beamlets_6MV",
        "denoiser": den,
        "beams_deg": [round(a, 2) for a in angles],
        "columns": int(plan.n_beamlets),
        "held_out_columns": int(len(held)),
        "reference_histories_per_beamlet": PLAN_REF_HISTORIES,
        "pilot_histories_per_beamlet": pilot_n,
        "pilot_sigma_eq": pilot,
        "plain": {"histories_per_beamlet": n_2pct, "histories": int(n_2pct * plan.n_beamlets),
                  "s_per_plan": seconds, "histories_per_s": n_2pct * plan.n_beamlets / seconds,
                  "sigma_eq_held_out": reached, "nnz": nnz,
                  "transport_ms": c["transport_ms"], "reduce_ms": c["reduce_ms"],
                  "measured": "timed at the 2 % count (not extrapolated)"},
    }


# ---- parity of the benchmark's phantom family ---------------------------------------
def batched_chi2(a, sa, n_a, b, sb, n_b):
    """chi2 over voxels of two batch means with batch-estimated sigmas, and its
    null (each voxel's z^2 is F(1, nu), nu by Welch-Satterthwaite: E = nu/(nu-2),
    Var = 2 nu^2 (nu-1) / ((nu-2)^2 (nu-4))); the one-sided normal p-value."""
    from math import erfc, sqrt

    va, vb = sa**2, sb**2
    nu = (va + vb) ** 2 / (va**2 / (n_a - 1) + vb**2 / (n_b - 1))
    chi2 = float(np.sum((a - b) ** 2 / (va + vb)))
    mean = float(np.sum(nu / (nu - 2.0)))
    var = float(np.sum(2.0 * nu**2 * (nu - 1.0) / ((nu - 2.0) ** 2 * (nu - 4.0))))
    z = (chi2 - mean) / sqrt(var)
    return chi2, mean, 0.5 * erfc(z / sqrt(2.0))


def parity_block(device):
    """The benchmark Dij's phantom family at reduced size against pyRadMC's
    ReferenceEngine (the committed fixtures tests/golden/ref_ct_beamlets_*.npz,
    made by tests/golden/make_golden.py): a 40^3 CT-like phantom at 2.5 mm, a
    2x2 fan of 5 mm 6 MV beamlets, uneven per-column counts; batched chi-squared
    per column on the voxels >= 10 % and >= 1 % of the column maximum.  Also
    quotes the test session's chi-squared report when it was written on this
    host ($PMC_PARITY_REPORT or .parity/chi2.json)."""
    from pyradmc_b200 import B200Engine, phantoms
    from pyradmc_b200.model import AnalyticWaterTables

    golden = ROOT / "tests" / "golden"
    grid = phantoms.ellipsoid_phantom(shape=(40, 40, 40), spacing=(0.25, 0.25, 0.25), seed=20260805)
    src = phantoms.beamlet_fan(grid, n_x=2, n_y=2, pitch=0.5, width=0.5, sad=100.0)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    counts = [40_000, 120_000, 40_000, 120_000]
    dij = B200Engine(grid, xs, device=device).run_dij(
        src, n_histories_per_beamlet=[4 * c for c in counts], n_batches=10, seed=SEED + 1,
        truncation=0.0)
    records = []
    for j, c in enumerate(counts):
        with np.load(golden / f"ref_ct_beamlets_{c}.npz") as z:
            a, sa, n_a = z["dose"][j], z["dose_sigma"][j], int(z["n_batches"])
        b, sb = dij.column_dense(j).reshape(-1), dij.sigma_dense(j).reshape(-1)
        for fraction in (0.1, 0.01):
            m = (a > fraction * a.max()) & (sa > 0) & (sb > 0)
            chi2, mean, p = batched_chi2(a[m], sa[m], n_a, b[m], sb[m], dij.n_batches)
            records.append({"case": f"ct_beamlets column {j} ({c} histories, >= {fraction:g} of max)",
                            "chi2_per_dof": chi2 / m.sum(), "null_mean_per_dof": mean / m.sum(),
                            "p": p, "n_voxels": int(m.sum()), "passed": p > 0.01})
    out = {"reference": "pyRadMC ReferenceEngine fixtures (tests/golden/ref_ct_beamlets_*.npz)",
           "records": records, "passed": sum(r["passed"] for r in records),
           "total": len(records)}
    report = Path(os.environ.get("PMC_PARITY_REPORT", str(ROOT / ".parity" / "chi2.json")))
    if report.exists():
        tests = json.loads(report.read_text())
        tests = tests.get("records", tests) if isinstance(tests, dict) else tests
        out["test_session"] = {"file": str(report), "cases": len(tests),
                               "passed": sum(1 for r in tests if r.get("passed")),
                               "min_p": min((r["p"] for r in tests), default=None)}
    return out


def presolve_leg(device):
    """The treatment-head pre-solve (pyradmc_b200.presolve) on the case of
    tests/golden/presolve_case.py — a jaw pair, a three-pair MLC and an air
    column in front of a 6 MV-like fan: the reference fixture's totals
    (pyRadMC's host pre-solve, tests/golden/make_presolve_golden.py) against
    the GPU's at 1.2e5 primaries, and the throughput of presolve_head_device
    (host arrays in, phase space out, wall clock) at 4e6 primaries."""
    import time

    from pyradmc_b200 import presolve as PS
    from tests.golden import presolve_case as case

    g = np.load(ROOT / "tests" / "golden" / "presolve_golden.npz")
    names = [f for f in PS.CompiledHeadStack.__dataclass_fields__ if f not in ("materials", "densities", "_keep")]
    stack = PS.CompiledHeadStack(**{n: g[f"s1_{n}"] for n in names},
                                 materials=tuple(int(m) for m in g["s1_materials"]),
                                 densities=tuple(float(d) for d in g["s1_densities"]))
    mu = PS.HeadMuTables(g["mu_log_energy"], g["mu_log_total"], g["mu_log_compton"])
    kw = dict(exit_z=case.AIR_EXIT_Z, stack=stack, air=PS.AirColumn(**case.AIR), mode="first_compton",
              device=device, mu_tables=mu)
    ps = PS.presolve_head_device(case.FanSource(), n_histories=case.N, seed=case.SEED, **kw)
    c = ps.columns()
    w, e = c["weight"].astype(np.float64), c["energy"].astype(np.float64)
    host = g["air_totals"]
    parity = {"particles": [len(ps), int(host[0])], "weight": [float(w.sum()), float(host[1])],
              "weight_energy": [float((w * e).sum()), float(host[2])],
              "electrons": [int(np.count_nonzero(c["particle_type"] == 2)), int(host[4])]}
    n = 4_000_000
    cols = case.FanSource().sample_batch(case.SEED, 0, n)

    class Sampled:  # the same primaries every call: the timing excludes the NumPy sampler
        max_energy = case.FanSource.max_energy

        def sample_batch(self, seed, offset, m):
            return cols

    rate = {}
    for name, on_device in (("to_host", False), ("on_device", True)):
        PS.presolve_head_device(Sampled(), n_histories=n, seed=1, return_device_source=on_device, **kw)
        t0 = time.perf_counter()
        out = PS.presolve_head_device(Sampled(), n_histories=n, seed=2, return_device_source=on_device, **kw)
        rate[name] = {"seconds": time.perf_counter() - t0, "exit_particles": len(out)}
        rate[name]["primaries_per_s"] = n / rate[name]["seconds"]
        del out
    return {"case": "jaw pair + 3-pair MLC + air column, first Compton", "parity_vs_host": parity,
            "primaries": n, "exit_particles": rate["to_host"]["exit_particles"],
            "seconds": rate["to_host"]["seconds"], "primaries_per_s": rate["to_host"]["primaries_per_s"],
            "device_source": rate["on_device"],
            "reference_host_rate": "~1e5 rays/s with an MLC, one core (geometry/head.py:56-59)"}


DEN_GROUP = 25  # columns per group when MC and denoising overlap across groups
DEN_LATERALS = (64, 48)  # lateral window sizes tried (the network trains on 64); the faster at 2 % is the time
PLAN_WINDOW = (64, 64, 128)  # lateral x lateral x depth chunk of the plan's denoising windows
PLAN_GROUP = 100            # columns whose dense maps are on the device at once


def plan_denoiser(engine, plan, held_source, ref_dose, ref_sigma, n_plain, plain_seconds, device,
                  stream):
    """MC + denoiser on the plan.  Untimed: the held-out columns at 1/16 ..
    3/4 of the plain 2 % count, denoised along their beamlets (windows of
    PLAN_WINDOW oriented by each beam's direction, sheared along oblique
    beamlets), until the held-out error reaches 2 %; each rung also reports the
    history gain (plain MC histories for the denoised error / these).  Timed
    (CUDA events): ``run_dij_denoised`` of the whole plan at the 2 % count, or,
    where no rung reaches 2 %, at the lowest rung with its error;
    PLAN_GROUP columns at a time, CSC left in HBM."""
    import torch

    from pyradmc_b200 import denoise_dij as D
    from pyradmc_b200.denoiser import UNet3D

    weights = PLAN_DENOISER_WEIGHTS if PLAN_DENOISER_WEIGHTS.exists() else DENOISER_WEIGHTS
    net = UNet3D.load(weights, device=device)
    shape = tuple(engine.grid.shape)
    dirs = D.beam_directions(held_source)
    rho = torch.from_numpy(np.ascontiguousarray(engine.grid.density, dtype=np.float32).ravel()).to(device)
    ladder, chosen = [], None
    for frac in (1 / 16, 1 / 8, 1 / 4, 1 / 2, 3 / 4):
        n = max(N_BATCHES, int(round(n_plain * frac / N_BATCHES)) * N_BATCHES)
        view = engine.run_dij_device(held_source, n, N_BATCHES, SEED, truncation=0.0)
        dose, colmax, sg = D.dense_columns(view, device, with_sigma=True)
        den = D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg, window=PLAN_WINDOW,
                              directions=dirs, spacing=engine.grid.spacing)
        row = {"histories_per_beamlet": n, "fraction_of_plain": frac,
               "denoised": D.error_report(den, ref_dose, ref_sigma),
               "plain_same_histories": D.error_report(dose, ref_dose, ref_sigma)}
        # plain MC histories that reach the denoised error, over these (1/sqrt(N))
        row["history_gain"] = (row["plain_same_histories"]["0.5"]["sigma_eq"]
                               / row["denoised"]["0.5"]["sigma_eq"]) ** 2
        ladder.append(row)
        del dose, sg, den
        if row["denoised"]["0.5"]["sigma_eq"] <= 0.02:
            chosen = n
            break
    torch.cuda.empty_cache()
    out = {"weights": str(weights.relative_to(ROOT)), "window": list(PLAN_WINDOW),
           "group_columns": PLAN_GROUP, "ladder": ladder,
           "threshold": "metric: held-out voxels >= 50 % of the column maximum"}
    out["reached_2pct"] = chosen is not None
    timed_row = next(r for r in ladder if r["histories_per_beamlet"] == chosen) if chosen else ladder[0]
    if chosen is None:  # time the method where it gains most: the lowest count of the ladder
        chosen = timed_row["histories_per_beamlet"]
    stages: dict = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dij = D.run_dij_denoised(engine, net, plan, chosen, N_BATCHES, SEED, truncation=1e-3,
                             lateral=PLAN_WINDOW[0], depth=PLAN_WINDOW[2], to_host=False,
                             group_columns=PLAN_GROUP, overlap=True, timings=stages)
    e1.record(stream)
    e1.synchronize()
    seconds = e0.elapsed_time(e1) / 1e3
    out.update({"histories_per_beamlet": chosen, "histories": int(chosen * plan.n_beamlets),
                "s_per_plan": seconds, "sigma_eq_held_out": timed_row["denoised"]["0.5"]["sigma_eq"],
                "nnz": int(dij.indptr[-1]), "stage_ms": stages})
    if out["reached_2pct"]:
        out["speedup_vs_plain"] = plain_seconds / seconds
    del dij
    torch.cuda.empty_cache()
    return out


def conv_arm(args, local):
    """``--workload conv``: the denoiser's dominant convolution (decoder level 0,
    48 -> 16 channels, one inference chunk of 16 windows of 64 x 64 x 128) on
    both kernel paths; the case the tensor-memory kernel's ncu captures use."""
    import torch

    from pyradmc_b200 import _lib
    from pyradmc_b200.denoiser import kpad_for

    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    lib = _lib.load()
    b, d, h, w, cin, cout = 16, 64, 64, 128, 48, 16
    stream = torch.cuda.Stream(device=device)
    torch.cuda.set_stream(stream)
    gen = torch.Generator(device=device).manual_seed(SEED)
    x = torch.randn((b, d, h, w, cin), device=device, generator=gen).to(torch.bfloat16)
    wt = (0.05 * torch.randn((cout, kpad_for(cin)), device=device, generator=gen)).to(torch.bfloat16)
    y = torch.empty((b, d, h, w, cout), device=device, dtype=torch.bfloat16)
    flops = 2.0 * b * d * h * w * 27 * cin * cout
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(peaks_path.read_text()) if peaks_path.exists() else {}
    peak = float(peaks.get("bf16_tflops", 1590.0))
    out = {"workload": "conv3d 48->16, 16 x 64 x 64 x 128 voxels, bf16/fp32", "flops": flops}
    previous = lib.pmd_conv3d_impl(-1)
    for name, impl in (("warp_specialized", 4), ("tensor_memory_pipelined", 3), ("tensor_memory", 2),
                       ("mma_sync", 1)):
        lib.pmd_conv3d_impl(impl)
        for _ in range(args.warmup):
            assert lib.pmd_conv3d(x.data_ptr(), wt.data_ptr(), None, y.data_ptr(), b, d, h, w, cin,
                                  cout, kpad_for(cin), 1, stream.cuda_stream) == 0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            lib.pmd_conv3d(x.data_ptr(), wt.data_ptr(), None, y.data_ptr(), b, d, h, w, cin, cout,
                           kpad_for(cin), 1, stream.cuda_stream)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out[name] = {"ms": ms, "tflops": flops / ms / 1e9, "frac_of_measured_bf16": flops / ms / 1e9 / peak}
    lib.pmd_conv3d_impl(previous)
    del x, y

    # every layer of one inference chunk on each kernel path (-1: not covered)
    # with the default path's plan (pmd_conv3d_plan)
    import ctypes

    from pyradmc_b200.denoiser import layout

    level = {"enc0": 0, "enc1": 1, "enc2": 2, "mid_": 3, "dec2": 2, "dec1": 1, "dec0": 0}
    layers = {}
    for layer in layout()[0]:
        f = 2 ** level[layer.name[:4]]
        dims = (b, d // f, h // f, w // f)
        lx = torch.randn((*dims, layer.cin), device=device, generator=gen).to(torch.bfloat16)
        lw = (0.05 * torch.randn((layer.cout, layer.kpad), device=device, generator=gen)).to(torch.bfloat16)
        ly = torch.empty((*dims, layer.cout), device=device, dtype=torch.bfloat16)
        lflops = 2.0 * np.prod(dims) * 27 * layer.cin * layer.cout
        info = (ctypes.c_int * 8)()
        lib.pmd_conv3d_impl(previous)
        lib.pmd_conv3d_plan(*dims, layer.cin, layer.cout, info)
        row = {"plan": list(info)}
        for name, impl in (("default", 0), ("single_buffered", 2), ("mma_sync", 1)):
            lib.pmd_conv3d_impl(impl)
            call = lambda: lib.pmd_conv3d(lx.data_ptr(), lw.data_ptr(), None, ly.data_ptr(), *dims,
                                          layer.cin, layer.cout, layer.kpad, 1, stream.cuda_stream)
            if call() != 0:
                row[name] = -1
                continue
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                call()
            e1.record(stream)
            e1.synchronize()
            row[name] = round(e0.elapsed_time(e1) / args.steps, 4)
            row[name + "_tflops"] = round(lflops / row[name] / 1e9, 1)
        # the layer's weight gradient (training): tensor cores (default) and mma.sync
        gy = ly.clone()
        gw = torch.zeros((layer.cout, layer.kpad), device=device, dtype=torch.float32)
        gb = torch.zeros(layer.cout, device=device, dtype=torch.float32)
        winfo = (ctypes.c_int * 8)()
        row["wgrad_plan"] = list(winfo) if lib.pmd_conv3d_wgrad_plan(*dims, layer.cin, layer.cout,
                                                                     winfo) == 0 else None
        for name, impl in (("wgrad", 0), ("wgrad_mma_sync", 1)):
            lib.pmd_conv3d_impl(impl)
            call = lambda: lib.pmd_conv3d_wgrad(lx.data_ptr(), gy.data_ptr(), gw.data_ptr(), gb.data_ptr(),
                                                *dims, layer.cin, layer.cout, layer.kpad,
                                                stream.cuda_stream)
            if call() != 0:
                row[name] = -1
                continue
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(args.steps):
                call()
            e1.record(stream)
            e1.synchronize()
            row[name] = round(e0.elapsed_time(e1) / args.steps, 4)
            row[name + "_tflops"] = round(lflops / row[name] / 1e9, 1)
        layers[layer.name] = row
        del lx, lw, ly, gy, gw, gb
    lib.pmd_conv3d_impl(previous)
    out["layers_ms"] = layers

    # one inference chunk of the whole network (16 windows, the committed weights)
    from pyradmc_b200.denoiser import UNet3D, forward_flops_per_voxel

    net = UNet3D.load(DENOISER_WEIGHTS, device=device)
    dose = torch.rand((b, d, h, w), device=device, generator=gen)
    rho = torch.ones((b, d, h, w), device=device)
    sg = 0.1 * dose
    flops_net = forward_flops_per_voxel() * b * d * h * w
    for name, impl in (("unet_chunk", previous),):
        lib.pmd_conv3d_impl(impl)
        for _ in range(args.warmup):
            net.predict(dose, rho, sigma=sg)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = net.launches
        e0.record(stream)
        for _ in range(args.steps):
            net.predict(dose, rho, sigma=sg)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        out[name] = {"ms": ms, "tflops": flops_net / ms / 1e9,
                     "launches": (net.launches - launches) / args.steps}
    lib.pmd_conv3d_impl(previous)

    # one training step (forward, loss, backward with the tensor-core weight
    # gradients, Adam) on a batch of the trainer's shape: 4 windows of 64^3
    tb = (4, 64, 64, 64)
    t_dose = torch.rand(tb, device=device, generator=gen)
    t_rho = torch.ones(tb, device=device)
    t_target = 0.9 * t_dose
    t_sigma = 0.1 * t_dose
    trainer = UNet3D.load(DENOISER_WEIGHTS, device=device)
    trainer.lr = 1e-5
    for _ in range(args.warmup):
        trainer.train_step(t_dose, t_rho, t_target, sigma=t_sigma)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        trainer.train_step(t_dose, t_rho, t_target, sigma=t_sigma)
    e1.record(stream)
    e1.synchronize()
    out["train_step_ms"] = {"batch": list(tb), "ms": round(e0.elapsed_time(e1) / args.steps, 3)}
    out["failures"] = lib.pmd_conv3d_failures()
    print(json.dumps(out), flush=True)
    return 0


def b200_arm(args, world, rank, local):
    import torch

    from pyradmc_b200 import B200Engine, phantoms

    device = f"cuda:{local}"
    torch.cuda.set_device(local)
    grid, xs, source, counts = workload(rank)
    # N > 1: one Dij of N x 100 columns (the benchmark fan N times over, every
    # copy with its own history keys), each rank its share of the columns
    # (engine.column_shards, history-balanced): weak scaling through the
    # product's own sharding, no collective on the data path
    whole, whole_counts, span = source, counts, None
    if world > 1:
        from pyradmc_b200.engine import column_shards
        from pyradmc_b200.model import ConcatenatedBeamletSource

        whole = ConcatenatedBeamletSource([source] * world)
        whole_counts = np.tile(counts, world)
        span = column_shards(whole_counts, world)[rank]
    engine = B200Engine(grid, xs, device=device, use_graph=not args.no_graph)
    tune_report = None
    if not args.no_autotune:
        from pyradmc_b200 import autotune

        # probe the workload itself: shorter probes favour lower residency than
        # the full Dij wants
        engine, tune_report = autotune.tune(engine, source, counts, N_BATCHES, SEED,
                                            fraction=1.0, repeats=1)
    stream = torch.cuda.Stream(device=device)  # an explicit stream: the legacy default is 0
    torch.cuda.set_stream(stream)
    engine.use_stream(stream.cuda_stream)
    kw = dict(n_histories_per_beamlet=whole_counts, n_batches=N_BATCHES, seed=SEED)
    if span is not None:
        kw["columns"] = span
    histories = int(np.sum(whole_counts[span[0]:span[1]])) if span is not None else int(np.sum(counts))
    histories_all = int(all_sum(world, [histories])[0])
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=device)  # > 126 MB L2

    for _ in range(args.warmup):
        view = engine.run_dij_device(whole, truncation=1e-3, **kw)
    peaks_path = ROOT / "MEASURED_PEAKS.json"
    peaks = json.loads(peaks_path.read_text()) if peaks_path.exists() else {}
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))

    # device-resident steps
    step_ms, counters = [], []
    with ClockSampler(local) as clocks:
        barrier(world)
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.fill_(1)
            start = torch.cuda.Event(enable_timing=True)
            end = torch.cuda.Event(enable_timing=True)
            start.record(stream)
            view = engine.run_dij_device(whole, truncation=1e-3, **kw)  # CSC stays in HBM
            end.record(stream)
            end.synchronize()
            step_ms.append(start.elapsed_time(end))
            counters.append(engine.last_counters())
        torch.cuda.synchronize()
        barrier(world)
    total_ms = all_max(world, [sum(step_ms)])[0]
    value = job_value(histories_all, args.steps, total_ms)

    # end to end from host data: uploads and readback inside the timed region.
    # Warm-up first: each result holds its CSC in page-locked host blocks that
    # the caching allocator recycles once the result is dropped; the loop keeps
    # one result alive while the next runs, so two sets get pinned (a first
    # pinning of ~200 MB costs ~0.1 s) before timing starts.
    def e2e_call():
        if span is None:
            return engine.run_dij(whole, **kw)
        e2e_kw = {k: v for k, v in kw.items() if k != "columns"}
        return engine.run_dij_shard(whole, rank=rank, world=world, **e2e_kw)[0]

    dij = None
    for _ in range(max(args.warmup, 2)):
        engine.drop_uploads()
        dij = e2e_call()
    e2e_ms, h2d, d2h = [], [], []
    barrier(world)
    torch.cuda.synchronize()
    for _ in range(args.steps):
        engine.drop_uploads()
        before = engine.last_counters()
        t0 = time.perf_counter()
        dij = e2e_call()
        dense_ok = dij.indptr[-1] == dij.indices.size
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
        after = engine.last_counters()
        h2d.append(after["h2d_bytes_total"] - before["h2d_bytes_total"])
        d2h.append(after["d2h_bytes_total"] - before["d2h_bytes_total"])
        assert dense_ok
    torch.cuda.synchronize()
    barrier(world)
    e2e_total = all_max(world, [sum(e2e_ms)])[0]
    e2e_value = job_value(histories_all, args.steps, e2e_total)

    c = counters[-1]
    # the method comparisons are one-GPU workloads: rank 0 of a one-rank run
    den = None if args.no_denoiser or world > 1 else denoiser_leg(
        args, engine, source, counts, stream, device, total_ms / args.steps / 1e3)
    parity = parity_block(device) if world == 1 else None
    presolve = presolve_leg(device) if world == 1 else None
    plan = None
    if not args.no_plan and world == 1:
        engine.drop_uploads()
        torch.cuda.empty_cache()
        plan = plan_leg(args, device, stream)
    transport_s = c["transport_ms"] / 1e3
    achieved = algorithmic_bytes(c) / transport_s / 1e9
    sigma = phantoms.per_beamlet_sigma(dij)
    s_per_dij = total_ms / args.steps / 1e3
    s_at_2pct = s_per_dij * (sigma / 0.02) ** 2
    totals = all_sum(world, [dij.energy_deposited, dij.energy_escaped, dij.energy_emitted])
    if rank != 0:
        return 0
    clock = clocks.summary()
    base = cpu_baseline(grid, xs, source, counts) if world == 1 and not args.no_cpu_baseline else None
    traffic_path = ROOT / "profiles" / "transport_traffic.json"
    traffic = None
    if traffic_path.exists():
        t = json.loads(traffic_path.read_text())
        traffic = t.get("bytes_per_history", 0.0) * histories if t.get("bytes_per_history") else None
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "histories/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32 transport, int64 scoring, f64 statistics",
        "data": "synthetic (seeded phantom and beamlet counts)",
        "config": {**config_dict(counts, "256 MB buffer written between timed steps (flush)"),
                   "launch": {"block_size": engine.block_size, "blocks_per_sm": engine.blocks_per_sm,
                              "chunk_size": engine.chunk_size, "tail_steps": engine.tail_steps,
                              "smem_tables": engine.smem_tables,
                              "autotuned": tune_report is not None,
                              "tune_cached": None if tune_report is None else tune_report["cached"]}},
        "s_per_dij": s_per_dij,
        "per_beamlet_sigma": sigma,
        "s_per_dij_at_2pct_sigma": s_at_2pct,
        "plain_2pct": "extrapolated: measured s per Dij x (per-beamlet sigma / 2 %)^2 (1/sqrt(N) scaling)",
        "denoiser": den,
        "plan": plan,
        "parity": parity,
        "presolve": presolve,
        "e2e": {"value": e2e_value, "unit": "histories/s",
                "h2d_bytes_per_step": int(np.median(h2d)), "d2h_bytes_per_step": int(np.median(d2h)),
                "ms_per_step": e2e_total / args.steps},
        "roofline": {
            "bound": "hbm",
            "kernel": "photon_kernel+electron_kernel (transport graph)",
            "achieved": achieved,
            "peak": hbm_peak,
            "unit": "GB/s",
            "frac": achieved / hbm_peak,
            "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
            "traffic": traffic,
            "issue_bound": {
                "what": "transport is bounded by instruction issue and load latency, not HBM: "
                        "fraction of cycles each SM sub-partition issued, ncu on a main round "
                        "of this workload",
                "photon_kernel": 0.343, "electron_kernel": 0.540,
                "simd_lanes_active": {"photon_kernel": 7.9 / 32, "electron_kernel": 16.3 / 32},
                "source": "profiles/transport_main_round_dij100_ncu.md"},
            "algorithmic_bytes": algorithmic_bytes(c),
            "transport_ms": c["transport_ms"],
            "reduce_ms": c["reduce_ms"],
        },
        "gpu_launches": int(sum(x["kernel_launches"] for x in counters)),
        "counters": {k: c[k] for k in ("photon_flights", "photon_interactions", "electron_substeps",
                                       "deposits", "queue_pushes", "primaries", "rounds")},
        "energy_balance": (totals[0] + totals[1]) / totals[2],
        "clocks": clock,
        "cpu_baseline": base,
    }
    print(json.dumps(line), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("b200", "reference"), default="b200")
    ap.add_argument("--workload", choices=("dij100", "dij10", "conv"), default="dij100",
                    help="dij10: the reduced transport case of the ncu captures; conv: the "
                         "denoiser's dominant convolution alone")
    ap.add_argument("--no-graph", action="store_true",
                    help="drain batches with the host loop instead of the CUDA graph (bit-identical; "
                         "ncu cannot profile kernels inside graphs with conditional nodes)")
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline leg (profiling runs)")
    ap.add_argument("--no-denoiser", action="store_true",
                    help="skip the MC + denoiser leg (profiling runs)")
    ap.add_argument("--no-plan", action="store_true",
                    help="skip the full-plan leg (2,800 columns on a 256 x 256 x 128 phantom)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="default launch shape instead of the autotuned one")
    args = ap.parse_args()
    global WORKLOAD
    WORKLOAD = args.workload
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            return reference_arm(args, world, rank)
        if args.workload == "conv":
            return conv_arm(args, local)
        return b200_arm(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    sys.exit(main())
