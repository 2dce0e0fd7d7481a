"""Train the Dij-column denoiser on pairs the engine makes, and evaluate it.

``python -m pyradmc_b200.train_denoiser --out weights.npz`` builds the training
set of the denoiser workload: seeded CT-like phantoms (128^3, water plus 6-12
random ellipsoids), each with one 10x10 lattice of 6 MV beamlets, every column
run at each ``--n-low`` count and at ``--n-high`` histories per beamlet,
cropped to 64^3 windows along the beamlet (input: the low-history dose and its
Monte Carlo sigma, plus the density).  With ``--geometry mixed`` (the default)
the phantoms alternate 2.5 and 3 mm voxels and the beams vary: a third travel
along +z as in the benchmark Dij, the rest come from a random gantry angle in
the x-y plane as in a coplanar plan, with beamlet widths of 3-10 mm and focal
distances of 80-120 cm; ``--geometry axial`` keeps the benchmark's 5 mm fan at
100 cm on 2.5 mm phantoms; ``--geometry coplanar`` draws gantry beams only
(mostly 3 mm voxels and 5 mm beamlets, focal distances 90-110 cm);
``--geometry plan`` uses the coplanar plan's own phantom family (256x256x128 at
3 mm, ellipsoids scaled with the box) with one 10x10 gantry beam of 5 mm
beamlets at SAD 100 from a random angle each, the training set of the network
the plan uses.  The U-Net then trains with Adam on the device (the
project's own forward and backward kernels) and is evaluated on held-out
phantoms against high-statistics Monte Carlo.  One JSON line with the loss
curve and the evaluation goes to stdout.
"""

from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np

from . import denoise_dij as D
from .denoiser import UNet3D
from .model import AnalyticWaterTables
from .phantoms import beamlet_fan, ellipsoid_phantom, gantry_beam

TRAIN_SEED0 = 1000      # phantom seeds of the training set: TRAIN_SEED0 + i
HELD_OUT_SEED = 999     # the evaluation phantom


def phantom(seed: int):
    grid = ellipsoid_phantom(seed=seed)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, beamlet_fan(grid)


BEAMLET_WIDTHS_CM = (0.3, 0.5, 0.7, 1.0)


def training_case(i: int, geometry: str = "mixed"):
    """(grid, cross sections, beamlet source) of training phantom i."""
    if geometry == "axial":
        return phantom(TRAIN_SEED0 + i)
    rng = np.random.default_rng(TRAIN_SEED0 + 7 * i)
    if geometry == "plan":  # the coplanar plan's phantom family and beamlets, one gantry beam
        grid = plan_phantom(TRAIN_SEED0 + i)
        xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
        return grid, xs, gantry_beam(grid, float(rng.uniform(0.0, 360.0)))
    if geometry == "coplanar":  # gantry beams as in a coplanar plan, mostly 5 mm at 3 mm voxels
        spacing = 0.3 if i % 4 else 0.25
        grid = ellipsoid_phantom(seed=TRAIN_SEED0 + i, spacing=(spacing,) * 3)
        xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
        width = 0.5 if i % 2 == 0 else float(rng.choice(BEAMLET_WIDTHS_CM))
        return grid, xs, gantry_beam(grid, float(rng.uniform(0.0, 360.0)), pitch=width,
                                     width=width, sad=float(rng.uniform(90.0, 110.0)))
    spacing = 0.25 if i % 2 == 0 else 0.3
    grid = ellipsoid_phantom(seed=TRAIN_SEED0 + i, spacing=(spacing,) * 3)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    width = float(rng.choice(BEAMLET_WIDTHS_CM))
    sad = float(rng.uniform(80.0, 120.0))
    if i % 3 == 0:
        return grid, xs, beamlet_fan(grid, pitch=width, width=width, sad=sad)
    return grid, xs, gantry_beam(grid, float(rng.uniform(0.0, 360.0)), pitch=width, width=width,
                                 sad=sad)


def plan_phantom(seed: int, shape=(256, 256, 128), spacing: float = 0.3):
    """The coplanar plan's phantom family: water plus seeded ellipsoids of
    density U(0.2, 1.9), semi-axes scaled with the box from the 128^3 at 2.5 mm
    case's 1-4 cm."""
    scale = shape[0] * spacing / (128 * 0.25)
    return ellipsoid_phantom(shape=shape, spacing=(spacing,) * 3, seed=seed,
                             semi_axis_range=(1.0 * scale, 4.0 * scale))


def held_out_oblique():
    """A held-out geometry outside the training draws: a phantom seed the
    training set does not use at 3 mm, 8 mm beamlets from a focal spot 90 cm
    away at gantry angle 33 degrees."""
    grid = ellipsoid_phantom(seed=HELD_OUT_SEED - 1, spacing=(0.3, 0.3, 0.3))
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, gantry_beam(grid, 33.0, n_u=10, n_v=1, pitch=0.8, width=0.8, sad=90.0)


def held_out_plan_like():
    """A held-out case shaped like one beam of the coplanar plan: 3 mm voxels, a
    row of ten 5 mm beamlets at SAD 100 from gantry angle 102.86 degrees (the
    plan's third beam), on a phantom seed the training set does not use."""
    grid = ellipsoid_phantom(seed=HELD_OUT_SEED - 2, spacing=(0.3, 0.3, 0.3))
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, gantry_beam(grid, 360.0 * 2 / 7, n_u=10, n_v=1)


def build_pairs(n_phantoms: int, n_low, n_high: int, n_batches: int, device: str, log,
                geometry: str = "mixed"):
    import torch

    sets = []
    for i in range(n_phantoms):
        t0 = time.perf_counter()
        grid, xs, fan = training_case(i, geometry)
        sets.append(D.make_pairs(grid, xs, fan, n_low=n_low, n_high=n_high, n_batches=n_batches,
                                 seed=20260726 + 101 * i, device=device,
                                 rng=np.random.default_rng(i)))
        torch.cuda.empty_cache()
        log(f"phantom {i}: {len(sets[-1])} pairs in {time.perf_counter() - t0:.1f} s")
    return D.concat(sets)


def evaluate(net: UNet3D, n_levels, n_ref: int, n_batches: int, device: str, laterals=(64,),
             case=None, depth=None):
    """Per-beamlet sigma-equivalent error of plain MC and of MC + denoiser (for
    each lateral window size) at each history level, on a held-out case (the
    axial fan on phantom HELD_OUT_SEED by default), against an n_ref-history
    run; ``depth`` is the window's depth chunk (default: the z extent)."""
    import torch

    from .engine import B200Engine

    grid, xs, fan = case if case is not None else phantom(HELD_OUT_SEED)
    directions = D.beam_directions(fan)
    engine = B200Engine(grid=grid, cross_sections=xs, device=device)
    shape = tuple(grid.shape)
    ref = engine.run_dij_device(fan, n_ref, n_batches, 424242, truncation=0.0)
    ref_dose, _, ref_sigma = D.dense_columns(ref, device, with_sigma=True)
    rho = torch.from_numpy(np.ascontiguousarray(grid.density, dtype=np.float32).ravel()).to(device)
    out = {"n_ref": n_ref, "levels": []}
    for n in n_levels:
        run = engine.run_dij_device(fan, int(n), n_batches, 7 + int(n), truncation=0.0)
        dose, colmax, sg = D.dense_columns(run, device, with_sigma=True)
        plain = D.sigma_equivalent_error(dose, ref_dose, ref_sigma)
        level = {"n_per_beamlet": int(n), "plain": float(np.nanmean(plain))}
        for lateral in laterals:
            window = D.inference_window(shape, lateral, depth)
            D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg, window=window,
                            directions=directions, spacing=grid.spacing)  # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            den = D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg, window=window,
                                  directions=directions, spacing=grid.spacing)
            torch.cuda.synchronize()
            t_den = time.perf_counter() - t0
            denoised = D.sigma_equivalent_error(den, ref_dose, ref_sigma)
            level[f"denoised_w{lateral}"] = float(np.nanmean(denoised))
            level[f"denoise_s_w{lateral}"] = t_den
            del den
        out["levels"].append(level)
        del dose, sg
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", required=True, help="weights file (.npz)")
    ap.add_argument("--device", default="cuda:0")
    ap.add_argument("--phantoms", type=int, default=40)
    ap.add_argument("--n-low", default="10000,30000,100000",
                    help="comma-separated input history counts")
    ap.add_argument("--n-high", type=int, default=1_000_000)
    ap.add_argument("--n-batches", type=int, default=10)
    ap.add_argument("--steps", type=int, default=16000)
    ap.add_argument("--batch", type=int, default=4)
    ap.add_argument("--lr", type=float, default=3.0e-4)
    ap.add_argument("--lr-final", type=float, default=3.0e-5)
    ap.add_argument("--loss-lambda", type=float, default=50.0)
    ap.add_argument("--warmup", type=int, default=1000,
                    help="steps of linear learning-rate warm-up (a fine-tune from --init at full "
                         "rate measured a collapse to the identity)")
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--eval-only", action="store_true",
                    help="evaluate the --init weights without training")
    ap.add_argument("--eval-levels", default="10000,30000,100000,300000")
    ap.add_argument("--n-ref", type=int, default=4_000_000)
    ap.add_argument("--eval-lateral", default="64")
    ap.add_argument("--geometry", choices=("mixed", "axial", "coplanar", "plan"), default="mixed",
                    help="training beams: mixed gantry angles, widths and focal distances; the "
                         "benchmark's axial 5 mm fan; coplanar gantry beams as in a plan; or the "
                         "plan's own 256x256x128 phantom family with one gantry beam each")
    args = ap.parse_args(argv)

    def log(msg):
        print(msg, file=sys.stderr, flush=True)

    import torch

    n_low = [int(v) for v in args.n_low.split(",") if v]
    n_pairs, t_data, t_train, history = 0, 0.0, 0.0, []
    if args.init:
        net = UNet3D.load(args.init, device=args.device, lr=args.lr, loss_lambda=args.loss_lambda)
    else:
        net = UNet3D(args.device, seed=0, lr=args.lr, loss_lambda=args.loss_lambda)
    if not args.eval_only:
        t0 = time.perf_counter()
        pairs = build_pairs(args.phantoms, n_low, args.n_high, args.n_batches, args.device, log,
                            args.geometry)
        n_pairs = len(pairs)
        t_data = time.perf_counter() - t0
        t0 = time.perf_counter()
        history = D.train(net, pairs, steps=args.steps, batch=args.batch, lr_final=args.lr_final,
                          log_every=max(args.steps // 40, 1), log=log, warmup=args.warmup)
        t_train = time.perf_counter() - t0
        net.save(args.out)
        del pairs
    net.release_workspaces()
    torch.cuda.empty_cache()  # the engine allocates outside torch's cache
    levels = [int(v) for v in args.eval_levels.split(",") if v]
    laterals = [int(v) for v in args.eval_lateral.split(",") if v]
    ev = evaluate(net, levels, args.n_ref, args.n_batches, args.device, laterals)
    log(f"axial evaluation: {ev}")
    ev_oblique = evaluate(net, levels, args.n_ref, args.n_batches, args.device, laterals,
                          case=held_out_oblique(), depth=64)
    log(f"oblique evaluation: {ev_oblique}")
    ev_plan = evaluate(net, levels, args.n_ref, args.n_batches, args.device, laterals,
                       case=held_out_plan_like(), depth=64)
    print(json.dumps({"pairs": n_pairs, "n_low": n_low, "n_high": args.n_high,
                      "geometry": args.geometry, "loss_lambda": args.loss_lambda,
                      "data_s": t_data, "train_s": t_train, "steps": args.steps, "loss": history,
                      "evaluation": ev, "evaluation_oblique": ev_oblique,
                      "evaluation_plan_beam": ev_plan}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
