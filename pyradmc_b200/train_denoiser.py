"""Train the Dij-column denoiser on pairs the engine makes, and evaluate it.

``python -m pyradmc_b200.train_denoiser --out weights.npz`` builds the training
set of the denoiser workload: seeded CT-like phantoms (128^3 at 2.5 mm, water
plus 6-12 random ellipsoids), a 10x10 lattice of 5x5 mm 6 MV beamlets on each,
every column run at each ``--n-low`` count and at ``--n-high`` histories per
beamlet, cropped to 64^3 windows around the beamlet (input: the low-history
dose and its Monte Carlo sigma, plus the density); then trains the U-Net with Adam on the
device (the project's own forward and backward kernels) and evaluates it on a
held-out phantom against high-statistics Monte Carlo.  One JSON line with the
loss curve and the evaluation goes to stdout.
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
from .phantoms import beamlet_fan, ellipsoid_phantom

TRAIN_SEED0 = 1000      # phantom seeds of the training set: TRAIN_SEED0 + i
HELD_OUT_SEED = 999     # the evaluation phantom


def phantom(seed: int):
    grid = ellipsoid_phantom(seed=seed)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    return grid, xs, beamlet_fan(grid)


def build_pairs(n_phantoms: int, n_low, n_high: int, n_batches: int, device: str, log):
    import torch

    sets = []
    for i in range(n_phantoms):
        t0 = time.perf_counter()
        grid, xs, fan = phantom(TRAIN_SEED0 + i)
        sets.append(D.make_pairs(grid, xs, fan, n_low=n_low, n_high=n_high, n_batches=n_batches,
                                 seed=20260726 + 101 * i, device=device,
                                 rng=np.random.default_rng(i)))
        torch.cuda.empty_cache()
        log(f"phantom {i}: {len(sets[-1])} pairs in {time.perf_counter() - t0:.1f} s")
    return D.concat(sets)


def evaluate(net: UNet3D, n_levels, n_ref: int, n_batches: int, device: str, laterals=(64,)):
    """Per-beamlet sigma-equivalent error of plain MC and of MC + denoiser (for
    each lateral window size) at each history level, on the held-out phantom,
    against an n_ref-history run."""
    import torch

    from .engine import B200Engine

    grid, xs, fan = phantom(HELD_OUT_SEED)
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
            window = D.inference_window(shape, lateral)
            D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg, window=window)  # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            den = D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg, window=window)
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
    ap.add_argument("--init", default=None, help="start from these weights")
    ap.add_argument("--eval-only", action="store_true",
                    help="evaluate the --init weights without training")
    ap.add_argument("--eval-levels", default="10000,30000,100000,300000")
    ap.add_argument("--n-ref", type=int, default=4_000_000)
    ap.add_argument("--eval-lateral", default="64")
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
        pairs = build_pairs(args.phantoms, n_low, args.n_high, args.n_batches, args.device, log)
        n_pairs = len(pairs)
        t_data = time.perf_counter() - t0
        t0 = time.perf_counter()
        history = D.train(net, pairs, steps=args.steps, batch=args.batch, lr_final=args.lr_final,
                          log_every=max(args.steps // 40, 1), log=log)
        t_train = time.perf_counter() - t0
        net.save(args.out)
        del pairs
    net.release_workspaces()
    torch.cuda.empty_cache()  # the engine allocates outside torch's cache
    levels = [int(v) for v in args.eval_levels.split(",") if v]
    laterals = [int(v) for v in args.eval_lateral.split(",") if v]
    ev = evaluate(net, levels, args.n_ref, args.n_batches, args.device, laterals)
    print(json.dumps({"pairs": n_pairs, "n_low": n_low, "n_high": args.n_high,
                      "loss_lambda": args.loss_lambda, "data_s": t_data, "train_s": t_train,
                      "steps": args.steps, "loss": history, "evaluation": ev}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
