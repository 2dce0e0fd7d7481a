"""What the trained denoiser gains over the method without it.

The committed network (``pyradmc_b200/data/denoiser_unet.npz``, trained on the
engine's own pairs from other phantoms) denoises a row of ten beamlets on a
held-out CT-like phantom at 3e4 histories per beamlet.  Judged by a
high-statistics run of the same beamlets (4e6 histories each), its
per-beamlet sigma-equivalent error must be well below plain Monte Carlo's at
the same histories — and plain Monte Carlo stays the fallback and the judge.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_denoiser_beats_plain_monte_carlo_at_equal_histories(gpu):
    import torch

    from pyradmc_b200 import B200Engine, denoise_dij as D, phantoms
    from pyradmc_b200.denoiser import UNet3D
    from pyradmc_b200.model import AnalyticWaterTables

    grid = phantoms.ellipsoid_phantom(seed=4242)  # not one of the training phantoms
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    fan = phantoms.beamlet_fan(grid, n_x=10, n_y=1)
    engine = B200Engine(grid, xs, device=gpu)
    net = UNet3D.load(D.__file__.replace("denoise_dij.py", "data/denoiser_unet.npz"), device=gpu)
    shape = tuple(grid.shape)
    ref = engine.run_dij_device(fan, 4_000_000, 10, 99, truncation=0.0)
    ref_dose, _, ref_sigma = D.dense_columns(ref, gpu, with_sigma=True)
    low = engine.run_dij_device(fan, 30_000, 10, 5, truncation=0.0)
    dose, colmax, sg = D.dense_columns(low, gpu, with_sigma=True)
    rho = torch.from_numpy(np.ascontiguousarray(grid.density, dtype=np.float32).ravel()).to(gpu)
    den = D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg,
                          window=D.inference_window(shape, 64),
                          directions=D.beam_directions(fan), spacing=grid.spacing)
    plain = float(np.nanmean(D.sigma_equivalent_error(dose, ref_dose, ref_sigma)))
    denoised = float(np.nanmean(D.sigma_equivalent_error(den, ref_dose, ref_sigma)))
    assert net.lib.pmd_conv3d_failures() == 0
    assert np.isfinite(den.cpu().numpy()).all()
    assert denoised < 0.6 * plain, (plain, denoised)


WEIGHTS = "data/denoiser_unet.npz"                     # the axial fan's network
COPLANAR_WEIGHTS = "data/denoiser_unet_coplanar.npz"   # gantry beams (oblique beamlets)


def _gain(gpu, grid, fan, n_low, n_ref=4_000_000, window=None, weights=WEIGHTS):
    import torch

    from pyradmc_b200 import B200Engine, denoise_dij as D
    from pyradmc_b200.denoiser import UNet3D
    from pyradmc_b200.model import AnalyticWaterTables

    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    engine = B200Engine(grid, xs, device=gpu)
    net = UNet3D.load(D.__file__.replace("denoise_dij.py", weights), device=gpu)
    shape = tuple(grid.shape)
    ref = engine.run_dij_device(fan, n_ref, 10, 99, truncation=0.0)
    ref_dose, _, ref_sigma = D.dense_columns(ref, gpu, with_sigma=True)
    low = engine.run_dij_device(fan, n_low, 10, 5, truncation=0.0)
    dose, colmax, sg = D.dense_columns(low, gpu, with_sigma=True)
    rho = torch.from_numpy(np.ascontiguousarray(grid.density, dtype=np.float32).ravel()).to(gpu)
    den = D.denoise_dense(net, dose, colmax, rho, shape, sigma=sg,
                          window=window or D.inference_window(shape, 64),
                          directions=D.beam_directions(fan), spacing=grid.spacing)
    assert net.lib.pmd_conv3d_failures() == 0
    return D.error_report(dose, ref_dose, ref_sigma), D.error_report(den, ref_dose, ref_sigma)


def test_denoiser_is_unbiased_where_the_dij_keeps_entries(gpu):
    """The signed error of the denoised columns (against 4e6-history Monte
    Carlo) stays small in the beamlet core and in the penumbra, not only the
    sigma-equivalent (absolute) error: a network that shrank or widened the
    beamlet would show here."""
    from pyradmc_b200 import phantoms

    grid = phantoms.ellipsoid_phantom(seed=4242)
    plain, den = _gain(gpu, grid, phantoms.beamlet_fan(grid, n_x=10, n_y=1), 100_000)
    for t in ("0.5", "0.1"):
        assert abs(den[t]["bias_integral"]) < 0.02, (t, den[t])
        assert abs(den[t]["bias_integral"] - plain[t]["bias_integral"]) < 0.02, (t, den[t], plain[t])
    assert den["0.5"]["sigma_eq"] < plain["0.5"]["sigma_eq"]


def test_denoiser_gains_on_an_oblique_beam_outside_the_training_set(gpu):
    """The network for coplanar plans, on 8 mm beamlets from a focal spot 90 cm
    away at gantry angle 33 degrees, on a 3 mm phantom whose seed the training
    set does not use (training draws its gantry angles, widths and focal
    distances at random on other phantoms).  The windows follow the oblique
    beamlets (sheared along them); the network must beat plain Monte Carlo at
    equal histories in the beamlet core without a signed bias."""
    from pyradmc_b200 import train_denoiser as T

    grid, _, fan = T.held_out_oblique()
    plain, den = _gain(gpu, grid, fan, 30_000, window=(64, 64, 64), weights=COPLANAR_WEIGHTS)
    assert den["0.5"]["sigma_eq"] < 0.7 * plain["0.5"]["sigma_eq"], (plain, den)
    assert abs(den["0.5"]["bias_integral"]) < 0.02, den


def test_pipelined_groups_give_the_same_dij(gpu):
    """run_dij_denoised with the denoising of one column group overlapping the
    transport of the next (a second stream) equals the one-group call bit for
    bit: every column keeps its history keys and every kernel is deterministic."""
    from pyradmc_b200 import B200Engine, denoise_dij as D, phantoms
    from pyradmc_b200.denoiser import UNet3D
    from pyradmc_b200.model import AnalyticWaterTables

    grid = phantoms.ellipsoid_phantom(shape=(64, 64, 64), seed=4244)
    xs = AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    fan = phantoms.beamlet_fan(grid, n_x=3, n_y=2)
    engine = B200Engine(grid, xs, device=gpu)
    net = UNet3D.load(D.__file__.replace("denoise_dij.py", WEIGHTS), device=gpu)
    kw = dict(truncation=1e-3, lateral=32)
    one = D.run_dij_denoised(engine, net, fan, 20_000, 10, 3, **kw)
    two = D.run_dij_denoised(engine, net, fan, 20_000, 10, 3, group_columns=2, overlap=True, **kw)
    for f in ("indptr", "indices", "dose", "sigma"):
        np.testing.assert_array_equal(getattr(one, f), getattr(two, f))
    assert one.energy_deposited == two.energy_deposited
    assert net.lib.pmd_conv3d_failures() == 0
