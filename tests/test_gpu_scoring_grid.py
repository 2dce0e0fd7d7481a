"""A scoring grid decoupled from the transport grid (pyRadMC's ``ScoringGrid``,
``scoring/grid.py:67-219``): deposits land in the scoring voxel that contains
them, and deposits outside the scoring grid are booked as unscored energy.

Transport does not depend on where it is scored, so with the same seed:
* a scoring grid of 2 x 2 x 2-aligned coarse voxels holds exactly the energy of
  the transport-grid run summed over each coarse voxel;
* a scoring grid covering part of the phantom books the rest as unscored, and
  emitted = deposited + escaped + unscored still closes.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_coarse_and_partial_scoring_grids_book_exactly_the_transport_grid_energy(gpu):
    import pyradmc_b200 as P

    shape, spacing = (8, 8, 16), (0.5, 0.5, 0.5)
    rho = np.ones(shape)
    rho[:, :, 6:10] = 0.4
    grid = P.VoxelGrid(shape=shape, spacing=spacing, density=rho,
                       material=np.zeros(shape, dtype=np.int32))
    xs = P.AnalyticWaterTables(geometry_densities=grid.max_density_by_material())
    engine = P.B200Engine(grid, xs, device=gpu)
    src = P.ParallelBeamSource(6.0, -1.0, (0.5, 3.5), (0.5, 3.5))
    n, kw = 20_000, dict(n_batches=8, seed=20260711)
    fine = engine.run(src, n_histories=n, **kw)
    mass_f = np.asarray(grid.density) * grid.voxel_volume
    e_f = (fine.dose * mass_f).reshape(shape)

    # 2 x 2 x 2 coarse grid over the same box
    cshape = tuple(s // 2 for s in shape)
    mass_c = mass_f.reshape(cshape[0], 2, cshape[1], 2, cshape[2], 2).sum(axis=(1, 3, 5))
    coarse_grid = P.ScoringGrid(shape=cshape, spacing=tuple(2 * s for s in spacing),
                                origin=tuple(grid.origin), voxel_mass=mass_c)
    coarse = engine.run(src, n_histories=n, scoring_grid=coarse_grid, **kw)
    e_c = coarse.dose.reshape(cshape) * mass_c
    rebinned = e_f.reshape(cshape[0], 2, cshape[1], 2, cshape[2], 2).sum(axis=(1, 3, 5))
    np.testing.assert_allclose(e_c, rebinned, rtol=1e-12, atol=1e-15 * np.abs(rebinned).max())
    assert coarse.energy_deposited == pytest.approx(fine.energy_deposited, rel=1e-12)
    assert coarse.energy_escaped == pytest.approx(fine.energy_escaped, rel=1e-12)

    # the upstream half only: the downstream half's energy becomes unscored
    half = (shape[0], shape[1], shape[2] // 2)
    part_grid = P.ScoringGrid(shape=half, spacing=spacing, origin=tuple(grid.origin),
                              voxel_mass=mass_f[:, :, : shape[2] // 2])
    part = engine.run(src, n_histories=n, scoring_grid=part_grid, **kw)
    np.testing.assert_allclose(part.dose.reshape(half), fine.dose.reshape(shape)[:, :, : half[2]],
                               rtol=1e-12, atol=0)
    outside = float(e_f[:, :, half[2]:].sum()) * n  # MeV deposited downstream in the fine run
    assert part.energy_unscored == pytest.approx(outside, rel=1e-9)
    assert part.energy_deposited + part.energy_unscored == pytest.approx(fine.energy_deposited,
                                                                          rel=1e-12)
    balance = (part.energy_deposited + part.energy_escaped + part.energy_unscored) / part.energy_emitted
    assert abs(balance - 1.0) < 1e-4, balance


def test_cylindrical_scoring_books_the_energy_of_the_voxel_grid_run(gpu):
    """Depth bins by radial shells (CylindricalScoringGrid, scoring/cylinder.py:
    172) only decide where a deposit is filed: with the same seed the transport
    is identical, so scored plus unscored energy is the voxel-grid run's to the
    quantum, the escaped energy is unchanged, and the shells' dose times their
    analytic mass adds up to the scored energy."""
    import pyradmc_b200 as P
    from tests.conftest import build_case

    grid, xs, src, run = build_case("pencil_cylinder")
    cyl = run.pop("scoring_grid")
    run["n_histories"] = 40_000
    engine = P.B200Engine(grid, xs, device=gpu)
    shells = engine.run(src, scoring_grid=cyl, **run)
    voxels = engine.run(src, **run)
    assert shells.dose.shape == cyl.shape == (16, 12)
    # both books are integer quanta of 1e-9 MeV: equal to the quantum
    assert round((shells.energy_deposited + shells.energy_unscored) * 1e9) == round(
        (voxels.energy_deposited + voxels.energy_unscored) * 1e9)
    assert shells.energy_escaped == voxels.energy_escaped
    assert (shells.dose * cyl.voxel_mass).sum() * run["n_histories"] == pytest.approx(
        shells.energy_deposited, rel=1e-9)
    assert 0.0 < shells.energy_unscored < shells.energy_deposited  # the box corners lie outside
    # the pencil's axis: the central disc carries the highest dose of every depth past build-up
    assert np.all(np.argmax(shells.dose[4:], axis=1) == 0)
