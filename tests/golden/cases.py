"""Parity cases shared by the golden-fixture generator and the tests.

Each case is plain data: a grid, a source and the run options.  The generator
(``make_golden.py``) builds them with pyRadMC's own classes and runs its
``ReferenceEngine``; the tests build the same case with this package's mirror
classes and run it through the B200 engine, then compare statistically
(batched chi-squared, the reference's own detection oracle).

Geometries and sources follow the reference's own parity tests:
``tests/integration/test_warp_backend.py:39-49`` (slab + 6 MeV parallel field,
electron beam), ``tests/dij/test_dij_warp.py:41-55`` (2x2 lattice), and the
README quick start (``README.md:68-82``) for the 16^3 pencil-beam case.
"""

from __future__ import annotations

SEED = 20260711  # the reference test suite's fixed seed (tests/conftest.py:25)

# Water slab with a density step, for the heterogeneous spectral case: water,
# lung 0.26, bone 1.85, water, by voxel-centre depth in cm.
SLAB_LAYERS = ((0.0, 3.0, 1.0), (3.0, 7.0, 0.26), (7.0, 9.0, 1.85), (9.0, 1.0e9, 1.0))

CASES: dict[str, dict] = {
    "kerma_slab": dict(
        grid=dict(shape=(8, 8, 30), spacing=(2.0, 2.0, 0.2)),
        source=dict(kind="parallel", energy=6.0, z=-1.0, x_range=(0.0, 16.0), y_range=(0.0, 16.0)),
        run=dict(n_histories=6000, n_batches=12, seed=SEED, transport_electrons=False),
    ),
    "full_slab": dict(
        grid=dict(shape=(8, 8, 30), spacing=(2.0, 2.0, 0.2)),
        source=dict(kind="parallel", energy=6.0, z=-1.0, x_range=(0.0, 16.0), y_range=(0.0, 16.0)),
        run=dict(n_histories=4000, n_batches=8, seed=SEED, transport_electrons=True),
    ),
    "full_slab_gaussian": dict(
        grid=dict(shape=(8, 8, 30), spacing=(2.0, 2.0, 0.2)),
        source=dict(kind="parallel", energy=6.0, z=-1.0, x_range=(0.0, 16.0), y_range=(0.0, 16.0)),
        run=dict(n_histories=4000, n_batches=8, seed=SEED, transport_electrons=True,
                 msc_model="gaussian"),
    ),
    "electron_beam": dict(
        grid=dict(shape=(8, 8, 40), spacing=(2.0, 2.0, 0.1)),
        source=dict(kind="parallel", energy=5.0, z=-0.5, x_range=(0.0, 16.0), y_range=(0.0, 16.0)),
        run=dict(n_histories=1200, n_batches=8, seed=SEED, primary_kind="electron"),
    ),
    "readme_pencil": dict(
        grid=dict(shape=(16, 16, 16), spacing=(1.0, 1.0, 1.0)),
        source=dict(kind="pencil", energy=6.0, position=(8.0, 8.0, -1.0), direction=(0.0, 0.0, 1.0)),
        run=dict(n_histories=80000, n_batches=10, seed=20260726),
    ),
    "slab_spectral": dict(
        grid=dict(shape=(64, 64, 64), spacing=(0.2, 0.2, 0.2), layers=SLAB_LAYERS),
        source=dict(kind="spectral", focal_point=(6.4, 6.4, -100.0), center=(6.4, 6.4, 0.0),
                    width_u=10.0, width_v=10.0),
        run=dict(n_histories=8000, n_batches=16, seed=SEED),
    ),
    "dij_lattice": dict(
        grid=dict(shape=(8, 8, 16), spacing=(2.0, 2.0, 0.5)),
        source=dict(kind="lattice", energy=6.0, z=-1.0, x_range=(2.0, 14.0), y_range=(2.0, 14.0),
                    n_x=2, n_y=2),
        run=dict(n_histories_per_beamlet=800, n_batches=8, seed=SEED, truncation=0.0),
    ),
    "dij_spectral": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="spectral_beamlets", focal_point=(4.0, 4.0, -100.0),
                    centers=((3.0, 3.0, 0.0), (5.0, 3.0, 0.0), (3.0, 5.0, 0.0), (5.0, 5.0, 0.0)),
                    width_u=1.5, width_v=1.5),
        run=dict(n_histories_per_beamlet=480, n_batches=8, seed=SEED, truncation=0.0),
    ),
}


def layered_density(shape, spacing, origin, layers):
    """Density by voxel-centre depth: (z_lo, z_hi, density) slabs along z."""
    import numpy as np

    nz = shape[2]
    z = origin[2] + (np.arange(nz) + 0.5) * spacing[2]
    column = np.ones(nz)
    for lo, hi, rho in layers:
        column[(z >= lo) & (z < hi)] = rho
    return np.broadcast_to(column, shape).copy()
