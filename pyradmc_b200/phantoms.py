"""Synthetic phantoms and beam layouts of the benchmark workloads.

Seeded stand-ins for the CT-like inputs the benchmark names (there is no
dataset): the density maps are water (material 0) at varying density, the form
the analytic water-only cross sections accept (data/analytic.py:146-154).
"""

from __future__ import annotations

import numpy as np

from pyradmc_b200 import model


def ellipsoid_phantom(shape=(128, 128, 128), spacing=(0.25, 0.25, 0.25), seed=20260726,
                      n_range=(6, 12), density_range=(0.2, 1.9), semi_axis_range=(1.0, 4.0)):
    """Water background plus 6-12 random ellipsoids with densities U(0.2, 1.9).

    Centres are uniform over the middle 80 % of the box; semi-axes U(1, 4) cm;
    later ellipsoids overwrite earlier ones where they overlap.
    """
    rng = np.random.default_rng(seed)
    extent = np.array(shape) * np.array(spacing)
    axes = [(np.arange(n) + 0.5) * s for n, s in zip(shape, spacing, strict=True)]
    x, y, z = np.meshgrid(*axes, indexing="ij")
    density = np.ones(shape)
    for _ in range(int(rng.integers(n_range[0], n_range[1] + 1))):
        c = extent * (0.1 + 0.8 * rng.random(3))
        a = rng.uniform(*semi_axis_range, size=3)
        rho = rng.uniform(*density_range)
        inside = ((x - c[0]) / a[0]) ** 2 + ((y - c[1]) / a[1]) ** 2 + ((z - c[2]) / a[2]) ** 2 <= 1.0
        density[inside] = rho
    return model.VoxelGrid(shape=tuple(shape), spacing=tuple(spacing), density=density,
                           material=np.zeros(shape, dtype=np.int32))


def slab_phantom(shape=(64, 64, 64), spacing=(0.2, 0.2, 0.2)):
    """Water 0-3 cm, lung 0.26 3-7 cm, bone 1.85 7-9 cm, water beyond (by voxel-centre depth)."""
    z = (np.arange(shape[2]) + 0.5) * spacing[2]
    column = np.ones(shape[2])
    column[(z >= 3.0) & (z < 7.0)] = 0.26
    column[(z >= 7.0) & (z < 9.0)] = 1.85
    density = np.broadcast_to(column, shape).copy()
    return model.VoxelGrid(shape=tuple(shape), spacing=tuple(spacing), density=density,
                           material=np.zeros(shape, dtype=np.int32))


def beamlet_fan(grid, n_x=10, n_y=10, pitch=0.5, width=0.5, sad=100.0, spectrum=None):
    """A 10x10 lattice of pitch-spaced beamlet apertures at the isocentre plane.

    The isocentre is the phantom centre; the focal spot sits ``sad`` cm above it
    on the beam axis (+z travel).
    """
    extent = np.array(grid.shape) * np.array(grid.spacing)
    iso = np.asarray(grid.origin) + 0.5 * extent
    centers = [(iso[0] + (i - (n_x - 1) / 2) * pitch, iso[1] + (j - (n_y - 1) / 2) * pitch, iso[2])
               for i in range(n_x) for j in range(n_y)]
    focal = (iso[0], iso[1], iso[2] - sad)
    spectrum = spectrum if spectrum is not None else model.ali_rogers_varian_6mv()
    return model.SpectralBeamletSource(spectrum, focal, centers, width, width)


def gantry_beam(grid, angle_deg, n_u=10, n_v=10, pitch=0.5, width=0.5, sad=100.0, spectrum=None):
    """One coplanar beam at gantry angle `angle_deg` about the z axis through
    the phantom centre (the isocentre): the beam travels along (sin t, cos t, 0)
    from a focal spot `sad` cm before the isocentre, through an n_u x n_v
    lattice of pitch-spaced `width` apertures on the axes (cos t, -sin t, 0)
    and z."""
    extent = np.array(grid.shape) * np.array(grid.spacing)
    iso = np.asarray(grid.origin) + 0.5 * extent
    spectrum = spectrum if spectrum is not None else model.ali_rogers_varian_6mv()
    t = np.deg2rad(angle_deg)
    d = np.array([np.sin(t), np.cos(t), 0.0])
    u = np.array([np.cos(t), -np.sin(t), 0.0])
    v = np.array([0.0, 0.0, 1.0])
    centers = [tuple(iso + (i - (n_u - 1) / 2) * pitch * u + (j - (n_v - 1) / 2) * pitch * v)
               for i in range(n_u) for j in range(n_v)]
    return model.SpectralBeamletSource(spectrum, tuple(iso - sad * d), centers, width, width,
                                       tuple(u), tuple(v))


def coplanar_plan(grid, n_beams=7, n_u=20, n_v=20, pitch=0.5, width=0.5, sad=100.0,
                  spectrum=None, first_angle_deg=0.0):
    """A coplanar treatment plan: `n_beams` equi-spaced gantry angles
    (:func:`gantry_beam`), each an n_u x n_v lattice of beamlet apertures at
    the isocentre plane.  Returns a ConcatenatedBeamletSource of one
    SpectralBeamletSource per beam (beam-major column order) and the gantry
    angles in degrees.
    """
    spectrum = spectrum if spectrum is not None else model.ali_rogers_varian_6mv()
    angles = [float(first_angle_deg + 360.0 * k / n_beams) for k in range(n_beams)]
    beams = [gantry_beam(grid, a, n_u, n_v, pitch, width, sad, spectrum) for a in angles]
    return model.ConcatenatedBeamletSource(beams), angles


def log_uniform_counts(n_beamlets=100, lo=1.0e4, hi=1.0e6, n_batches=10, seed=20260726):
    """Per-beamlet history counts 10**U(log10 lo, log10 hi), rounded to n_batches multiples."""
    rng = np.random.default_rng(seed + 1)
    raw = 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), size=n_beamlets)
    counts = np.maximum(n_batches, np.round(raw / n_batches).astype(np.int64) * n_batches)
    return counts


def per_beamlet_sigma(dij, threshold=0.5) -> float:
    """Mean over columns of the median sigma/dose over entries >= 50 % of the column max
    (the reference's per-beamlet noise measure, examples/noise_bias_study.py:130-144)."""
    values = []
    for j in range(dij.n_beamlets):
        lo, hi = int(dij.indptr[j]), int(dij.indptr[j + 1])
        d = dij.dose[lo:hi]
        s = dij.sigma[lo:hi]
        if d.size == 0:
            continue
        sel = d >= threshold * d.max()
        if np.any(sel):
            values.append(float(np.median(s[sel] / d[sel])))
    return float(np.mean(values)) if values else float("nan")
