"""Host-side mirror of the pyRadMC objects the B200 engine consumes and returns.

The engine is a drop-in for ``WarpEngine``: it accepts pyRadMC's own
``VoxelGrid``, sources and ``CrossSectionSource`` objects unchanged, and returns
pyRadMC's ``TransportResult``/``DijResult`` when pyRadMC is importable.  Where it
is not (a GPU host with only this package), the classes below stand in with the
same names, fields and semantics, so the same calls work:

* :class:`VoxelGrid`            geometry/grid.py:227
* :class:`PencilBeamSource`     geometry/source.py:279
* :class:`ParallelBeamSource`   geometry/source.py:318
* :class:`BeamletGridSource`    geometry/source.py:350
* :class:`Spectrum`             geometry/spectrum.py:34
* :class:`SpectralBeamSource`   geometry/source.py:560
* :class:`SpectralBeamletSource` geometry/source.py:637
* :class:`CompositeBeamletSource` geometry/source.py:239
* :class:`ScoringGrid`          scoring/grid.py:67 (``for_grid`` only)
* :class:`CylindricalScoringGrid` scoring/cylinder.py:172, with
  :func:`uniform_edges` and :func:`geometric_edges` (:62, :76)
* :class:`RunProvenance`, :class:`TransportResult`  backends/results.py:19, :77
* :class:`DijResult`            scoring/dij.py:195
* :class:`ProgressEvent`, :class:`ProgressEmitter`  progress.py:30, :50
* :class:`AnalyticWaterTables`  the analytic water source's flattened tables
  (data/analytic.py:117 + data/tables.py:222), served from the packs that
  ``pyradmc_b200/data/make_packs.py`` generated with pyRadMC's own builders.
* :class:`PackedCrossSections`  any ``CrossSectionSource``'s flattened tables
  and GS node grid (multi-material, analytic or tabulated EPICS,
  data/tabulated/source.py:58), written by :func:`save_pack` where pyRadMC runs.
"""

from __future__ import annotations

import logging
import math
import threading
import time
from collections.abc import Callable, Sequence
from dataclasses import dataclass, field
from pathlib import Path
from types import SimpleNamespace

import numpy as np

__all__ = [
    "AnalyticWaterTables",
    "BeamletGridSource",
    "CompositeBeamletSource",
    "ConcatenatedBeamletSource",
    "CylindricalScoringGrid",
    "DijResult",
    "PackedCrossSections",
    "ParallelBeamSource",
    "PencilBeamSource",
    "ProgressEmitter",
    "ProgressEvent",
    "RunProvenance",
    "ScoringGrid",
    "SpectralBeamSource",
    "SpectralBeamletSource",
    "Spectrum",
    "TransmissionMaskBeamletSource",
    "TransmissionMaskSource",
    "TransportResult",
    "VoxelGrid",
    "ali_rogers_varian_6mv",
    "geometric_edges",
    "save_pack",
    "uniform_edges",
]

logger = logging.getLogger("pyradmc_b200.progress")

DATA = Path(__file__).resolve().parent / "data"
ELECTRON_MASS_MEV = 0.51099895069
MAJORANT_HEADROOM = 1.0 + 1.0e-6  # data/tables.py:73
GY_PER_MEV_PER_G = 1.602176634e-10
WATER = 0


# ---- geometry ---------------------------------------------------------------------
@dataclass(frozen=True)
class VoxelGrid:
    """Axis-aligned voxel grid with per-voxel density (g/cm^3) and material (cm)."""

    shape: tuple[int, int, int]
    spacing: tuple[float, float, float]
    density: np.ndarray
    material: np.ndarray
    origin: tuple[float, float, float] = (0.0, 0.0, 0.0)

    def __post_init__(self) -> None:
        if any(n < 1 for n in self.shape):
            raise ValueError(f"empty grid shape {self.shape}")
        if any(s <= 0.0 for s in self.spacing):
            raise ValueError(f"non-positive spacing {self.spacing}")
        if self.density.shape != tuple(self.shape):
            raise ValueError(f"density shape {self.density.shape} != grid shape {self.shape}")
        if self.material.shape != tuple(self.shape):
            raise ValueError(f"material shape {self.material.shape} != grid shape {self.shape}")
        if np.any(self.density <= 0.0):
            raise ValueError("non-positive voxel density; vacuum is not supported")
        if np.any(self.material < 0):
            raise ValueError("material index outside the registry")

    @classmethod
    def uniform_water(cls, shape, spacing, origin=(0.0, 0.0, 0.0)) -> VoxelGrid:
        return cls(
            shape=tuple(shape),
            spacing=tuple(spacing),
            origin=tuple(origin),
            density=np.ones(shape, dtype=np.float64),
            material=np.full(shape, WATER, dtype=np.int32),
        )

    @property
    def voxel_volume(self) -> float:
        return self.spacing[0] * self.spacing[1] * self.spacing[2]

    @property
    def upper_corner(self) -> tuple[float, float, float]:
        return tuple(self.origin[i] + self.shape[i] * self.spacing[i] for i in range(3))

    def max_density_by_material(self) -> tuple[tuple[int, float], ...]:
        pairs = []
        for material in np.unique(self.material):
            pairs.append((int(material), float(self.density[self.material == material].max())))
        return tuple(pairs)


@dataclass(frozen=True)
class ScoringGrid:
    """Rectilinear scoring grid; ``for_grid`` is the engines' default."""

    shape: tuple[int, int, int]
    spacing: tuple[float, float, float]
    origin: tuple[float, float, float]
    voxel_mass: np.ndarray

    @classmethod
    def for_grid(cls, grid) -> ScoringGrid:
        return cls(
            shape=tuple(grid.shape),
            spacing=tuple(grid.spacing),
            origin=tuple(grid.origin),
            voxel_mass=np.asarray(grid.density) * grid.voxel_volume,
        )

    @property
    def n_voxels(self) -> int:
        return int(self.shape[0] * self.shape[1] * self.shape[2])


def uniform_edges(r_max: float, n_shells: int) -> np.ndarray:
    """Equal-thickness shell edges 0 .. r_max (scoring/cylinder.py:62)."""
    if n_shells < 1:
        raise ValueError(f"a cylindrical scorer needs at least one shell, got {n_shells}")
    if r_max <= 0.0:
        raise ValueError(f"r_max must be positive, got {r_max}")
    return np.linspace(0.0, r_max, n_shells + 1, dtype=np.float64)


def geometric_edges(r_max: float, n_shells: int, r_min: float) -> np.ndarray:
    """A central disc [0, r_min), then n_shells - 1 equal-ratio shells to r_max
    (scoring/cylinder.py:76)."""
    if n_shells < 2:
        raise ValueError(
            f"geometric edges need at least two shells (a central disc plus one "
            f"geometric shell), got {n_shells}"
        )
    if r_max <= 0.0:
        raise ValueError(f"r_max must be positive, got {r_max}")
    if not 0.0 < r_min < r_max:
        raise ValueError(f"need 0 < r_min < r_max, got r_min={r_min}, r_max={r_max}")
    return np.concatenate(([0.0], np.geomspace(r_min, r_max, n_shells, dtype=np.float64)))


def _check_edges(depth, radial) -> tuple[np.ndarray, np.ndarray]:
    depth = np.asarray(depth, dtype=np.float64)
    radial = np.asarray(radial, dtype=np.float64)
    if depth.ndim != 1 or depth.size < 2:
        raise ValueError("depth_edges needs at least one depth bin, i.e. two depths")
    if np.any(np.diff(depth) <= 0.0):
        raise ValueError("depth_edges must be strictly increasing")
    if radial.ndim != 1 or radial.size < 2:
        raise ValueError("radial_edges needs at least one shell, i.e. two radii")
    if np.any(radial < 0.0):
        raise ValueError("negative radial edge")
    if np.any(np.diff(radial) <= 0.0):
        raise ValueError("radial_edges must be strictly increasing")
    return depth, radial


@dataclass(frozen=True)
class CylindricalScoringGrid:
    """Depth bins by radial shells about an axis parallel to z, the pencil-beam
    kernel geometry (scoring/cylinder.py:172): a scoring geometry only, the
    transport stays on the voxel grid.  Bins are half-open on both axes; the
    shell mass is analytic, ``rho * pi * (r_out^2 - r_in^2) * dz``, which is
    why :meth:`for_grid` refuses a medium that is not uniform over the bins."""

    axis: tuple[float, float]
    depth_edges: np.ndarray
    radial_edges: np.ndarray
    voxel_mass: np.ndarray

    def __post_init__(self) -> None:
        depth, radial = _check_edges(self.depth_edges, self.radial_edges)
        mass = np.asarray(self.voxel_mass, dtype=np.float64)
        if mass.shape != (depth.size - 1, radial.size - 1):
            raise ValueError(
                f"voxel_mass shape {mass.shape} != {(depth.size - 1, radial.size - 1)} "
                "(n_depth, n_shells)")
        if np.any(mass < 0.0):
            raise ValueError("negative shell mass")
        object.__setattr__(self, "depth_edges", depth)
        object.__setattr__(self, "radial_edges", radial)
        object.__setattr__(self, "voxel_mass", mass)

    @classmethod
    def uniform(cls, density: float, axis, depth_edges, radial_edges) -> CylindricalScoringGrid:
        """Bins in a medium of the stated uniform density (scoring/cylinder.py:274)."""
        if density <= 0.0:
            raise ValueError(f"non-positive density {density}")
        depth, radial = _check_edges(depth_edges, radial_edges)
        shell_area = math.pi * (radial[1:] ** 2 - radial[:-1] ** 2)
        mass = density * np.outer(np.diff(depth), shell_area)
        return cls(axis=tuple(axis), depth_edges=depth, radial_edges=radial, voxel_mass=mass)

    @classmethod
    def for_grid(cls, grid, radial_edges, axis=None, depth_edges=None) -> CylindricalScoringGrid:
        """Bins spanning a transport phantom, density read from it and checked
        uniform over every voxel the cylinder meets (scoring/cylinder.py:311)."""
        edges = np.asarray(radial_edges, dtype=np.float64)
        if edges.ndim != 1 or edges.size < 2:
            raise ValueError("radial_edges needs at least one shell, i.e. two radii")
        lo = np.asarray(grid.origin, dtype=np.float64)
        hi = lo + np.asarray(grid.shape) * np.asarray(grid.spacing, dtype=np.float64)
        if axis is None:
            axis = (0.5 * (lo[0] + hi[0]), 0.5 * (lo[1] + hi[1]))
        if depth_edges is None:
            n_depth = max(1, math.floor((hi[2] - lo[2]) / grid.spacing[2]))
            depth_edges = lo[2] + grid.spacing[2] * np.arange(n_depth + 1, dtype=np.float64)
        depth = np.asarray(depth_edges, dtype=np.float64)
        r_max = float(edges[-1])
        if (axis[0] - r_max < lo[0] or axis[0] + r_max > hi[0] or axis[1] - r_max < lo[1]
                or axis[1] + r_max > hi[1] or depth[0] < lo[2] or depth[-1] > hi[2]):
            raise ValueError(
                f"the scoring cylinder (axis {tuple(axis)}, r_max {r_max} cm, depth "
                f"[{depth[0]}, {depth[-1]}) cm) reaches outside the transport grid "
                f"{tuple(lo)} to {tuple(hi)}; its shells would claim mass the phantom does not have")
        nx, ny, nz = grid.shape
        sx, sy, sz = grid.spacing
        x0 = lo[0] + sx * np.arange(nx)
        y0 = lo[1] + sy * np.arange(ny)
        z0 = lo[2] + sz * np.arange(nz)
        dx = np.maximum(0.0, np.maximum(x0 - axis[0], axis[0] - (x0 + sx)))
        dy = np.maximum(0.0, np.maximum(y0 - axis[1], axis[1] - (y0 + sy)))
        lateral = (dx[:, None] ** 2 + dy[None, :] ** 2) < r_max**2
        deep = (z0 + sz > depth[0]) & (z0 < depth[-1])
        overlaps = lateral[:, :, None] & deep[None, None, :]
        densities = np.unique(np.asarray(grid.density)[overlaps])
        materials = np.unique(np.asarray(grid.material)[overlaps])
        if densities.size != 1 or materials.size != 1:
            raise ValueError(
                "cylindrical scoring needs a uniform medium over the binned region "
                f"(found {densities.size} densities and {materials.size} materials there)")
        return cls.uniform(float(densities[0]), axis, depth, edges)

    @property
    def n_depth(self) -> int:
        return self.depth_edges.size - 1

    @property
    def n_shells(self) -> int:
        return self.radial_edges.size - 1

    @property
    def shape(self) -> tuple[int, int]:
        return (self.n_depth, self.n_shells)

    @property
    def n_voxels(self) -> int:
        return self.n_depth * self.n_shells


# ---- sources ----------------------------------------------------------------------
def _normalized(v, name: str) -> tuple[float, float, float]:
    n = math.sqrt(sum(c * c for c in v))
    if n == 0.0:
        raise ValueError(f"zero {name} vector")
    return (v[0] / n, v[1] / n, v[2] / n)


@dataclass(frozen=True)
class PencilBeamSource:
    energy: float
    position: tuple[float, float, float]
    direction: tuple[float, float, float]

    def __post_init__(self) -> None:
        if self.energy <= 0.0:
            raise ValueError(f"non-positive energy {self.energy} MeV")
        object.__setattr__(self, "direction", _normalized(self.direction, "direction"))

    @property
    def max_energy(self) -> float:
        return self.energy


@dataclass(frozen=True)
class ParallelBeamSource:
    energy: float
    z: float
    x_range: tuple[float, float]
    y_range: tuple[float, float]

    def __post_init__(self) -> None:
        if self.energy <= 0.0:
            raise ValueError(f"non-positive energy {self.energy} MeV")
        if self.x_range[1] <= self.x_range[0] or self.y_range[1] <= self.y_range[0]:
            raise ValueError("empty field")

    @property
    def max_energy(self) -> float:
        return self.energy


@dataclass(frozen=True)
class BeamletGridSource:
    energy: float
    z: float
    x_range: tuple[float, float]
    y_range: tuple[float, float]
    n_x: int
    n_y: int

    def __post_init__(self) -> None:
        if self.energy <= 0.0:
            raise ValueError(f"non-positive energy {self.energy} MeV")
        if self.x_range[1] <= self.x_range[0] or self.y_range[1] <= self.y_range[0]:
            raise ValueError("empty field")
        if self.n_x < 1 or self.n_y < 1:
            raise ValueError(f"lattice must be at least 1x1, got {self.n_x}x{self.n_y}")

    @property
    def max_energy(self) -> float:
        return self.energy

    @property
    def n_beamlets(self) -> int:
        return self.n_x * self.n_y

    @staticmethod
    def _edge(bounds, i: int, n: int) -> float:
        lo, hi = bounds
        if i == 0:
            return lo
        if i == n:
            return hi
        return lo + (hi - lo) * (i / n)

    def beamlet_bounds(self, beamlet: int) -> tuple[float, float, float, float]:
        """``(x_lo, x_hi, y_lo, y_hi)``: edges interpolated, never accumulated."""
        if not 0 <= beamlet < self.n_beamlets:
            raise IndexError(f"beamlet {beamlet} outside lattice of {self.n_beamlets}")
        jx, jy = divmod(beamlet, self.n_y)
        return (
            self._edge(self.x_range, jx, self.n_x),
            self._edge(self.x_range, jx + 1, self.n_x),
            self._edge(self.y_range, jy, self.n_y),
            self._edge(self.y_range, jy + 1, self.n_y),
        )


class Spectrum:
    """Histogram photon spectrum sampled by CDF inversion (number convention)."""

    def __init__(self, edges, weights, convention: str = "number") -> None:
        e = np.asarray(edges, dtype=np.float64)
        w = np.asarray(weights, dtype=np.float64)
        if e.ndim != 1 or e.size < 2:
            raise ValueError(f"a spectrum needs at least two edges, got shape {e.shape}")
        if e[0] <= 0.0 or not np.all(np.diff(e) > 0.0):
            raise ValueError("spectrum edges must be positive and strictly increasing")
        if w.shape != (e.size - 1,) or np.any(w < 0.0):
            raise ValueError("need one non-negative weight per bin")
        if convention not in ("number", "energy_fluence"):
            raise ValueError(f"unknown convention {convention!r}")
        if convention == "energy_fluence":
            w = w / (0.5 * (e[:-1] + e[1:]))
        total = float(w.sum())
        if total <= 0.0:
            raise ValueError("spectrum weights must include at least one positive value")
        self._edges = e
        self._p = w / total
        self._cdf = np.cumsum(self._p)

    @property
    def max_energy(self) -> float:
        return float(self._edges[-1])

    @property
    def edges(self) -> np.ndarray:
        return self._edges

    @property
    def cdf(self) -> np.ndarray:
        return self._cdf

    @property
    def bin_probabilities(self) -> np.ndarray:
        return self._p

    @property
    def mean_energy(self) -> float:
        return float(np.sum(self._p * 0.5 * (self._edges[:-1] + self._edges[1:])))


def ali_rogers_varian_6mv() -> Spectrum:
    """The reference's ``ali_rogers_mv("varian-6mv", e_min=0.1)`` (from the pack)."""
    with np.load(DATA / "spectrum_varian_6mv.npz") as z:
        return Spectrum(z["edges"], z["weights"])


@dataclass(frozen=True)
class _Fan:
    focal_point: tuple[float, float, float]
    centers: tuple[tuple[float, float, float], ...]
    width_u: float
    width_v: float
    u_axis: tuple[float, float, float]
    v_axis: tuple[float, float, float]

    def __post_init__(self) -> None:
        if len(self.centers) == 0:
            raise ValueError("a spectral source needs at least one aperture centre")
        if self.width_u < 0.0 or self.width_v < 0.0:
            raise ValueError("aperture widths must be non-negative")
        u = _normalized(self.u_axis, "u_axis")
        v = _normalized(self.v_axis, "v_axis")
        cross = (u[1] * v[2] - u[2] * v[1], u[2] * v[0] - u[0] * v[2], u[0] * v[1] - u[1] * v[0])
        if math.sqrt(sum(c * c for c in cross)) < 1.0e-12:
            raise ValueError("aperture axes are parallel; they must span a plane")
        object.__setattr__(self, "u_axis", u)
        object.__setattr__(self, "v_axis", v)
        object.__setattr__(self, "centers", tuple(tuple(c) for c in self.centers))


class SpectralBeamSource:
    def __init__(self, spectrum, focal_point, center, width_u, width_v,
                 u_axis=(1.0, 0.0, 0.0), v_axis=(0.0, 1.0, 0.0)) -> None:
        self._spectrum = spectrum
        self._fan = _Fan(tuple(focal_point), (tuple(center),), width_u, width_v, u_axis, v_axis)

    max_energy = property(lambda self: self._spectrum.max_energy)
    spectrum = property(lambda self: self._spectrum)
    focal_point = property(lambda self: self._fan.focal_point)
    center = property(lambda self: self._fan.centers[0])
    width_u = property(lambda self: self._fan.width_u)
    width_v = property(lambda self: self._fan.width_v)
    u_axis = property(lambda self: self._fan.u_axis)
    v_axis = property(lambda self: self._fan.v_axis)


class SpectralBeamletSource:
    def __init__(self, spectrum, focal_point, centers, width_u, width_v,
                 u_axis=(1.0, 0.0, 0.0), v_axis=(0.0, 1.0, 0.0)) -> None:
        self._spectrum = spectrum
        self._fan = _Fan(tuple(focal_point), tuple(centers), width_u, width_v, u_axis, v_axis)

    max_energy = property(lambda self: self._spectrum.max_energy)
    n_beamlets = property(lambda self: len(self._fan.centers))
    spectrum = property(lambda self: self._spectrum)
    focal_point = property(lambda self: self._fan.focal_point)
    centers = property(lambda self: self._fan.centers)
    width_u = property(lambda self: self._fan.width_u)
    width_v = property(lambda self: self._fan.width_v)
    u_axis = property(lambda self: self._fan.u_axis)
    v_axis = property(lambda self: self._fan.v_axis)


class TransmissionMaskSource:
    """A source shaped by a 0..1 transmission mask on a plane rectangle
    (geometry/collimation.py:1205, the model :987-1080): each primary of
    ``inner`` carries the mask value where its full line crosses the plane as
    its weight; ``mask[i, j]`` is pixel i along ``u_axis`` and j along
    ``v_axis``.  The engine weights the primaries in-kernel when it generates
    ``inner`` there (pencil, parallel or spectral fan; pyRadMC's Warp engine
    does so for the spectral fan)."""

    def __init__(self, inner, *, mask, plane_center, width_u, width_v,
                 u_axis=(1.0, 0.0, 0.0), v_axis=(0.0, 1.0, 0.0)) -> None:
        values = np.array(mask, dtype=np.float64)
        if values.ndim != 2 or values.size == 0:
            raise ValueError(f"the mask must be a non-empty 2D array, got shape {values.shape}")
        if not np.all(np.isfinite(values)) or values.min() < 0.0 or values.max() > 1.0:
            raise ValueError("mask values must be finite and within 0..1")
        if width_u <= 0.0 or width_v <= 0.0:
            raise ValueError(f"widths must be positive, got {width_u}, {width_v}")
        u = _unit(u_axis, "u_axis")
        v = _unit(v_axis, "v_axis")
        if abs(u[0] * v[0] + u[1] * v[1] + u[2] * v[2]) > 1.0e-9:
            raise ValueError("u_axis and v_axis must be orthogonal")
        self._inner = inner
        self._mask = values
        self._center = tuple(float(c) for c in plane_center)
        self._widths = (float(width_u), float(width_v))
        self._axes = (u, v)

    inner = property(lambda self: self._inner)
    max_energy = property(lambda self: self._inner.max_energy)
    mask = property(lambda self: self._mask)
    plane_center = property(lambda self: self._center)
    width_u = property(lambda self: self._widths[0])
    width_v = property(lambda self: self._widths[1])
    u_axis = property(lambda self: self._axes[0])
    v_axis = property(lambda self: self._axes[1])


class TransmissionMaskBeamletSource(TransmissionMaskSource):
    """A beamlet source shaped by a 0..1 transmission mask
    (geometry/collimation.py:1264): every beamlet's primaries are weighted by
    the mask value where their rays cross its plane."""

    n_beamlets = property(lambda self: self._inner.n_beamlets)


def _unit(v, name: str) -> tuple[float, float, float]:
    n = math.sqrt(sum(float(c) * float(c) for c in v))
    if n <= 0.0:
        raise ValueError(f"{name} must be a nonzero vector")
    return (float(v[0]) / n, float(v[1]) / n, float(v[2]) / n)


def _selection_cdf(weights) -> np.ndarray:
    """Normalized cumulative mixture weights (geometry/source.py:192-202)."""
    w = np.asarray(weights, dtype=np.float64)
    if w.size == 0:
        raise ValueError("a composite source needs at least one component")
    if np.any(w < 0.0):
        raise ValueError("component weights must be non-negative")
    total = float(w.sum())
    if total <= 0.0:
        raise ValueError("component weights must sum to a positive value")
    return np.cumsum(w) / total


class CompositeBeamletSource:
    """A per-beamlet mixture of beamlet sources (geometry/source.py:239-277):
    every component describes the same beamlets, and beamlet ``j``'s primary
    comes from the first component whose cumulative weight reaches one uniform
    draw, then from that component's beamlet ``j``."""

    def __init__(self, components) -> None:
        if not components:
            raise ValueError("a composite beamlet source needs at least one component")
        self._sources = tuple(source for source, _ in components)
        counts = {source.n_beamlets for source in self._sources}
        if len(counts) != 1:
            raise ValueError(f"all components must share n_beamlets, got {sorted(counts)}")
        self._n_beamlets = counts.pop()
        self._cdf = _selection_cdf([weight for _, weight in components])
        self._max_energy = max(source.max_energy for source in self._sources)

    max_energy = property(lambda self: self._max_energy)
    n_beamlets = property(lambda self: self._n_beamlets)

    def emit(self, beamlet: int, rng_state):
        """One uniform picks the component, then it emits (only when the
        components are pyRadMC objects with ``emit``)."""
        from pyradmc.rng import uniform

        index = min(int(np.searchsorted(self._cdf, uniform(rng_state))), len(self._sources) - 1)
        return self._sources[index].emit(beamlet, rng_state)


class ConcatenatedBeamletSource:
    """Several beamlet sources as one Dij: the columns of ``sources[0]``, then
    those of ``sources[1]``, ...  A treatment plan of several beams (each its
    own focal spot and aperture axes) is one call, one set of persistent
    launches and one CSC, where pyRadMC would run one ``run_dij`` per beam and
    stack the matrices.  Beamlet ``j`` of the concatenation is beamlet
    ``j - first(part)`` of its part, with the history and stream mapping of the
    concatenated column index, so it also runs on pyRadMC's ReferenceEngine
    when the parts are pyRadMC sources (``emit`` dispatches)."""

    def __init__(self, sources) -> None:
        self._sources = tuple(sources)
        if not self._sources:
            raise ValueError("a concatenation needs at least one beamlet source")
        self._first = np.concatenate([[0], np.cumsum([int(s.n_beamlets) for s in self._sources])])

    sources = property(lambda self: self._sources)
    n_beamlets = property(lambda self: int(self._first[-1]))
    max_energy = property(lambda self: max(float(s.max_energy) for s in self._sources))

    def part_of(self, beamlet: int) -> tuple[int, int]:
        """(part index, beamlet index within the part) of a concatenated column."""
        if not 0 <= beamlet < self.n_beamlets:
            raise IndexError(f"beamlet {beamlet} outside a concatenation of {self.n_beamlets}")
        k = int(np.searchsorted(self._first, beamlet, side="right")) - 1
        return k, beamlet - int(self._first[k])

    def emit(self, beamlet: int, rng_state):
        k, j = self.part_of(beamlet)
        return self._sources[k].emit(j, rng_state)

    def sample_beamlet_batch(self, seed: int, history_offset: int, n: int, beamlet: int):
        k, j = self.part_of(beamlet)
        return self._sources[k].sample_beamlet_batch(seed, history_offset, n, j)


# ---- results ----------------------------------------------------------------------
@dataclass(frozen=True)
class RunProvenance:
    version: str
    backend: str
    device: str
    seed: int
    pcut_mev: float
    ecut_mev: float
    msc_model: str
    step_energy_fraction: float
    cross_sections: str
    deposit_resolution_cm: float | None = None

    def summary(self) -> str:
        return (
            f"pyradmc {self.version} {self.backend}/{self.device} seed={self.seed} "
            f"pcut={self.pcut_mev} ecut={self.ecut_mev} msc={self.msc_model} "
            f"step={self.step_energy_fraction} deposit_res={self.deposit_resolution_cm} "
            f"xs=[{self.cross_sections}]"
        )


@dataclass(frozen=True)
class TransportResult:
    dose: np.ndarray
    dose_sigma: np.ndarray
    energy_emitted: float
    energy_deposited: float
    energy_escaped: float
    n_histories: int
    n_batches: int
    energy_unscored: float = 0.0
    scoring_mode: str = "dose_to_medium"
    provenance: RunProvenance | None = None


@dataclass(frozen=True)
class DijResult:
    grid_shape: tuple[int, int, int]
    n_beamlets: int
    n_histories_per_beamlet: int
    n_batches: int
    truncation: float
    indptr: np.ndarray
    indices: np.ndarray
    dose: np.ndarray
    sigma: np.ndarray
    energy_emitted: float
    energy_deposited: float
    energy_escaped: float
    energy_unscored: float = 0.0
    correlated: bool = False
    scoring_mode: str = "dose_to_medium"
    provenance: RunProvenance | None = None

    @property
    def n_voxels(self) -> int:
        return int(np.prod(self.grid_shape))

    def _scatter(self, values: np.ndarray, beamlet: int) -> np.ndarray:
        if not 0 <= beamlet < self.n_beamlets:
            raise IndexError(f"beamlet {beamlet} outside 0..{self.n_beamlets - 1}")
        lo, hi = int(self.indptr[beamlet]), int(self.indptr[beamlet + 1])
        out = np.zeros(self.n_voxels, dtype=np.float64)
        out[self.indices[lo:hi]] = values[lo:hi]
        return out.reshape(self.grid_shape)

    def column_dense(self, beamlet: int) -> np.ndarray:
        return self._scatter(self.dose, beamlet)

    def sigma_dense(self, beamlet: int) -> np.ndarray:
        return self._scatter(self.sigma, beamlet)

    def dose_for_weights(self, weights: np.ndarray) -> np.ndarray:
        w = np.asarray(weights, dtype=np.float64)
        if w.shape != (self.n_beamlets,):
            raise ValueError(f"weights shape {w.shape} != ({self.n_beamlets},)")
        out = np.zeros(self.n_voxels, dtype=np.float64)
        for j in range(self.n_beamlets):
            lo, hi = int(self.indptr[j]), int(self.indptr[j + 1])
            np.add.at(out, self.indices[lo:hi], w[j] * self.dose[lo:hi])
        return out.reshape(self.grid_shape)

    def dose_csc(self, unit: str = "mev_per_g"):
        from scipy.sparse import csc_array

        if unit not in ("mev_per_g", "gy"):
            raise ValueError(f"unknown unit {unit!r}; expected 'mev_per_g' or 'gy'")
        factor = 1.0 if unit == "mev_per_g" else GY_PER_MEV_PER_G
        data = self.dose if factor == 1.0 else self.dose * factor
        return csc_array((data, self.indices, self.indptr), shape=(self.n_voxels, self.n_beamlets))


# ---- progress -----------------------------------------------------------------------
@dataclass(frozen=True)
class ProgressEvent:
    histories_done: int
    histories_total: int
    elapsed_s: float
    rate_hz: float


class ProgressEmitter:
    """Thread-safe progress ticks; a raising callback is logged and ignored."""

    def __init__(self, callback: Callable | None, histories_total: int) -> None:
        self._callback = callback
        self._total = histories_total
        self._done = 0
        self._lock = threading.Lock()
        self._start = time.monotonic()
        self._last_t = self._start

    def tick(self, histories: int) -> None:
        with self._lock:
            self._done += histories
            now = time.monotonic()
            dt = now - self._last_t
            rate = histories / dt if dt > 0 else 0.0
            self._last_t = now
            event = ProgressEvent(self._done, self._total, now - self._start, rate)
            logger.debug("progress: %d/%d histories (%.1f Hz)", event.histories_done,
                         event.histories_total, event.rate_hz)
            if self._callback is None:
                return
            try:
                self._callback(event)
            except Exception:
                logger.exception("Progress callback raised; ignoring.")


# ---- cross sections from the packs ----------------------------------------------------
def _energy_label(energy: float) -> str:
    return f"{energy:.4f}".rstrip("0").rstrip(".")


class AnalyticWaterTables:
    """The analytic water ``CrossSectionSource`` as flattened tables, from the packs.

    Same constructor as ``AnalyticCrossSections(geometry_densities=...)``
    (data/analytic.py:131): the Woodcock majorant is taken over the declared
    ``(material, max density)`` pairs.  For water the majorant is the declared
    maximum density times the unit-density majorant row of the pack (data/
    analytic.py:196-206: ``max(density * mu_total)``), which is what scaling the
    stored row does.  ``build_tables`` serves the pack whose ``e_max`` matches
    the request exactly; other energies need pyRadMC's own builder.
    """

    _cache: dict = {}
    _lock = threading.Lock()

    def __init__(self, geometry_densities=((WATER, 1.0),)) -> None:
        for material, density in geometry_densities:
            if material != WATER:
                raise ValueError(f"material index {material} beyond the analytic source (water only)")
            if density <= 0.0:
                raise ValueError(f"non-positive density {density} for material {material}")
        self._geometry_densities = tuple(geometry_densities)
        self._rho_max = max(d for _, d in geometry_densities)

    n_materials = 1
    provenance = (
        "analytic closed-form water (Klein-Nishina without binding, power-law "
        "photoelectric, fitted pair, Berger-Seltzer ICRU-37 stopping)"
    )

    @classmethod
    def available_energies(cls) -> list[float]:
        out = []
        for path in sorted(DATA.glob("water_tables_*.npz")):
            out.append(float(path.stem.split("_")[-1]))
        return out

    def _pack(self, e_max: float, ecut: float, pcut: float) -> dict:
        """The pack built for exactly `e_max`, else the smallest one whose
        energy range covers it (a source whose top energy is data, such as a
        phase space, rarely sits on a pack energy; wider tables interpolate the
        same physics on a log grid that reaches a little further)."""
        e_primary = e_max / (1.0 + 1.0e-6)
        path = DATA / f"water_tables_{_energy_label(e_primary)}.npz"
        if not path.exists():
            above = [e for e in self.available_energies() if e * (1.0 + 1.0e-6) >= e_max]
            if above:
                path = DATA / f"water_tables_{_energy_label(min(above))}.npz"
        with self._lock:
            cached = self._cache.get(path)
            if cached is None:
                if not path.exists():
                    raise ValueError(
                        f"no water table pack for e_max={e_max} MeV (packs: "
                        f"{self.available_energies()}); pass pyRadMC's AnalyticCrossSections "
                        "to build tables for other energies"
                    )
                with np.load(path) as z:
                    cached = {k: z[k] for k in z.files}
                self._cache[path] = cached
        if not (
            float(cached["e_max"]) >= e_max - 1e-12
            and float(cached["ecut"]) == ecut
            and float(cached["pcut"]) == pcut
        ):
            raise ValueError(
                f"the water table packs are built at ecut={float(cached['ecut'])}, "
                f"pcut={float(cached['pcut'])}, e_max={float(cached['e_max'])}; "
                f"requested ecut={ecut}, pcut={pcut}, e_max={e_max}"
            )
        return cached

    def build_tables(self, ecut: float, pcut: float, e_max: float, n_points=None):
        z = self._pack(e_max, ecut, pcut)
        fields = {k: v for k, v in z.items() if k != "provenance"}
        for k in ("n_points", "n_coherent"):
            fields[k] = int(fields[k])
        for k in ("ecut", "pcut", "e_max", "photon_log_e_min", "photon_inv_dlog",
                  "electron_log_e_min", "electron_inv_dlog", "range_log_r_min", "range_inv_dlog"):
            fields[k] = float(fields[k])
        # AnalyticCrossSections.majorant (data/analytic.py:198-206) times the
        # node headroom (data/tables.py:73, :272), in the reference's operation
        # order: rho * ((compton + photoelectric) + pair), then * headroom.
        mu_total = (np.asarray(z["mu_compton"][0]) + np.asarray(z["mu_photo"][0])) + np.asarray(z["mu_pair"][0])
        fields["majorant"] = (self._rho_max * mu_total) * MAJORANT_HEADROOM
        return SimpleNamespace(**fields)

    def gs_grid_for(self, tables, materials: Sequence[int]):
        """The GS node grid covering the window the kernels can reach.

        The window is ``gs_window_from_tables`` (data/goudsmit_saunderson.py:
        1222) restated; the packed grid is uploaded whole when it covers it, as
        pyRadMC's own cached grid is (build_gs_grid returns a covering stored
        grid as is, :1181-1196).
        """
        return gs_grid_from_pack(tables, materials)


_gs_pack = None


def gs_window(tables, materials) -> tuple[float, float, float]:
    rows = np.asarray(sorted({int(m) for m in materials}), dtype=int)
    if rows.size == 0:
        raise ValueError("no materials given; the window would be empty")
    log_eta = np.asarray(tables.log_eta)[rows]
    ceiling = float(np.max(np.asarray(tables.scattering_power)[rows].max(axis=1)
                           * np.asarray(tables.restricted_range)[rows].max(axis=1)))
    return float(log_eta.min()), float(log_eta.max()), ceiling


def gs_grid_from_pack(tables, materials):
    global _gs_pack
    if _gs_pack is None:
        with np.load(DATA / "water_gs_grid.npz") as z:
            _gs_pack = SimpleNamespace(values=np.ascontiguousarray(z["values"], dtype=np.float32),
                                       ix0=int(z["ix0"]), iy0=int(z["iy0"]), n_u=int(z["n_u"]),
                                       bins_per_log=float(z["bins_per_log"]))
    lo, hi, t2 = gs_window(tables, materials)
    bins = _gs_pack.bins_per_log
    ix0, ix_top = math.floor(lo * bins), math.floor(hi * bins) + 1
    iy0, iy_top = math.floor(math.log(1.0e-12) * bins), math.floor(math.log(t2) * bins) + 1
    g = _gs_pack
    covered = (g.ix0 <= ix0 and ix_top < g.ix0 + g.values.shape[0]
               and g.iy0 <= iy0 and iy_top < g.iy0 + g.values.shape[1])
    if not covered:
        raise ValueError("the packed Goudsmit-Saunderson grid does not cover this run's window; "
                         "use pyRadMC's build_gs_grid")
    return g


# ---- any cross-section source, packed ---------------------------------------------
PACK_TABLE_FIELDS = ("mu_compton", "mu_photo", "mu_pair", "mu_rayleigh", "majorant",
                     "stopping_restricted", "stopping_radiative", "moller", "csda_range",
                     "scattering_power", "log_eta", "restricted_range",
                     "energy_of_restricted_range", "coherent_x", "coherent_cumulative")
PACK_TABLE_SCALARS = ("n_points", "ecut", "pcut", "e_max", "photon_log_e_min", "photon_inv_dlog",
                      "electron_log_e_min", "electron_inv_dlog", "range_log_r_min",
                      "range_inv_dlog", "n_coherent")


def save_pack(cross_sections, path, *, ecut: float, pcut: float, e_max: float,
              materials: Sequence[int]) -> None:
    """Write one ``CrossSectionSource``'s flattened tables
    (``build_tables(ecut, pcut, e_max)``, data/interface.py:413) and the
    Goudsmit-Saunderson node grid of the window its `materials` reach
    (``build_gs_grid(*gs_window_from_tables(tables, materials))``,
    data/goudsmit_saunderson.py:1108, :1222) to `path`, for
    :class:`PackedCrossSections`.  Needs pyRadMC; `e_max` is the table edge
    (the primary energy times the engine's 1 + 1e-6 margin)."""
    from pyradmc.data.goudsmit_saunderson import build_gs_grid, gs_window_from_tables

    tab = cross_sections.build_tables(ecut=ecut, pcut=pcut, e_max=e_max)
    gs = build_gs_grid(*gs_window_from_tables(tab, list(materials)))
    payload = {name: np.asarray(getattr(tab, name), dtype=np.float64) for name in PACK_TABLE_FIELDS}
    payload.update({name: np.asarray(getattr(tab, name)) for name in PACK_TABLE_SCALARS})
    payload.update(gs_values=np.asarray(gs.values, dtype=np.float32), gs_ix0=np.int64(gs.ix0),
                   gs_iy0=np.int64(gs.iy0), gs_n_u=np.int64(gs.n_u),
                   gs_bins_per_log=np.float64(gs.bins_per_log),
                   gs_materials=np.asarray(sorted({int(m) for m in materials}), dtype=np.int64),
                   n_materials=np.int64(cross_sections.n_materials),
                   provenance=np.asarray(str(getattr(cross_sections, "provenance",
                                                     type(cross_sections).__name__))))
    np.savez_compressed(path, **payload)


class PackedCrossSections:
    """A ``CrossSectionSource`` for the B200 engine from a :func:`save_pack`
    file: the flattened tables of any number of materials and the GS node grid
    they need, built where pyRadMC (and its data, such as the EPICS libraries
    of ``TabulatedCrossSections``) is available and used where it is not.

    ``build_tables`` serves the packed tables for exactly the packed
    (ecut, pcut, e_max); ``gs_grid_for`` serves the packed grid when it covers
    the requested materials' window, and raises otherwise."""

    def __init__(self, path) -> None:
        with np.load(path) as z:
            data = {k: z[k] for k in z.files}
        self._fields = {k: data[k] for k in PACK_TABLE_FIELDS}
        for k in ("n_points", "n_coherent"):
            self._fields[k] = int(data[k])
        for k in PACK_TABLE_SCALARS:
            if k not in ("n_points", "n_coherent"):
                self._fields[k] = float(data[k])
        self._gs = SimpleNamespace(values=np.ascontiguousarray(data["gs_values"], dtype=np.float32),
                                   ix0=int(data["gs_ix0"]), iy0=int(data["gs_iy0"]),
                                   n_u=int(data["gs_n_u"]), bins_per_log=float(data["gs_bins_per_log"]))
        self._gs_materials = {int(m) for m in data["gs_materials"]}
        self.n_materials = int(data["n_materials"])
        self.provenance = str(data["provenance"])

    def build_tables(self, ecut: float, pcut: float, e_max: float, n_points=None):
        f = self._fields
        if not (math.isclose(f["e_max"], e_max, rel_tol=0, abs_tol=1e-12)
                and f["ecut"] == ecut and f["pcut"] == pcut
                and (n_points is None or n_points == f["n_points"])):
            raise ValueError(
                f"this pack holds tables at ecut={f['ecut']}, pcut={f['pcut']}, e_max={f['e_max']}; "
                f"requested ecut={ecut}, pcut={pcut}, e_max={e_max}")
        return SimpleNamespace(**f)

    def gs_grid_for(self, tables, materials: Sequence[int]):
        wanted = {int(m) for m in materials}
        if not wanted <= self._gs_materials:
            raise ValueError(f"the packed GS grid covers materials {sorted(self._gs_materials)}, "
                             f"not {sorted(wanted)}")
        return self._gs
