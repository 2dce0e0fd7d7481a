"""Treatment-head pre-solve on the GPU: the drop-in for pyRadMC's
``presolve_head_device`` (backends/warp/presolve.py:572-687), the device twin of
the host ``presolve_head`` (geometry/head.py:373-575).

Primaries are sampled on the host (``source.sample_batch``), traced through the
beam-limiting stack and an optional air column by ``pmc_presolve_head`` (one
GPU thread per primary; the physics and its stated approximations are those of
geometry/head.py: a forced first Compton in the stack and in the air, Beer-
Lambert transmission, roulette of secondaries below ``weight_floor``), and the
exit-plane particles come back as an :class:`InMemoryPhaseSpaceSource` with
every weight scaled by (particles kept / primaries), as ``_Population.build``
(head.py:296-314) normalizes them — a phase space the engine then transports
like any other.  The random streams are this backend's own, so a result agrees
with the host oracle in distribution, never bit for bit (as pyRadMC's device
twin).

The stack is pyRadMC's ``BeamLimitingStack`` (its ``flatten()`` gives the
column-parallel arrays, collimation.py:871-903) or a :class:`CompiledHeadStack`
holding the same arrays; the attenuation tables come from the cross-section
source's ``mu_over_rho_total`` / ``mu_over_rho`` (head.py:119-180) or are
passed ready-made as :class:`HeadMuTables`.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .engine import ECUT_MEV, PCUT_MEV
from .phasespace import InMemoryPhaseSpaceSource

PHOTON, ELECTRON = 1, 2  # IAEA particle codes (geometry/phasespace.py)
COMPTON = 0              # PhotonProcess.COMPTON (data/interface.py:74)
MODES = ("auto", "first_compton", "attenuation")


AIR = 1  # the registry's air (data/materials.py:151)


@dataclass(frozen=True)
class AirColumn:
    """The air gap z_start <= w <= z_end (beam frame, cm) below the stack, with
    its material index and density in g/cm^3 (head.py:97-116; the same
    defaults and validation)."""

    z_start: float
    z_end: float
    material: int = AIR
    density: float = 1.205e-3

    def __post_init__(self) -> None:
        if not 0.0 < self.z_start < self.z_end:
            raise ValueError(f"need 0 < z_start < z_end, got {self.z_start}, {self.z_end}")
        if self.density <= 0.0:
            raise ValueError(f"density must be positive, got {self.density}")


@dataclass
class CompiledHeadStack:
    """The beam-limiting stack as flat arrays (the fields of pyRadMC's
    CompiledStack, collimation.py:871-903) with each device's material and
    density."""

    origin: np.ndarray
    rotation: np.ndarray
    kind: np.ndarray
    z_top: np.ndarray
    z_bottom: np.ndarray
    jaw_axis: np.ndarray
    jaw_edge_neg: np.ndarray
    jaw_edge_pos: np.ndarray
    jaw_focused: np.ndarray
    mlc_tip_radius: np.ndarray
    mlc_focused_sides: np.ndarray
    mlc_n_pairs: np.ndarray
    mlc_edges_off: np.ndarray
    mlc_tips_off: np.ndarray
    leaf_edges_v: np.ndarray
    tips_neg: np.ndarray
    tips_pos: np.ndarray
    materials: tuple = ()
    densities: tuple = ()
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_devices(self) -> int:
        return int(np.asarray(self.kind).size)

    @property
    def exit_z(self) -> float:
        return float(np.asarray(self.z_bottom)[-1])

    @classmethod
    def from_stack(cls, stack) -> "CompiledHeadStack":
        """From pyRadMC's BeamLimitingStack (or anything with ``flatten()``,
        ``materials`` and ``densities``)."""
        c = stack.flatten()
        names = [f for f in cls.__dataclass_fields__ if f not in ("materials", "densities", "_keep")]
        return cls(**{n: np.asarray(getattr(c, n)) for n in names},
                   materials=tuple(int(m) for m in stack.materials),
                   densities=tuple(float(d) for d in stack.densities))

    def to_c(self) -> _lib.HeadStack:
        """The C-ABI descriptor; the arrays it points into stay alive with self."""
        d = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        i = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        arr = {n: (i if n in ("kind", "jaw_axis", "jaw_focused", "mlc_focused_sides", "mlc_n_pairs",
                              "mlc_edges_off", "mlc_tips_off") else d)(getattr(self, n))
               for n in ("kind", "z_top", "z_bottom", "jaw_axis", "jaw_edge_neg", "jaw_edge_pos",
                         "jaw_focused", "mlc_tip_radius", "mlc_focused_sides", "mlc_n_pairs",
                         "mlc_edges_off", "mlc_tips_off", "leaf_edges_v", "tips_neg", "tips_pos")}
        self._keep = list(arr.values())
        s = _lib.HeadStack(n_devices=self.n_devices)
        s.origin[:] = [float(v) for v in np.asarray(self.origin).reshape(3)]
        s.rotation[:] = [float(v) for v in np.asarray(self.rotation).reshape(9)]
        for n, a in arr.items():
            setattr(s, n, _lib.ptr(a, C.c_int32 if a.dtype == np.int32 else C.c_double))
        s.n_leaf_edges = int(arr["leaf_edges_v"].size)
        s.n_tips = int(arr["tips_pos"].size)
        return s


@dataclass
class HeadMuTables:
    """Macroscopic attenuation (1/cm) per row — the stack's devices, then the
    air column — as log-log tables on a log-uniform energy grid (head.py:119-180)."""

    log_energy: np.ndarray   # [n_table]
    log_total: np.ndarray    # [rows][n_table]
    log_compton: np.ndarray  # [rows][n_table]

    @classmethod
    def build(cls, cross_sections, pairs, e_min: float, e_max: float, n_table: int) -> "HeadMuTables":
        """From a cross-section source's mass attenuation coefficients for each
        (material, density) pair, at n_table energies from e_min to e_max."""
        if max(m for m, _ in pairs) >= cross_sections.n_materials:
            raise ValueError("a device or air material index is beyond this cross-section source")
        energies = np.geomspace(e_min, max(e_max, e_min * (1.0 + 1e-9)), n_table)
        total = np.array([[rho * cross_sections.mu_over_rho_total(float(e), m) for e in energies]
                          for m, rho in pairs])
        compton = np.array([[rho * cross_sections.mu_over_rho(float(e), m, COMPTON) for e in energies]
                            for m, rho in pairs])
        return cls(np.log(energies), np.log(total), np.log(np.maximum(compton, 1e-300)))

    def to_c(self):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (self.log_energy, self.log_total,
                                                                     self.log_compton)]
        mu = _lib.HeadMu(n_rows=int(arrs[1].shape[0]), n_table=int(arrs[0].size),
                         log_energy=_lib.ptr(arrs[0], C.c_double), log_total=_lib.ptr(arrs[1], C.c_double),
                         log_compton=_lib.ptr(arrs[2], C.c_double))
        return mu, arrs


def resolve_presolve(stack, air, exit_z: float, mode: str) -> str:
    """The mode (``auto`` -> ``first_compton``) after head.py:340-370's checks:
    a known mode, exit_z at or below the stack's exit face and the air column's
    end, the air column below the stack."""
    if mode not in MODES:
        raise ValueError(f"mode must be one of {MODES}, got {mode!r}")
    if stack is None:
        raise ValueError("the device pre-solve requires a stack; use presolve_head on the host")
    if exit_z < stack.exit_z:
        raise ValueError(f"exit_z {exit_z} is above the stack exit {stack.exit_z}")
    if air is not None:
        if air.z_start < stack.exit_z:
            raise ValueError(f"the air column starts at {air.z_start}, inside the stack (exit {stack.exit_z})")
        if exit_z < air.z_end:
            raise ValueError(f"exit_z {exit_z} is above the air column end {air.z_end}")
    return "first_compton" if mode == "auto" else mode


class DevicePhaseSpace:
    """A pre-solve's exit-plane phase space kept on its GPU (the analogue of
    pyRadMC's DevicePhaseSpace, backends/warp/presolve.py:710): torch tensors
    particle_type (IAEA codes, int32), energy, pos [n, 3], dir [n, 3] and
    weight (float32), already normalized per original primary.  B200Engine.run
    transports it without a copy to the host; ``columns()`` copies it back."""

    def __init__(self, particle_type, energy, pos, dirs, weight, max_energy: float):
        self.particle_type, self.energy, self.pos, self.dir, self.weight = (
            particle_type, energy, pos, dirs, weight)
        self.max_energy = float(max_energy)
        self.device = str(energy.device)

    def __len__(self) -> int:
        return int(self.energy.shape[0])

    def columns(self) -> dict:
        pos, d = self.pos.cpu().numpy().astype(np.float64), self.dir.cpu().numpy().astype(np.float64)
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        return {"particle_type": self.particle_type.cpu().numpy(), "energy": self.energy.cpu().numpy().astype(np.float64),
                "x": pos[:, 0], "y": pos[:, 1], "z": pos[:, 2], "ux": d[:, 0], "uy": d[:, 1], "uz": d[:, 2],
                "weight": self.weight.cpu().numpy().astype(np.float64)}

    def to_phase_space(self) -> InMemoryPhaseSpaceSource:
        return InMemoryPhaseSpaceSource(**self.columns())


def presolve_head_device(source, *, cross_sections=None, n_histories: int, seed: int, exit_z: float,
                         stack, air: AirColumn | None = None, mode: str = "auto",
                         device: str = "cuda:0", pcut: float = PCUT_MEV, ecut: float = ECUT_MEV,
                         weight_floor: float = 1.0e-3, e_min: float = 0.010, n_table: int = 512,
                         mu_tables: HeadMuTables | None = None, return_device_source: bool = False,
                         return_dropped: bool = False):
    """Pre-solve the head on the GPU and return the exit-plane phase space
    (presolve.py:572-687's arguments and contract; ``device`` selects the
    CUDA device).  ``return_device_source`` keeps the population on the device
    as a :class:`DevicePhaseSpace` that the engine transports with no copy
    back (the reference's return_device_source).  ``mu_tables`` replaces the
    tables built from ``cross_sections``; ``return_dropped`` also returns the
    dropped weight x energy (MeV)."""
    import torch

    compiled = stack if isinstance(stack, CompiledHeadStack) else (
        None if stack is None else CompiledHeadStack.from_stack(stack))
    resolved = resolve_presolve(compiled, air, exit_z, mode)
    columns = source.sample_batch(seed, 0, n_histories)
    if not np.all(np.asarray(columns["particle_type"]) == PHOTON):
        raise ValueError("the pre-solve transports photon sources only")
    pairs = tuple(zip(compiled.materials, compiled.densities, strict=True))
    air_row = len(pairs)
    if air is not None:
        pairs = (*pairs, (air.material, air.density))
    if mu_tables is None:
        if cross_sections is None:
            raise ValueError("pass cross_sections (or ready-made mu_tables)")
        mu_tables = HeadMuTables.build(cross_sections, pairs, e_min, float(source.max_energy), n_table)
    if np.asarray(mu_tables.log_total).shape[0] < len(pairs):
        raise ValueError(f"the mu tables have {np.asarray(mu_tables.log_total).shape[0]} rows, need {len(pairs)}")

    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)  # noqa: E731
    n = int(n_histories)
    energy = f32(columns["energy"])
    pos = f32(np.stack([columns["x"], columns["y"], columns["z"]], axis=1))
    dirs = f32(np.stack([columns["ux"], columns["uy"], columns["uz"]], axis=1))
    weight = f32(columns["weight"])
    fc = 1 if resolved == "first_compton" else 0
    capacity = n * (1 + fc * (1 + 2 * (air is not None)))
    if return_device_source:  # the compaction writes straight into these device tensors
        dev = torch.device(device)
        t_kind = torch.empty(capacity, dtype=torch.int32, device=dev)
        t_e = torch.empty(capacity, dtype=torch.float32, device=dev)
        t_p = torch.empty((capacity, 3), dtype=torch.float32, device=dev)
        t_d = torch.empty((capacity, 3), dtype=torch.float32, device=dev)
        t_w = torch.empty(capacity, dtype=torch.float32, device=dev)
        as_ptr = lambda t, ct: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ct))  # noqa: E731
        outs = (as_ptr(t_kind, C.c_int32), as_ptr(t_e, C.c_float), as_ptr(t_p, C.c_float),
                as_ptr(t_d, C.c_float), as_ptr(t_w, C.c_float))
    else:
        out_kind = np.empty(capacity, dtype=np.int32)
        out_e = np.empty(capacity, dtype=np.float32)
        out_p = np.empty((capacity, 3), dtype=np.float32)
        out_d = np.empty((capacity, 3), dtype=np.float32)
        out_w = np.empty(capacity, dtype=np.float32)
        outs = (_lib.ptr(out_kind, C.c_int32), _lib.ptr(out_e, C.c_float), _lib.ptr(out_p, C.c_float),
                _lib.ptr(out_d, C.c_float), _lib.ptr(out_w, C.c_float))
    cs = compiled.to_c()
    mu, keep = mu_tables.to_c()
    params = _lib.HeadParams(first_compton=fc, has_air=int(air is not None), air_row=air_row,
                             air_z_start=float(air.z_start) if air else 0.0,
                             air_z_end=float(air.z_end) if air else 0.0, exit_z=float(exit_z),
                             pcut=float(pcut), ecut=float(ecut), weight_floor=float(weight_floor),
                             seed=int(seed) & 0xFFFFFFFFFFFFFFFF,
                             outputs_on_device=int(bool(return_device_source)))
    count, dropped = C.c_int64(), C.c_double()
    lib = _lib.load()
    with torch.cuda.device(torch.device(device)):
        code = lib.pmc_presolve_head(C.byref(cs), C.byref(mu), C.byref(params), n,
                                     _lib.ptr(energy, C.c_float), _lib.ptr(pos, C.c_float),
                                     _lib.ptr(dirs, C.c_float), _lib.ptr(weight, C.c_float), capacity,
                                     *outs, C.byref(count), C.byref(dropped))
    del keep
    if code != _lib.PMC_OK:
        raise RuntimeError(f"pmc_presolve_head failed ({code})")
    k = int(count.value)
    if k == 0:
        raise ValueError("the pre-solve kept no particles; check the geometry and cutoffs")
    if return_device_source:
        # the host path's arithmetic on the device: directions renormalized
        # and weights scaled per original primary (head.py:296-314) in
        # float64, then rounded to float32 as the engine's upload rounds them,
        # so both hand-offs carry the same records bit for bit
        d64 = t_d[:k].double()
        n2 = (d64[:, 0] * d64[:, 0] + d64[:, 1] * d64[:, 1]) + d64[:, 2] * d64[:, 2]
        dps = DevicePhaseSpace(t_kind[:k].clone(), t_e[:k].clone(), t_p[:k].clone(),
                               (d64 / torch.sqrt(n2).unsqueeze(1)).float(),
                               (t_w[:k].double() * (k / n)).float(), float(source.max_energy))
        return (dps, float(dropped.value)) if return_dropped else dps
    d = out_d[:k].astype(np.float64)
    d /= np.linalg.norm(d, axis=1, keepdims=True)  # float32 round-off
    ps = InMemoryPhaseSpaceSource(
        particle_type=out_kind[:k].copy(), energy=out_e[:k].astype(np.float64),
        x=out_p[:k, 0].astype(np.float64), y=out_p[:k, 1].astype(np.float64),
        z=out_p[:k, 2].astype(np.float64), ux=d[:, 0], uy=d[:, 1], uz=d[:, 2],
        # normalized per original primary (head.py:296-314)
        weight=out_w[:k].astype(np.float64) * (k / n))
    return (ps, float(dropped.value)) if return_dropped else ps


def stack_path_lengths(stack, points, directions, from_origin: bool = False) -> np.ndarray:
    """Chord lengths (cm) of engine-frame rays through each device of the stack,
    computed on the GPU (float32): [n, n_devices], the device twin of
    BeamLimitingStack.path_lengths (collimation.py)."""
    compiled = stack if isinstance(stack, CompiledHeadStack) else CompiledHeadStack.from_stack(stack)
    p = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
    out = np.empty((p.shape[0], compiled.n_devices), dtype=np.float32)
    cs = compiled.to_c()
    code = _lib.load().pmc_head_path_lengths(C.byref(cs), p.shape[0], _lib.ptr(p, C.c_float),
                                             _lib.ptr(d, C.c_float), int(bool(from_origin)),
                                             _lib.ptr(out, C.c_float))
    if code != _lib.PMC_OK:
        raise RuntimeError(f"pmc_head_path_lengths failed ({code})")
    return out
