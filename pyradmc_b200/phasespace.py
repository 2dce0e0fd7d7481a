"""IAEA phase-space files and phase-space sources for the B200 engine.

The two-file IAEA format (Capote et al., *Phase-space database for external
beam radiotherapy*, IAEA(NDS)-0484, 2006): an ASCII ``.IAEAheader`` naming the
record layout and a binary ``.IAEAphsp`` of fixed-length records -- an int8
particle code whose sign is the sign of the third direction cosine ``w``, a
float32 energy whose sign flags a new primary history, then the float32
coordinates the header marks as stored (x, y, z, u, v, weight; the others are
header constants), then any extra floats and ints.  ``w`` is never stored:
``w = sign * sqrt(1 - u^2 - v^2)``.

pyRadMC reads the format in ``geometry/phasespace.py`` (header :141, records
:291, ``PhaseSpaceSource`` :428, ``InMemoryPhaseSpaceSource`` :654); this module
restates that reading, vectorized, so phase spaces run where pyRadMC is not
installed, and adds :func:`write_iaea`.  The sources offer both routes the
engine knows: ``sample_batch`` (host pre-sampling with pyRadMC's chunk-invariant
PCG64 index stream, geometry/phasespace.py:377) and ``columns`` -- the whole
phase space, which :class:`~pyradmc_b200.engine.B200Engine` keeps resident on
the device and samples in-kernel, one record per history from the history's
own counter-based stream (the contract of ``PhaseSpaceSource.emit``, :546).
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass
from pathlib import Path

import numpy as np

__all__ = ["IAEA_ELECTRON", "IAEA_PHOTON", "IAEA_POSITRON", "IAEAHeader", "InMemoryPhaseSpaceSource",
           "PhaseSpaceSource", "load_iaea", "read_iaea_header", "write_iaea"]

IAEA_PHOTON, IAEA_ELECTRON, IAEA_POSITRON = 1, 2, 3
ELECTRON_MASS_MEV = 0.51099895069
COORDS = ("x", "y", "z", "u", "v", "weight")  # the storable coordinates, in file order
HEADER_EXT, PHSP_EXT = ".IAEAheader", ".IAEAphsp"


@dataclass(frozen=True)
class IAEAHeader:
    byte_order: str              # "<" ($BYTE_ORDER 1234) or ">" (4321)
    record_length: int
    n_particles: int
    n_extra_floats: int
    n_extra_ints: int
    stored: tuple[bool, ...]     # per COORDS
    constants: dict


def _paths(path) -> tuple[Path, Path]:
    p = Path(path)
    stem = p.with_suffix("") if p.suffix in (HEADER_EXT, PHSP_EXT) else p
    return stem.with_suffix(HEADER_EXT), stem.with_suffix(PHSP_EXT)


def _sections(text: str) -> dict[str, list[str]]:
    out: dict[str, list[str]] = {}
    key = None
    for raw in text.splitlines():
        line = raw.strip()
        if line.startswith("$") and line.endswith(":"):
            key = line[1:-1]
            out[key] = []
        elif key is not None:
            value = line.split("//", 1)[0].strip()
            if value:
                out[key].append(value)
    return out


def read_iaea_header(path) -> IAEAHeader:
    """Parse and check a ``.IAEAheader`` (geometry/phasespace.py:141-246)."""
    header_path, phsp_path = _paths(path)
    sec = _sections(header_path.read_text())
    contents = sec.get("RECORD_CONTENTS", [])
    if len(contents) < 9:
        raise ValueError(f"RECORD_CONTENTS needs 7 flags plus Nf and Ni, got {len(contents)} entries")
    flags = [int(t) for t in contents[:7]]
    n_f, n_i = int(contents[7]), int(contents[8])
    if flags[5] != 1:
        raise ValueError("w must be stored (RECORD_CONTENTS flag 6 = 1); w is reconstructed, never a constant")
    stored = tuple(bool(flags[i]) for i in (0, 1, 2, 3, 4, 6))
    values = [float(t) for t in sec.get("RECORD_CONSTANT", [])]
    if len(values) != sum(not s for s in stored):
        raise ValueError(f"RECORD_CONSTANT has {len(values)} values but "
                         f"{sum(not s for s in stored)} coordinates are constant")
    it = iter(values)
    constants = {c: next(it) for c, s in zip(COORDS, stored, strict=True) if not s}
    order_tok = (sec.get("BYTE_ORDER") or ["1234"])[0]
    if order_tok not in ("1234", "4321"):
        raise ValueError(f"unknown BYTE_ORDER {order_tok!r}; expected 1234 or 4321")
    order = "<" if order_tok == "1234" else ">"
    length = 1 + 4 + 4 * sum(stored) + 4 * n_f + 4 * n_i
    declared = sec.get("RECORD_LENGTH")
    if declared and int(declared[0]) != length:
        raise ValueError(f"RECORD_LENGTH {declared[0]} disagrees with the {length} bytes "
                         "implied by RECORD_CONTENTS")
    n_declared = int(sec["PARTICLES"][0]) if sec.get("PARTICLES") else None
    if phsp_path.exists():
        size = phsp_path.stat().st_size
        if size % length:
            raise ValueError(f"{phsp_path.name} size {size} is not a multiple of record length {length}")
        n = size // length
        if n_declared is not None and n_declared != n:
            warnings.warn(f"PARTICLES header says {n_declared} but {phsp_path.name} holds {n} "
                          "records; using the on-disk count", stacklevel=2)
    elif n_declared is None:
        raise ValueError("cannot determine particle count: no PARTICLES and no phsp file")
    else:
        n = n_declared
    return IAEAHeader(order, length, n, n_f, n_i, stored, constants)


def _dtype(h: IAEAHeader) -> np.dtype:
    names, formats, offsets, off = ["typ", "e"], [np.int8, h.byte_order + "f4"], [0, 1], 5
    for c, s in zip(COORDS, h.stored, strict=True):
        if s:
            names.append(c)
            formats.append(h.byte_order + "f4")
            offsets.append(off)
            off += 4
    return np.dtype({"names": names, "formats": formats, "offsets": offsets,
                     "itemsize": h.record_length})


def _decode(recs: np.ndarray, h: IAEAHeader) -> dict[str, np.ndarray]:
    """Column arrays of decoded records (geometry/phasespace.py:291 and :569)."""
    n = recs.shape[0]
    typ = recs["typ"].astype(np.int32)

    def col(name):
        if name in recs.dtype.names:
            return np.asarray(recs[name], dtype=np.float32)
        return np.full(n, h.constants[name], dtype=np.float32)

    u, v = col("u"), col("v")
    tmp = u.astype(np.float64) ** 2 + v.astype(np.float64) ** 2
    sign = np.where(typ < 0, -1.0, 1.0)
    w = np.where(tmp <= 1.0, sign * np.sqrt(np.maximum(0.0, 1.0 - tmp)), 0.0).astype(np.float32)
    over = tmp > 1.0
    if over.any():  # a degenerate direction: u, v renormalized, w = 0
        scale = np.sqrt(tmp[over]).astype(np.float32)
        u, v = u.copy(), v.copy()
        u[over] /= scale
        v[over] /= scale
    return {"particle_type": np.abs(typ), "energy": np.abs(recs["e"].astype(np.float32)),
            "x": col("x"), "y": col("y"), "z": col("z"), "ux": u, "uy": v, "uz": w,
            "weight": col("weight"), "new_history": recs["e"] < 0}


def load_iaea(path, *, skip_unsupported: bool = True) -> dict[str, np.ndarray]:
    """Every transportable record of an IAEA phase space as column arrays;
    records of other particles (IAEA codes 4, 5) are dropped with a warning, or
    refused with ``skip_unsupported=False`` (geometry/phasespace.py:458-513)."""
    h = read_iaea_header(path)
    _, phsp = _paths(path)
    recs = np.fromfile(phsp, dtype=_dtype(h), count=h.n_particles)
    cols = _decode(recs, h)
    ok = np.isin(cols["particle_type"], (IAEA_PHOTON, IAEA_ELECTRON, IAEA_POSITRON))
    if not ok.all():
        if not skip_unsupported:
            raise ValueError(f"unsupported particle type {int(cols['particle_type'][~ok][0])} in "
                             f"{path}; this photon MC transports only photons, electrons and "
                             "positrons (pass skip_unsupported=True to drop them)")
        warnings.warn(f"{int((~ok).sum())} of {ok.size} records in {Path(phsp).name} are "
                      "unsupported particle types (not photon/electron/positron); "
                      "dropping them from the sampled population", stacklevel=2)
        cols = {k: v[ok] for k, v in cols.items()}
    if cols["energy"].size == 0:
        raise ValueError(f"phase-space file {path} has no transportable particles")
    return cols


def write_iaea(stem, columns: dict, *, byte_order: str = "<", store_all: bool = True) -> Path:
    """Write column arrays (particle_type, energy, x, y, z, ux, uy, uz, weight,
    optional new_history) as an IAEA phase space ``stem.IAEAheader`` +
    ``stem.IAEAphsp``; returns the header path.  With ``store_all`` False, a
    coordinate that is constant over the records becomes a header constant."""
    n = int(np.asarray(columns["energy"]).size)
    cols = {"x": columns["x"], "y": columns["y"], "z": columns["z"], "u": columns["ux"],
            "v": columns["uy"], "weight": columns["weight"]}
    stored = []
    constants = []
    for c in COORDS:
        a = np.asarray(cols[c], dtype=np.float32)
        if store_all or not np.all(a == a[0]):
            stored.append(True)
        else:
            stored.append(False)
            constants.append(float(a[0]))
    h = IAEAHeader(byte_order, 5 + 4 * sum(stored), n, 0, 0, tuple(stored), {})
    recs = np.zeros(n, dtype=_dtype(h))
    uz = np.asarray(columns["uz"], dtype=np.float32)
    code = np.asarray(columns["particle_type"], dtype=np.int8)
    recs["typ"] = np.where(uz < 0, -code, code)
    new = np.asarray(columns.get("new_history", np.ones(n, bool)))
    e = np.asarray(columns["energy"], dtype=np.float32)
    recs["e"] = np.where(new, -e, e)
    for c, s in zip(COORDS, stored, strict=True):
        if s:
            recs[c] = np.asarray(cols[c], dtype=np.float32)
    header_path, phsp_path = _paths(stem)
    recs.tofile(phsp_path)
    flags = [int(stored[0]), int(stored[1]), int(stored[2]), int(stored[3]), int(stored[4]), 1,
             int(stored[5])]
    lines = ["$IAEA_INDEX:", "0", "$TITLE:", "pyradmc_b200 phase space", "$FILE_TYPE:", "0",
             "$RECORD_CONTENTS:", *[str(f) for f in flags], "0", "0",
             "$RECORD_CONSTANT:", *[f"{c:.9g}" for c in constants],
             "$RECORD_LENGTH:", str(h.record_length),
             "$BYTE_ORDER:", "1234" if byte_order == "<" else "4321",
             "$PARTICLES:", str(n), ""]
    header_path.write_text("\n".join(lines))
    return header_path


def sample_indices(seed: int, history_offset: int, n: int, n_valid: int) -> np.ndarray:
    """Chunk-invariant record indices of histories [offset, offset + n): one
    PCG64(seed) stream advanced to the offset (geometry/phasespace.py:377)."""
    bitgen = np.random.PCG64(seed)
    bitgen.advance(history_offset)
    k = (np.random.Generator(bitgen).random(n) * n_valid).astype(np.int64)
    np.clip(k, 0, n_valid - 1, out=k)
    return k


class InMemoryPhaseSpaceSource:
    """A phase space held as column arrays (geometry/phasespace.py:654-769):
    the same constructor, checks and ``columns()``; particle_type uses the IAEA
    codes 1 (photon), 2 (electron), 3 (positron)."""

    def __init__(self, particle_type, energy, x, y, z, ux, uy, uz, weight) -> None:
        codes = np.asarray(particle_type, dtype=np.int32)
        if codes.size == 0:
            raise ValueError("an in-memory phase space needs at least one particle")
        arrays = {name: np.asarray(col, dtype=np.float64) for name, col in
                  (("energy", energy), ("x", x), ("y", y), ("z", z), ("ux", ux), ("uy", uy),
                   ("uz", uz), ("weight", weight))}
        for name, col in arrays.items():
            if col.shape != codes.shape:
                raise ValueError(f"column {name!r} length {col.shape} != particle_type length {codes.shape}")
        if not np.all(np.isin(codes, (IAEA_PHOTON, IAEA_ELECTRON, IAEA_POSITRON))):
            raise ValueError("particle_type must use the supported IAEA codes 1/2/3")
        if not np.all(arrays["energy"] > 0.0):
            raise ValueError("every particle needs a positive energy")
        norms = arrays["ux"] ** 2 + arrays["uy"] ** 2 + arrays["uz"] ** 2
        if not np.all(np.abs(norms - 1.0) < 1.0e-5):
            raise ValueError("directions must be unit vectors")
        if not np.all(np.isfinite(arrays["weight"])) or np.any(arrays["weight"] < 0.0):
            raise ValueError("weights must be finite and non-negative")
        self._codes = codes
        self._columns = arrays

    def __len__(self) -> int:
        return int(self._codes.size)

    def columns(self) -> dict:
        """A copy of the stored population as column arrays."""
        out = {"particle_type": self._codes.copy()}
        out.update({name: col.copy() for name, col in self._columns.items()})
        return out

    @property
    def max_energy(self) -> float:
        return float(self._columns["energy"].max())

    def sample_batch(self, seed: int, history_offset: int, n: int) -> dict:
        """Upload columns of histories [offset, offset + n) (geometry/phasespace.py:757)."""
        k = sample_indices(seed, history_offset, n, len(self))
        out = {"particle_type": self._codes[k].copy()}
        out.update({name: col[k].astype(np.float32) for name, col in self._columns.items()})
        return out


class PhaseSpaceSource(InMemoryPhaseSpaceSource):
    """A phase space read from an IAEA file (geometry/phasespace.py:428): every
    transportable record, sampled uniformly with replacement.  The file is read
    once into memory (pyRadMC memory-maps it); the engine keeps it resident on
    the device."""

    def __init__(self, path, *, skip_unsupported: bool = True) -> None:
        self.path = Path(path)
        cols = load_iaea(path, skip_unsupported=skip_unsupported)
        super().__init__(cols["particle_type"], cols["energy"], cols["x"], cols["y"], cols["z"],
                         cols["ux"], cols["uy"], cols["uz"], cols["weight"])
