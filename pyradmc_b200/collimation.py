"""Sources seen through a beam-limiting stack (pyRadMC geometry/collimation.py).

``CollimatedSource`` and ``CollimatedBeamletSource`` (collimation.py:1154 and
:1185) wrap a source and multiply each primary's weight by the stack's
narrow-beam transmission along its ray, ``exp(-sum_j mu_j(E) rho_j t_j)``
(``_StackTransmission``, :927-985): t_j the chord of the primary's full line
through device j, mu_j / rho the total mass attenuation of that device's
material on a log-log table over ``np.geomspace(e_min, inner.max_energy,
n_table)``.  The wrapper draws no random numbers.

The engine evaluates the transmission in its primary generator
(``pmc_source_desc.stack`` / ``pmc_beamlet_desc.stack``) whenever it generates
the inner source in-kernel; pyRadMC's own wrappers are accepted as well (their
stack and table are read from the wrapper).  The tables here come from a
cross-section source with ``mu_over_rho_total(energy, material)`` (pyRadMC's
``CrossSectionSource``), or ready-made through :meth:`from_tables`.
"""

from __future__ import annotations

import numpy as np

__all__ = ["CollimatedBeamletSource", "CollimatedSource", "stack_transmission_tables"]


def _compiled(stack):
    from .presolve import CompiledHeadStack

    return stack if isinstance(stack, CompiledHeadStack) else CompiledHeadStack.from_stack(stack)


class _Collimated:
    def __init__(self, inner, stack, cross_sections, *, e_min: float = 0.010, n_table: int = 512) -> None:
        compiled = _compiled(stack)
        if max(compiled.materials) >= cross_sections.n_materials:
            raise ValueError(
                f"stack material index {max(compiled.materials)} is beyond this "
                f"cross-section source ({cross_sections.n_materials} materials); "
                "device materials like tungsten need the tabulated backend"
            )
        e_max = float(inner.max_energy)
        if not 0.0 < e_min < e_max:
            raise ValueError(f"need 0 < e_min < e_max, got {e_min}, {e_max}")
        energies = np.geomspace(e_min, e_max, n_table)
        log_mu = np.log([[cross_sections.mu_over_rho_total(float(e), int(m)) for e in energies]
                         for m in compiled.materials])
        self._set(inner, compiled, np.log(energies), log_mu + np.log(compiled.densities)[:, None])

    def _set(self, inner, compiled, log_energy, log_total) -> None:
        log_energy = np.asarray(log_energy, dtype=np.float64)
        log_total = np.asarray(log_total, dtype=np.float64)
        if log_total.shape != (compiled.n_devices, log_energy.size) or log_energy.size < 2:
            raise ValueError(f"need one attenuation row per device, got {log_total.shape}")
        self._inner = inner
        self.stack = compiled
        self.log_energy = log_energy
        self.log_total = log_total

    @classmethod
    def from_tables(cls, inner, stack, log_energy, log_total):
        """A wrapper with a ready-made table: ``log_total[j]`` the log of device
        j's macroscopic attenuation (1/cm, density included) at ``log_energy``,
        log-uniform energies."""
        self = cls.__new__(cls)
        self._set(inner, _compiled(stack), log_energy, log_total)
        return self

    inner = property(lambda self: self._inner)
    max_energy = property(lambda self: self._inner.max_energy)


class CollimatedSource(_Collimated):
    """A forward source seen through a beam-limiting stack (collimation.py:1154)."""


class CollimatedBeamletSource(_Collimated):
    """A beamlet source seen through a beam-limiting stack (collimation.py:1185):
    the beamlet-dependent transmission along each bixel's rays is the
    collimation signal of the Dij columns."""

    n_beamlets = property(lambda self: self._inner.n_beamlets)


def stack_transmission_tables(source):
    """(inner, compiled stack, log energies, log macroscopic attenuation rows)
    of a collimated source, this package's or pyRadMC's, else None."""
    if type(source).__name__ not in ("CollimatedSource", "CollimatedBeamletSource"):
        return None
    if isinstance(source, _Collimated):
        return source.inner, source.stack, source.log_energy, source.log_total
    model = getattr(source, "_model", None)  # pyRadMC's _StackTransmission
    if model is None or not hasattr(model, "_log_mu"):
        return None
    log_total = np.asarray(model._log_mu) + np.log(np.asarray(model._densities, dtype=np.float64))[:, None]
    inner = getattr(source, "inner", None) or source._inner  # the beamlet wrapper keeps it private
    return inner, _compiled(model._stack), np.asarray(model._log_energies), log_total
