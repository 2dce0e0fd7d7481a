"""Generate the water data packs this package ships, with pyRadMC's own builders.

The B200 engine consumes exactly what pyRadMC's host side produces for the Warp
backend: the flattened ``CrossSectionTables`` of
``CrossSectionSource.build_tables`` (pyradmc/data/tables.py:222) and the
Goudsmit-Saunderson node grid of ``build_gs_grid``
(pyradmc/data/goudsmit_saunderson.py:1108).  When pyRadMC is importable the
engine calls those builders directly.  These packs carry the same arrays for the
analytic water source, so the engine and its tests also run where pyRadMC is not
installed (the GPU hosts).

Usage (needs a pyRadMC checkout; writes next to this file)::

    python -m pyradmc_b200.data.make_packs /path/to/pyRadMC

Packs written:

``water_tables_<e_max>.npz``
    ``AnalyticCrossSections().build_tables(ecut=0.2, pcut=0.05,
    e_max=E * (1 + 1e-6))`` for each primary energy E in :data:`ENERGIES`
    (the margin is WarpEngine's ``_E_MAX_MARGIN``, engine.py:80).
``water_gs_grid.npz``
    The GS window ``build_gs_grid(*gs_window_from_tables(tables_6MeV, [water]))``,
    float32.  GS nodes are pure functions of their node coordinates, and every
    water window with e_max <= 6 MeV at ECUT 0.2 MeV is a sub-rectangle of it.
``spectrum_varian_6mv.npz``
    ``ali_rogers_mv("varian-6mv", e_min=0.1)``: bin edges and photon-number weights.
"""

from __future__ import annotations

import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ENERGIES = (1.0, 2.0, 5.0, 5.76, 6.0)
ECUT = 0.2
PCUT = 0.05
E_MAX_MARGIN = 1.0 + 1.0e-6
TABLE_FIELDS = (
    "mu_compton",
    "mu_photo",
    "mu_pair",
    "mu_rayleigh",
    "majorant",
    "stopping_restricted",
    "stopping_radiative",
    "moller",
    "csda_range",
    "scattering_power",
    "log_eta",
    "restricted_range",
    "energy_of_restricted_range",
    "coherent_x",
    "coherent_cumulative",
)
TABLE_SCALARS = (
    "n_points",
    "ecut",
    "pcut",
    "e_max",
    "photon_log_e_min",
    "photon_inv_dlog",
    "electron_log_e_min",
    "electron_inv_dlog",
    "range_log_r_min",
    "range_inv_dlog",
    "n_coherent",
)


def energy_label(energy: float) -> str:
    return f"{energy:.4f}".rstrip("0").rstrip(".")


def main(reference: str) -> None:
    sys.path.insert(0, reference)
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.data.goudsmit_saunderson import build_gs_grid, gs_window_from_tables
    from pyradmc.geometry.spectrum import ali_rogers_mv

    source = AnalyticCrossSections()
    tables_6 = None
    for energy in ENERGIES:
        tab = source.build_tables(ecut=ECUT, pcut=PCUT, e_max=energy * E_MAX_MARGIN)
        payload = {name: np.asarray(getattr(tab, name), dtype=np.float64) for name in TABLE_FIELDS}
        for name in TABLE_SCALARS:
            payload[name] = np.asarray(getattr(tab, name))
        payload["provenance"] = np.asarray(source.provenance)
        np.savez_compressed(HERE / f"water_tables_{energy_label(energy)}.npz", **payload)
        if energy == 6.0:
            tables_6 = tab
    window = gs_window_from_tables(tables_6, [0])
    grid = build_gs_grid(*window)
    np.savez_compressed(
        HERE / "water_gs_grid.npz",
        values=grid.values.astype(np.float32),
        ix0=np.int64(grid.ix0),
        iy0=np.int64(grid.iy0),
        n_u=np.int64(grid.n_u),
        bins_per_log=np.float64(grid.bins_per_log),
    )
    spectrum = ali_rogers_mv("varian-6mv", e_min=0.1)
    weights = spectrum.bin_probabilities
    np.savez_compressed(
        HERE / "spectrum_varian_6mv.npz",
        edges=np.asarray(spectrum.edges, dtype=np.float64),
        weights=np.asarray(weights, dtype=np.float64),
        cdf=np.asarray(spectrum.cdf, dtype=np.float64),
    )
    print("packs written to", HERE, "GS window", window, grid.values.shape, math.nan)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: python -m pyradmc_b200.data.make_packs /path/to/pyRadMC")
    os.environ.setdefault("PYRADMC_PACKS_FROM", sys.argv[1])
    main(sys.argv[1])
