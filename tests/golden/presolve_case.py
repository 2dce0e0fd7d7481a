"""The head pre-solve parity case, shared by the fixture script and the tests.

The geometry follows the reference's own device pre-solve test
(tests/physics/test_warp_presolve.py:37-80): a 6 MV-like photon fan from a
focal spot at (8, 8, -100) cm through a half-blocking jaw pair and a three-pair
staircase MLC of water (the analytic backend is water-only), exit plane at
w = 60 cm, and an air column of low-density water for the contaminant-electron
case.  The primaries come from :class:`FanSource`, a seeded NumPy sampler that
both the host oracle and the device run consume, so the two see the same
primaries.
"""

from __future__ import annotations

import numpy as np

N = 120_000
SEED = 20260726
FOCAL = (8.0, 8.0, -100.0)
EXIT_Z = 60.0
AIR_EXIT_Z = 95.0
AIR = dict(z_start=51.0, z_end=95.0, material=0, density=1.2e-3)
SPECTRUM_EDGES = (0.5, 1.0, 2.0, 4.0, 6.0)
SPECTRUM_WEIGHTS = (1.0, 3.0, 4.0, 2.0)

JAW = dict(axis="u", z_top=40.0, z_bottom=45.0, edge_neg=-1000.0, edge_pos=0.5, material=0, density=1.0)
MLC = dict(z_top=46.0, z_bottom=50.0, leaf_edges_v=(-3.0, -1.0, 1.0, 3.0), tips_neg=(-1.5, 0.2, -1.5),
           tips_pos=(1.5, 0.2, 1.5), tip_radius=8.0, material=0, density=1.0)
# a second stack for the chord-length check: focused jaws on both axes and a
# focused-side MLC with open and closed pairs
JAW_U_FOCUSED = dict(axis="u", z_top=30.0, z_bottom=37.0, edge_neg=-2.0, edge_pos=2.5, material=0,
                     density=1.0, focused=True)
JAW_V = dict(axis="v", z_top=38.0, z_bottom=44.0, edge_neg=-3.0, edge_pos=1.0, material=0, density=1.0)
MLC_FOCUSED = dict(z_top=46.0, z_bottom=52.0, leaf_edges_v=(-4.0, -2.0, 0.0, 2.0, 4.0),
                   tips_neg=(-2.0, -0.5, -3.0, 0.0), tips_pos=(2.0, 1.0, -0.5, 0.0), tip_radius=10.0,
                   material=0, density=1.0, focused_sides=True)


class FanSource:
    """Photons aimed from a Gaussian focal spot (sigma 0.1 cm) at points spread
    uniformly over a 6 x 6 cm square on the plane z = -70 cm, energies from a
    piecewise-uniform spectrum, unit weights; seeded by (seed, history_offset)."""

    max_energy = SPECTRUM_EDGES[-1]

    def sample_batch(self, seed: int, history_offset: int, n: int) -> dict:
        rng = np.random.Generator(np.random.PCG64([seed, history_offset]))
        edges = np.asarray(SPECTRUM_EDGES)
        w = np.asarray(SPECTRUM_WEIGHTS) * np.diff(edges)
        k = rng.choice(w.size, size=n, p=w / w.sum())
        energy = edges[k] + rng.random(n) * (edges[k + 1] - edges[k])
        spot = np.asarray(FOCAL) + np.column_stack([rng.normal(0.0, 0.1, (n, 2)), np.zeros(n)])
        target = np.column_stack([FOCAL[0] + 6.0 * (rng.random(n) - 0.5),
                                  FOCAL[1] + 6.0 * (rng.random(n) - 0.5), np.full(n, -70.0)])
        d = target - spot
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        return {"particle_type": np.ones(n, dtype=np.int32), "energy": energy, "x": spot[:, 0],
                "y": spot[:, 1], "z": spot[:, 2], "ux": d[:, 0], "uy": d[:, 1], "uz": d[:, 2],
                "weight": np.ones(n)}


def random_rays(n: int, seed: int = 7):
    """Engine-frame rays through and around the stacks: origins near the focal
    spot and inside the device slabs, directions mostly downstream, a few
    parallel to the slabs and a few exactly along w."""
    rng = np.random.default_rng(seed)
    p = np.column_stack([FOCAL[0] + rng.normal(0, 3, n), FOCAL[1] + rng.normal(0, 3, n),
                         -100.0 + rng.uniform(0.0, 160.0, n)])
    d = np.column_stack([rng.normal(0, 0.08, n), rng.normal(0, 0.08, n), np.ones(n)])
    flip = rng.random(n) < 0.1
    d[flip, 2] *= -1.0
    flat = rng.random(n) < 0.03  # parallel to the slabs
    d[flat, 2] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    axial = rng.random(n) < 0.02
    d[axial] = (0.0, 0.0, 1.0)
    return p, d
