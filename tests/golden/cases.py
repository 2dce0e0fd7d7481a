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
BONE_LAYERS = ((0.0, 2.0, 1.0), (2.0, 4.0, 1.85), (4.0, 1.0e9, 1.0))
BONE_MATERIAL = 4  # cortical_bone in pyRadMC's registry (data/materials.py:295)

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
    # 160,000 histories: enough that a 2 % bias in the lung or bone layer fails
    # the batched chi-squared.  Generated as 16 one-batch shards (see
    # make_golden.py), since the reference engine is single-threaded.
    "slab_spectral": dict(
        grid=dict(shape=(64, 64, 64), spacing=(0.2, 0.2, 0.2), layers=SLAB_LAYERS),
        source=dict(kind="spectral", focal_point=(6.4, 6.4, -100.0), center=(6.4, 6.4, 0.0),
                    width_u=10.0, width_v=10.0),
        run=dict(n_histories=160_000, n_batches=16, seed=SEED),
        shards=16,
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
    # An IAEA phase space (tests/golden/phsp_beam.*, written by make_golden.py):
    # a divergent 6 x 6 cm field of 6 MV photons with electron and positron
    # contamination at non-unit weights, sampled with replacement.
    "phasespace": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="phasespace", file="phsp_beam"),
        run=dict(n_histories=80_000, n_batches=10, seed=SEED),
        shards=10,
    ),
    # A 6 MeV pencil-beam kernel scored in depth bins by radial shells
    # (CylindricalScoringGrid.for_grid, scoring/cylinder.py:311): a central
    # 1 mm disc and 11 geometric shells out to 6 cm, depth bins on the grid's
    # z planes.
    "pencil_cylinder": dict(
        grid=dict(shape=(16, 16, 16), spacing=(1.0, 1.0, 1.0)),
        source=dict(kind="pencil", energy=6.0, position=(8.0, 8.0, -1.0), direction=(0.0, 0.0, 1.0)),
        run=dict(n_histories=200_000, n_batches=10, seed=SEED),
        scoring=dict(kind="cylinder", r_max=6.0, n_shells=12, r_min=0.1),
        shards=10,
        chi2_fraction=1e-3,  # a pencil kernel spans decades: compare down to 0.1 % of the maximum
    ),
    # Dose to water and dose to medium behind a cortical-bone layer (material 4
    # of pyRadMC's registry at 1.85 g/cc) in water: the stopping-power ratio
    # water/bone weights every bone deposit (scoring/dose_to_water.py:67-84).
    # The cross sections are the analytic source with the registry's first
    # five materials addressable, packed in pack_water_bone.npz.
    "dtw_bone": dict(
        grid=dict(shape=(16, 16, 30), spacing=(0.5, 0.5, 0.2), layers=BONE_LAYERS,
                  material_layers=((2.0, 4.0, 4),)),
        source=dict(kind="parallel", energy=6.0, z=-1.0, x_range=(0.0, 8.0), y_range=(0.0, 8.0)),
        run=dict(n_histories=80_000, n_batches=10, seed=SEED, scoring_mode="dose_to_water"),
        cross_sections="water_bone", shards=10,
    ),
    "dtm_bone": dict(
        grid=dict(shape=(16, 16, 30), spacing=(0.5, 0.5, 0.2), layers=BONE_LAYERS,
                  material_layers=((2.0, 4.0, 4),)),
        source=dict(kind="parallel", energy=6.0, z=-1.0, x_range=(0.0, 8.0), y_range=(0.0, 8.0)),
        run=dict(n_histories=80_000, n_batches=10, seed=SEED, scoring_mode="dose_to_medium"),
        cross_sections="water_bone", shards=10,
    ),
    # A fan entering through the -x face (its aperture axes y and z): the
    # geometry of a beam of a coplanar plan at gantry angle 90 degrees.
    "dij_oblique": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="spectral_beamlets", focal_point=(-100.0, 4.0, 4.0),
                    centers=((4.0, 3.0, 3.0), (4.0, 5.0, 3.0), (4.0, 3.0, 5.0), (4.0, 5.0, 5.0)),
                    width_u=1.5, width_v=1.5, u_axis=(0.0, 1.0, 0.0), v_axis=(0.0, 0.0, 1.0)),
        run=dict(n_histories_per_beamlet=8000, n_batches=8, seed=SEED, truncation=0.0),
    ),
    # A spectral fan through a transmission mask (TransmissionMaskSource,
    # geometry/collimation.py:1205): a 6 x 5 pixel mask with exact zeros and
    # ones on a plane halfway to the focal spot, its u axis along y, and a
    # rectangle narrower than the fan there, so the rim of the fan is cut.
    "spectral_masked": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="masked",
                    inner=dict(kind="spectral", focal_point=(4.0, 4.0, -100.0), center=(4.0, 4.0, 0.0),
                               width_u=6.0, width_v=6.0),
                    mask=((1.0, 0.9, 0.6, 0.3, 0.0),
                          (1.0, 1.0, 0.7, 0.2, 0.0),
                          (0.8, 1.0, 1.0, 0.5, 0.1),
                          (0.5, 0.7, 1.0, 1.0, 0.4),
                          (0.2, 0.4, 0.8, 1.0, 1.0),
                          (0.0, 0.1, 0.5, 0.9, 1.0)),
                    plane_center=(4.0, 4.0, -50.0), width_u=2.4, width_v=2.4,
                    u_axis=(0.0, 1.0, 0.0), v_axis=(1.0, 0.0, 0.0)),
        run=dict(n_histories=80_000, n_batches=10, seed=SEED),
        shards=10,
    ),
    # A spectral fan seen through a beam-limiting stack (CollimatedSource,
    # geometry/collimation.py:1154): the stack of COLLIMATION weights every
    # primary by its narrow-beam transmission.
    "collimated_spectral": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="collimated",
                    inner=dict(kind="spectral", focal_point=(4.0, 4.0, -100.0), center=(4.0, 4.0, 0.0),
                               width_u=6.0, width_v=6.0)),
        run=dict(n_histories=80_000, n_batches=10, seed=SEED),
        shards=10,
    ),
    # Four spectral beamlets through the same stack (CollimatedBeamletSource,
    # :1185): each column carries its own transmission pattern.
    "dij_collimated": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="collimated_beamlets",
                    inner=dict(kind="spectral_beamlets", focal_point=(4.0, 4.0, -100.0),
                               centers=((3.0, 3.0, 0.0), (5.0, 3.0, 0.0), (3.0, 5.0, 0.0), (5.0, 5.0, 0.0)),
                               width_u=2.0, width_v=2.0)),
        run=dict(n_histories_per_beamlet=8000, n_batches=8, seed=SEED, truncation=0.0),
    ),
    # Four spectral beamlets through a transmission mask
    # (TransmissionMaskBeamletSource, geometry/collimation.py:1264): the mask
    # of spectral_masked on a 3 x 3 cm rectangle halfway to the focus.
    "dij_masked": dict(
        grid=dict(shape=(16, 16, 16), spacing=(0.5, 0.5, 0.5)),
        source=dict(kind="masked_beamlets",
                    inner=dict(kind="spectral_beamlets", focal_point=(4.0, 4.0, -100.0),
                               centers=((3.0, 3.0, 0.0), (5.0, 3.0, 0.0), (3.0, 5.0, 0.0), (5.0, 5.0, 0.0)),
                               width_u=2.0, width_v=2.0),
                    mask=((1.0, 0.9, 0.6, 0.3, 0.0),
                          (1.0, 1.0, 0.7, 0.2, 0.0),
                          (0.8, 1.0, 1.0, 0.5, 0.1),
                          (0.5, 0.7, 1.0, 1.0, 0.4),
                          (0.2, 0.4, 0.8, 1.0, 1.0),
                          (0.0, 0.1, 0.5, 0.9, 1.0)),
                    plane_center=(4.0, 4.0, -50.0), width_u=3.0, width_v=3.0,
                    u_axis=(0.0, 1.0, 0.0), v_axis=(1.0, 0.0, 0.0)),
        run=dict(n_histories_per_beamlet=8000, n_batches=8, seed=SEED, truncation=0.0),
    ),
    # A per-beamlet mixture (CompositeBeamletSource): beamlet j is 60 % the
    # lattice rectangle j, 40 % the spectral fan j.
    "dij_composite": dict(
        grid=dict(shape=(8, 8, 16), spacing=(2.0, 2.0, 0.5)),
        source=dict(kind="composite", components=(
            (dict(kind="lattice", energy=6.0, z=-1.0, x_range=(2.0, 14.0), y_range=(2.0, 14.0),
                  n_x=2, n_y=2), 0.6),
            (dict(kind="spectral_beamlets", focal_point=(8.0, 8.0, -100.0),
                  centers=((5.0, 5.0, 0.0), (5.0, 11.0, 0.0), (11.0, 5.0, 0.0), (11.0, 11.0, 0.0)),
                  width_u=3.0, width_v=3.0), 0.4))),
        run=dict(n_histories_per_beamlet=6400, n_batches=8, seed=SEED, truncation=0.0),
    ),
}


# The beam-limiting stack of the collimated cases, in a beam frame at the
# focal spot (w along +z): a jaw pair closing the +x side beyond u = 0.4 cm
# at 42.5 cm from the focus, and a three-pair MLC whose middle pair is shut.
# The analytic cross sections know water only, so the devices are water at
# 3 g/cc.
COLLIMATION = dict(
    focal=(4.0, 4.0, -100.0),
    jaw=dict(axis="u", z_top=40.0, z_bottom=45.0, edge_neg=-1000.0, edge_pos=0.4, material=0, density=3.0),
    mlc=dict(z_top=50.0, z_bottom=56.0, leaf_edges_v=(-1.5, -0.5, 0.5, 1.5), tips_neg=(-1.0, 0.1, -1.0),
             tips_pos=(1.0, 0.1, 1.0), tip_radius=8.0, material=0, density=3.0),
)


def make_source(s: dict, ns):
    """A case's source built from the classes of `ns` (pyRadMC's modules or this
    package): PencilBeamSource, ParallelBeamSource, SpectralBeamSource,
    BeamletGridSource, SpectralBeamletSource, CompositeBeamletSource,
    TransmissionMaskSource, TransmissionMaskBeamletSource, PhaseSpaceSource, a 6 MV spectrum factory
    ``spectrum()`` and ``collimated(inner, beamlets)``, the inner source seen
    through the COLLIMATION stack."""
    kind = s["kind"]
    if kind == "parallel":
        return ns.ParallelBeamSource(s["energy"], s["z"], s["x_range"], s["y_range"])
    if kind == "pencil":
        return ns.PencilBeamSource(s["energy"], s["position"], s["direction"])
    if kind == "spectral":
        return ns.SpectralBeamSource(ns.spectrum(), s["focal_point"], s["center"], s["width_u"],
                                     s["width_v"])
    if kind == "lattice":
        return ns.BeamletGridSource(s["energy"], s["z"], s["x_range"], s["y_range"], s["n_x"], s["n_y"])
    if kind == "spectral_beamlets":
        axes = {k: s[k] for k in ("u_axis", "v_axis") if k in s}
        return ns.SpectralBeamletSource(ns.spectrum(), s["focal_point"], s["centers"], s["width_u"],
                                        s["width_v"], **axes)
    if kind in ("collimated", "collimated_beamlets"):
        return ns.collimated(make_source(s["inner"], ns), kind == "collimated_beamlets")
    if kind in ("masked", "masked_beamlets"):
        import numpy as np

        cls = ns.TransmissionMaskSource if kind == "masked" else ns.TransmissionMaskBeamletSource
        return cls(make_source(s["inner"], ns), mask=np.asarray(s["mask"]),
                                         plane_center=s["plane_center"], width_u=s["width_u"],
                                         width_v=s["width_v"], u_axis=s["u_axis"], v_axis=s["v_axis"])
    if kind == "composite":
        return ns.CompositeBeamletSource([(make_source(c, ns), w) for c, w in s["components"]])
    if kind == "phasespace":
        from pathlib import Path

        return ns.PhaseSpaceSource(Path(__file__).resolve().parent / s["file"])
    raise ValueError(kind)


# Scaled-down batched-Dij case: the benchmark's CT-like phantom family (water
# plus seeded ellipsoids of density U(0.2, 1.9), pyradmc_b200.phantoms) at
# 40^3 x 2.5 mm, a 2x2 fan of 5 mm Varian 6 MV spectral beamlets at SAD 100 cm
# through the phantom centre, GS multiple scattering.  The reference's run_dij
# takes one count for every column, so it runs once per count of CT_COUNTS;
# the B200 run gives the columns uneven counts and each column is compared
# with the reference run at its own count (ref_ct_beamlets_<count>.npz).
CT_CASE = dict(
    grid=dict(shape=(40, 40, 40), spacing=(0.25, 0.25, 0.25), ellipsoid_seed=20260805),
    fan=dict(n_x=2, n_y=2, pitch=0.5, width=0.5, sad=100.0),
    run=dict(n_batches=10, seed=SEED, truncation=0.0),
    counts=(40_000, 120_000),
)


def make_scoring(case: dict, grid, ns):
    """The case's scoring geometry built with `ns` (CylindricalScoringGrid and
    geometric_edges), or None for the transport grid."""
    sc = case.get("scoring")
    if sc is None:
        return None
    return ns.CylindricalScoringGrid.for_grid(grid, ns.geometric_edges(sc["r_max"], sc["n_shells"],
                                                                       sc["r_min"]))


def layered_material(shape, spacing, origin, layers):
    """Material index by voxel-centre depth: (z_lo, z_hi, material) slabs along z."""
    import numpy as np

    nz = shape[2]
    z = origin[2] + (np.arange(nz) + 0.5) * spacing[2]
    column = np.zeros(nz, dtype=np.int32)
    for lo, hi, m in layers:
        column[(z >= lo) & (z < hi)] = m
    return np.broadcast_to(column, shape).copy()


def layered_density(shape, spacing, origin, layers):
    """Density by voxel-centre depth: (z_lo, z_hi, density) slabs along z."""
    import numpy as np

    nz = shape[2]
    z = origin[2] + (np.arange(nz) + 0.5) * spacing[2]
    column = np.ones(nz)
    for lo, hi, rho in layers:
        column[(z >= lo) & (z < hi)] = rho
    return np.broadcast_to(column, shape).copy()
