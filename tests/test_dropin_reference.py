"""The drop-in boundary with pyRadMC's own objects, on a CPU-only host.

``B200Engine`` accepts pyRadMC's ``VoxelGrid``, ``AnalyticCrossSections`` and
beamlet sources unchanged.  Where pyRadMC is importable (its checkout named by
``PYRADMC_SOURCE``), this builds the engine from those objects and checks,
without a GPU, that everything the engine hands the C-ABI equals what the
mirror classes and packed tables hand it on the GPU hosts:

* the flattened cross-section tables (``CrossSectionSource.build_tables``,
  data/tables.py:222) equal the packed arrays, field by field;
* the Goudsmit-Saunderson node grid comes from pyRadMC's own
  ``build_gs_grid(*gs_window_from_tables(...))`` (the branch
  ``WarpEngine._gs_grid_host`` takes, engine.py:3431-3451), and every node it
  shares with the pack is bit-identical as uploaded (float32);
* the Dij descriptors (spectral fan, lattice, and a composite mixture) carry
  the same geometry, spectra and mixture weights as the mirror sources'.
"""

from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np
import pytest

from tests.conftest import CT_CASE

SOURCE = os.environ.get("PYRADMC_SOURCE", "/root/reference")


@pytest.fixture(scope="module")
def pyradmc(tmp_path_factory):
    if not os.path.isdir(os.path.join(SOURCE, "pyradmc")):
        pytest.skip("pyRadMC is not available on this host")
    if SOURCE not in sys.path:
        sys.path.insert(0, SOURCE)
    import pyradmc.data.goudsmit_saunderson as gs

    # keep pyRadMC's on-disk GS cache inside the test's scratch directory
    gs._GS_GRID_CACHE_DIR = tmp_path_factory.mktemp("gs-grid")
    import pyradmc

    return pyradmc


def _ct_grids(pyradmc):
    from pyradmc.geometry.grid import VoxelGrid

    from pyradmc_b200 import phantoms

    g = CT_CASE["grid"]
    mirror = phantoms.ellipsoid_phantom(shape=g["shape"], spacing=g["spacing"], seed=g["ellipsoid_seed"])
    ref = VoxelGrid(shape=g["shape"], spacing=g["spacing"], density=mirror.density,
                    material=np.zeros(g["shape"], dtype=np.int32))
    return mirror, ref


def test_reference_tables_and_gs_grid_drive_the_engine(pyradmc):
    from pyradmc.data.analytic import AnalyticCrossSections

    import pyradmc_b200 as P

    mirror_grid, ref_grid = _ct_grids(pyradmc)
    assert ref_grid.max_density_by_material() == mirror_grid.max_density_by_material()
    ref_xs = AnalyticCrossSections(geometry_densities=ref_grid.max_density_by_material())
    mirror_xs = P.AnalyticWaterTables(geometry_densities=mirror_grid.max_density_by_material())
    ref_engine = P.B200Engine(ref_grid, ref_xs)
    mirror_engine = P.B200Engine(mirror_grid, mirror_xs)
    e_max = 5.76  # the 6 MV spectrum's top edge: one of the packed energies
    ref_tab = ref_engine._host_tables(e_max, 0.05, 0.2)
    mirror_tab = mirror_engine._host_tables(e_max, 0.05, 0.2)
    for name in ("mu_compton", "mu_photo", "mu_pair", "mu_rayleigh", "majorant",
                 "stopping_restricted", "stopping_radiative", "moller", "csda_range",
                 "scattering_power", "log_eta", "restricted_range", "energy_of_restricted_range"):
        np.testing.assert_array_equal(np.asarray(getattr(ref_tab, name)),
                                      np.asarray(getattr(mirror_tab, name)), err_msg=name)
    for name in ("n_points", "photon_log_e_min", "photon_inv_dlog", "electron_log_e_min",
                 "electron_inv_dlog", "range_log_r_min", "range_inv_dlog"):
        assert getattr(ref_tab, name) == getattr(mirror_tab, name), name

    # no gs_grid_for on pyRadMC's source: the engine builds the window itself
    assert not hasattr(ref_xs, "gs_grid_for")
    ref_gs = ref_engine._gs_host(ref_tab, 0.2, e_max)
    pack_gs = mirror_engine._gs_host(mirror_tab, 0.2, e_max)
    assert ref_gs.bins_per_log == pack_gs.bins_per_log
    rv, pv = np.asarray(ref_gs.values), np.asarray(pack_gs.values)
    assert rv.shape[2] == pv.shape[2]
    ix0, iy0 = max(ref_gs.ix0, pack_gs.ix0), max(ref_gs.iy0, pack_gs.iy0)
    ix1 = min(ref_gs.ix0 + rv.shape[0], pack_gs.ix0 + pv.shape[0])
    iy1 = min(ref_gs.iy0 + rv.shape[1], pack_gs.iy0 + pv.shape[1])
    assert ix1 - ix0 >= 2 and iy1 - iy0 >= 2, "the windows do not overlap"
    # the pack covers every window the reference derives for these tables
    assert pack_gs.ix0 <= ref_gs.ix0 and pack_gs.iy0 <= ref_gs.iy0
    assert ix1 == ref_gs.ix0 + rv.shape[0] and iy1 == ref_gs.iy0 + rv.shape[1]
    # the engine uploads float32 nodes, as the Warp engine does
    np.testing.assert_array_equal(
        rv[ix0 - ref_gs.ix0:ix1 - ref_gs.ix0, iy0 - ref_gs.iy0:iy1 - ref_gs.iy0].astype(np.float32),
        pv[ix0 - pack_gs.ix0:ix1 - pack_gs.ix0, iy0 - pack_gs.iy0:iy1 - pack_gs.iy0].astype(np.float32))


def _desc_fields(desc, n):
    from pyradmc_b200 import _lib

    out = {"type": desc.type, "n_beamlets": desc.n_beamlets, "n_components": desc.n_components}
    if desc.type == _lib.PMC_BEAMLET_SPECTRAL:
        out.update(centers=np.ctypeslib.as_array(desc.centers, (n * 3,)).copy(),
                   edges=np.ctypeslib.as_array(desc.edges, (desc.n_bins + 1,)).copy(),
                   cdf=np.ctypeslib.as_array(desc.cdf, (desc.n_bins,)).copy(),
                   focal=tuple(desc.focal), u=tuple(desc.u_axis), v=tuple(desc.v_axis),
                   w=(desc.width_u, desc.width_v))
    elif desc.type == _lib.PMC_BEAMLET_LATTICE:
        out.update({k: np.ctypeslib.as_array(getattr(desc, k), (n,)).copy()
                    for k in ("x_lo", "x_extent", "y_lo", "y_extent")},
                   energy=desc.energy, z0=desc.z0)
    elif desc.type == _lib.PMC_BEAMLET_RECORDS:
        recs = C.cast(desc.records, C.POINTER(_lib.BeamletRec * (n * desc.n_components))).contents
        out["records"] = bytes(recs)
        out["cdf"] = np.ctypeslib.as_array(desc.component_cdf, (desc.n_components,)).copy()
        out["bins"] = np.ctypeslib.as_array(desc.spectrum_bins, (desc.n_spectra,)).copy()
        total = int(out["bins"].sum())
        out["edges"] = np.ctypeslib.as_array(desc.spectrum_edges, (total + desc.n_spectra,)).copy()
        out["spectrum_cdf"] = np.ctypeslib.as_array(desc.spectrum_cdf, (total,)).copy()
    return out


def _assert_same(a, b):
    assert a.keys() == b.keys()
    for k in a:
        if isinstance(a[k], np.ndarray):
            np.testing.assert_array_equal(a[k], b[k], err_msg=k)
        else:
            assert a[k] == b[k], k


def test_reference_beamlet_sources_give_the_mirror_descriptors(pyradmc):
    from pyradmc.geometry.source import (
        BeamletGridSource,
        CompositeBeamletSource,
        SpectralBeamletSource,
    )
    from pyradmc.geometry.spectrum import ali_rogers_mv

    import pyradmc_b200 as P
    from pyradmc_b200 import _lib, phantoms
    from pyradmc_b200.engine import beamlet_descriptor

    mirror_grid, _ = _ct_grids(pyradmc)
    fan = phantoms.beamlet_fan(mirror_grid, n_x=3, n_y=2)
    ref_fan = SpectralBeamletSource(ali_rogers_mv("varian-6mv", e_min=0.1), fan.focal_point,
                                    fan.centers, fan.width_u, fan.width_v)
    lattice = P.BeamletGridSource(6.0, -1.0, (1.0, 9.0), (2.0, 8.0), 3, 2)
    ref_lattice = BeamletGridSource(6.0, -1.0, (1.0, 9.0), (2.0, 8.0), 3, 2)
    mix = P.CompositeBeamletSource([(lattice, 0.3), (fan, 0.7)])
    ref_mix = CompositeBeamletSource([(ref_lattice, 0.3), (ref_fan, 0.7)])
    for mirror, ref, kind in ((fan, ref_fan, _lib.PMC_BEAMLET_SPECTRAL),
                              (lattice, ref_lattice, _lib.PMC_BEAMLET_LATTICE),
                              (mix, ref_mix, _lib.PMC_BEAMLET_RECORDS)):
        n = int(ref.n_beamlets)
        keep_a, keep_b = [], []
        a = beamlet_descriptor(ref, slice(0, n), 7, keep_a)
        b = beamlet_descriptor(mirror, slice(0, n), 7, keep_b)
        assert a.type == kind
        _assert_same(_desc_fields(a, n), _desc_fields(b, n))
    # the reference spectrum object and the packed one are the same histogram
    np.testing.assert_array_equal(np.asarray(ref_fan.spectrum.edges), fan.spectrum.edges)
    np.testing.assert_array_equal(np.asarray(ref_fan.spectrum.cdf), fan.spectrum.cdf)


def test_mask_source_mirror_matches_the_reference_class(pyradmc):
    """The engine reads a TransmissionMaskSource (geometry/collimation.py:1205)
    through its properties alone: the mirror exposes the same values and
    refuses the same masks with the same messages."""
    from pyradmc.geometry.collimation import TransmissionMaskSource as Ref
    from pyradmc.geometry.source import SpectralBeamSource
    from pyradmc.geometry.spectrum import ali_rogers_mv

    import pyradmc_b200 as P

    inner_ref = SpectralBeamSource(ali_rogers_mv("varian-6mv", e_min=0.1), (4.0, 4.0, -100.0),
                                   (4.0, 4.0, 0.0), 6.0, 6.0)
    inner = P.SpectralBeamSource(P.ali_rogers_varian_6mv(), (4.0, 4.0, -100.0), (4.0, 4.0, 0.0), 6.0, 6.0)
    good = dict(mask=np.linspace(0.0, 1.0, 12).reshape(3, 4), plane_center=(4.0, 4.0, -50.0),
                width_u=2.4, width_v=3.0, u_axis=(0.0, 2.0, 0.0), v_axis=(1.0, 0.0, 0.0))
    a, b = Ref(inner_ref, **good), P.TransmissionMaskSource(inner, **good)
    np.testing.assert_array_equal(a.mask, b.mask)
    for name in ("plane_center", "width_u", "width_v", "u_axis", "v_axis"):
        assert getattr(a, name) == getattr(b, name), name
    assert a.max_energy == b.max_energy
    for bad in (dict(mask=np.zeros(3)), dict(mask=np.full((2, 2), 1.5)), dict(width_u=0.0),
                dict(u_axis=(0.0, 0.0, 0.0)), dict(v_axis=(0.0, 1.0, 0.0))):
        kw = {**good, **bad}
        with pytest.raises(ValueError) as ref_err:
            Ref(inner_ref, **kw)
        with pytest.raises(ValueError, match=str(ref_err.value).replace("(", r"\(").replace(")", r"\)")):
            P.TransmissionMaskSource(inner, **kw)


def test_collimated_wrappers_read_the_reference_stack_and_table(pyradmc):
    """pyRadMC's CollimatedSource / CollimatedBeamletSource
    (geometry/collimation.py:1154-1204) hand the engine the same compiled stack
    and attenuation rows as this package's wrappers built from the same stack
    and cross sections: the Dij-compatible collimation route with the
    reference's own objects."""
    from pyradmc.data.analytic import AnalyticCrossSections
    from pyradmc.geometry.collimation import MLC, BeamFrame, BeamLimitingStack, CollimatedBeamletSource, JawPair
    from pyradmc.geometry.source import SpectralBeamletSource
    from pyradmc.geometry.spectrum import ali_rogers_mv

    import pyradmc_b200 as P
    from pyradmc_b200.collimation import stack_transmission_tables
    from tests.golden.cases import COLLIMATION as c

    stack = BeamLimitingStack(frame=BeamFrame(origin=c["focal"]), devices=(JawPair(**c["jaw"]), MLC(**c["mlc"])))
    xs = AnalyticCrossSections()
    inner = SpectralBeamletSource(ali_rogers_mv("varian-6mv", e_min=0.1), c["focal"], ((3.0, 3.0, 0.0),), 2.0, 2.0)
    ref = stack_transmission_tables(CollimatedBeamletSource(inner, stack, xs))
    mine = stack_transmission_tables(P.CollimatedBeamletSource(inner, stack, xs))
    assert ref[0] is inner and mine[0] is inner
    for name in ("kind", "z_top", "z_bottom", "jaw_edge_pos", "leaf_edges_v", "tips_neg", "tips_pos"):
        np.testing.assert_array_equal(getattr(ref[1], name), getattr(mine[1], name))
    assert ref[1].densities == mine[1].densities == (3.0, 3.0)
    np.testing.assert_array_equal(ref[2], mine[2])
    np.testing.assert_allclose(mine[3], ref[3], rtol=0, atol=1e-12)
    with pytest.raises(ValueError, match="e_min < e_max"):
        P.CollimatedBeamletSource(inner, stack, xs, e_min=10.0)


def test_reference_mask_beamlet_source_gives_the_mirror_descriptor(pyradmc):
    """pyRadMC's TransmissionMaskBeamletSource (geometry/collimation.py:1264)
    exposes neither its inner source nor its mask; the engine reads them from
    the wrapper's model and builds the descriptor the mirror class gives."""
    from pyradmc.geometry.collimation import TransmissionMaskBeamletSource
    from pyradmc.geometry.source import SpectralBeamletSource
    from pyradmc.geometry.spectrum import ali_rogers_mv

    import pyradmc_b200 as P
    from pyradmc_b200.engine import beamlet_descriptor

    spectrum = ali_rogers_mv("varian-6mv", e_min=0.1)
    kw = dict(mask=np.linspace(0.0, 1.0, 6).reshape(2, 3), plane_center=(4.0, 4.0, -50.0), width_u=3.0,
              width_v=2.0, u_axis=(0.0, 1.0, 0.0), v_axis=(1.0, 0.0, 0.0))
    centers = ((3.0, 3.0, 0.0), (5.0, 3.0, 0.0))
    ref = TransmissionMaskBeamletSource(SpectralBeamletSource(spectrum, (4.0, 4.0, -100.0), centers, 2.0, 2.0),
                                        **kw)
    mine = P.TransmissionMaskBeamletSource(
        P.SpectralBeamletSource(P.ali_rogers_varian_6mv(), (4.0, 4.0, -100.0), centers, 2.0, 2.0), **kw)
    keep: list = []
    a, b = beamlet_descriptor(ref, slice(0, 2), 1, keep), beamlet_descriptor(mine, slice(0, 2), 1, keep)
    assert a.type == b.type and a.mask_n_u == b.mask_n_u == 2 and a.mask_n_v == b.mask_n_v == 3
    for name in ("mask_center", "mask_u_axis", "mask_v_axis"):
        assert list(getattr(a, name)) == list(getattr(b, name))
    assert (a.mask_width_u, a.mask_width_v) == (b.mask_width_u, b.mask_width_v) == (3.0, 2.0)
    assert [a.mask[i] for i in range(6)] == [b.mask[i] for i in range(6)]
