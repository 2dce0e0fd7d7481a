"""IAEA phase-space files on the host: the reader restates pyRadMC's
(geometry/phasespace.py) record decoding, the writer round-trips, malformed
headers are refused with the reference's messages, and pyRadMC's own reader
(where it is importable) decodes the committed fixture to the same columns."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

from pyradmc_b200 import phasespace as ps
from tests.conftest import GOLDEN


def _columns(n=64, seed=3):
    rng = np.random.default_rng(seed)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return dict(particle_type=rng.choice([1, 2, 3], size=n).astype(np.int32),
                energy=rng.uniform(0.1, 6.0, n), x=rng.normal(size=n), y=rng.normal(size=n),
                z=np.full(n, -1.0), ux=d[:, 0], uy=d[:, 1], uz=d[:, 2], weight=rng.uniform(0.5, 2, n))


@pytest.mark.parametrize("byte_order", ["<", ">"])
@pytest.mark.parametrize("store_all", [True, False])
def test_write_then_read_round_trips(tmp_path, byte_order, store_all):
    cols = _columns()
    ps.write_iaea(tmp_path / "beam", cols, byte_order=byte_order, store_all=store_all)
    h = ps.read_iaea_header(tmp_path / "beam.IAEAheader")
    assert h.n_particles == 64 and h.byte_order == byte_order
    assert ("z" in h.constants) == (not store_all)  # z is constant: a header constant when allowed
    got = ps.load_iaea(tmp_path / "beam")
    for k in ("energy", "x", "y", "z", "weight"):
        np.testing.assert_array_equal(got[k], np.asarray(cols[k], np.float32), err_msg=k)
    np.testing.assert_array_equal(got["particle_type"], cols["particle_type"])
    # w is rebuilt from float32 u, v and the sign: a few ulps of u, v become ~1e-5 near w = 0
    np.testing.assert_allclose(got["uz"], cols["uz"], atol=1e-4)
    assert np.all(got["new_history"])


def test_unsupported_particles_are_dropped_or_refused(tmp_path):
    cols = _columns()
    cols["particle_type"][:3] = 4  # neutrons
    ps.write_iaea(tmp_path / "mixed", cols)
    with pytest.warns(UserWarning, match="unsupported particle types"):
        assert ps.load_iaea(tmp_path / "mixed")["energy"].size == 61
    with pytest.raises(ValueError, match="unsupported particle type 4"):
        ps.load_iaea(tmp_path / "mixed", skip_unsupported=False)


def test_malformed_headers_are_refused(tmp_path):
    ps.write_iaea(tmp_path / "b", _columns())
    head = (tmp_path / "b.IAEAheader").read_text()  # 29-byte records: type, energy, six floats
    (tmp_path / "b.IAEAheader").write_text(head.replace("$RECORD_LENGTH:\n29", "$RECORD_LENGTH:\n40"))
    with pytest.raises(ValueError, match="RECORD_LENGTH 40 disagrees"):
        ps.read_iaea_header(tmp_path / "b")
    with open(tmp_path / "b.IAEAphsp", "ab") as f:
        f.write(b"\0")
    (tmp_path / "b.IAEAheader").write_text(head)
    with pytest.raises(ValueError, match="not a multiple of record length"):
        ps.read_iaea_header(tmp_path / "b")


def test_in_memory_source_checks_and_samples_chunk_invariantly():
    cols = _columns()
    src = ps.InMemoryPhaseSpaceSource(**cols)
    whole = src.sample_batch(11, 0, 100)
    part = src.sample_batch(11, 40, 60)
    for k in whole:
        np.testing.assert_array_equal(whole[k][40:], part[k])
    bad = dict(cols, ux=cols["ux"] * 2)
    with pytest.raises(ValueError, match="unit vectors"):
        ps.InMemoryPhaseSpaceSource(**bad)


def test_fixture_decodes_like_pyradmc_reader():
    source = os.environ.get("PYRADMC_SOURCE", "/root/reference")
    if not os.path.isdir(os.path.join(source, "pyradmc")):
        pytest.skip("pyRadMC is not available on this host")
    sys.path.insert(0, source)
    from pyradmc.geometry.phasespace import IAEAPhaseSpace

    ours = ps.load_iaea(GOLDEN / "phsp_beam")
    with IAEAPhaseSpace(GOLDEN / "phsp_beam") as f:
        recs = list(f)
    assert len(recs) == ours["energy"].size
    ref = {k: np.array([getattr(r, a) for r in recs], dtype=np.float32)
           for k, a in (("energy", "energy"), ("x", "x"), ("y", "y"), ("z", "z"), ("ux", "u"),
                        ("uy", "v"), ("uz", "w"), ("weight", "weight"))}
    for k, v in ref.items():
        np.testing.assert_array_equal(ours[k], v, err_msg=k)
    np.testing.assert_array_equal(ours["particle_type"], [r.particle_type for r in recs])
