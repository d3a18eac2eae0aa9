"""Beam geometry: rotations, calc_range, canonical beamlets, the ray step.

Pinned against golden fixtures made by running the reference's own host code
(tests/golden/make_golden_geometry.py): the oracle and the library must agree
with it bit for bit.
"""
import math
import os

import numpy as np
import pytest

import oracle
from fastdose_b200 import api, phantoms
from fastdose_b200.types import BEAM_DTYPE, make_bundle, make_volume

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


def test_rotation_known_answers():
    # FastDoseLib/src/geom.cu:65-79 (printed there, asserted here)
    r = oracle.rotate_axis([3, 0, 0], [0, 0, 1], math.pi / 3)
    np.testing.assert_allclose(r, [1.5, 2.5980762, 0.0], atol=1e-5)
    c = math.sqrt(1 / 3)
    r = oracle.rotate_axis([3, 0, 0], [c, c, c], 2 * math.pi / 3)
    np.testing.assert_allclose(r, [0.0, 3.0, 0.0], atol=1e-5)


def test_rotation_inverse_round_trip():
    # geom.cu:99-110: inverse then forward returns the vector
    rng = np.random.default_rng(0)
    for _ in range(50):
        v = rng.uniform(0, 1, 3).astype(np.float32)
        th, ph, co = rng.uniform(-math.pi, math.pi, 3)
        back = oracle.rotate_beam(oracle.inv_rotate_beam(v, th, ph, co), th, ph, co)
        np.testing.assert_allclose(back, v, atol=1e-5)


def test_rotations_match_reference_bitwise():
    g = _load("geometry_c1.npz")
    for i in range(len(g["rot_v"])):
        v, ax, t = g["rot_v"][i], g["rot_axes"][i], float(g["rot_t"][i])
        th, ph, co = (float(a) for a in g["rot_angles"][i])
        assert np.array_equal(oracle.rotate_axis(v, ax, t), g["rot_axis_out"][i])
        assert np.array_equal(oracle.rotate_beam(v, th, ph, co), g["rot_fwd_out"][i])
        assert np.array_equal(oracle.inv_rotate_beam(v, th, ph, co), g["rot_inv_out"][i])


@pytest.mark.parametrize("fixture", ["geometry_c1.npz", "geometry_c2.npz"])
def test_oracle_beamlets_match_reference(fixture):
    g = _load(fixture)
    for bb, (ix, iy), ref, st in zip(g["bundles"], g["ixy"], g["beams"], g["status"]):
        s, b = oracle.beamlet_init(bb, int(ix), int(iy), g["volume"])
        assert (s != 0) == (st != 0)
        if st == 0:
            assert b.tobytes() == np.array(ref).tobytes(), (ix, iy)


@pytest.mark.parametrize("fixture", ["geometry_c1.npz", "geometry_c2.npz"])
def test_library_beamlets_match_reference(fixture):
    g = _load(fixture)
    for bb, (ix, iy), ref, st in zip(g["bundles"], g["ixy"], g["beams"], g["status"]):
        if st != 0:
            with pytest.raises(Exception):
                api.beamlet_init(bb, int(ix), int(iy), g["volume"])
            continue
        b = api.beamlet_init(bb, int(ix), int(iy), g["volume"])
        assert b.tobytes() == np.array(ref).tobytes(), (ix, iy)


def test_calc_range_miss_is_an_error():
    vol = make_volume((16, 16, 16), (0.25, 0.25, 0.25))
    b = np.zeros((), BEAM_DTYPE)
    b["isocenter"] = (100.0, 100.0, 100.0)  # far outside the box
    b["beamlet_size"] = (0.5, 0.5)
    b["fmap_size"] = (4, 4)
    b["sad"] = 100.0
    b["long_spacing"] = 0.25
    st, _ = oracle.calc_range(b, vol)
    assert st != 0
    with pytest.raises(Exception):
        api.calc_range(b, vol)


def test_calc_range_gantry0_depths():
    # gantry-0 beam through a cube centred on the isocentre: the central ray
    # enters at depth sad - half and leaves at sad + half (geom on the y axis)
    vol = make_volume((64, 64, 64), (0.25, 0.25, 0.25))
    b = np.zeros((), BEAM_DTYPE)
    b["isocenter"] = (8.0, 8.0, 8.0)
    b["beamlet_size"] = (0.1, 0.1)
    b["fmap_size"] = (2, 2)
    b["sad"] = 100.0
    b["long_spacing"] = 0.25
    out = api.calc_range(b, vol)
    assert out["lim_min"] == pytest.approx(92.0, abs=1e-3)
    assert out["lim_max"] == pytest.approx(108.0, abs=2e-3)
    np.testing.assert_allclose(out["source"], (8.0, -92.0, 8.0), atol=1e-4)
    assert int(out["long_dim"]) == math.ceil((out["lim_max"] - out["lim_min"]) / 0.25)


def test_next_point_steps_to_a_boundary():
    # d_nextPoint (DoseComp.cu:76-111): a step ends on a voxel boundary of the
    # limiting axis, or snaps onto the next z plane
    rng = np.random.default_rng(1)
    for _ in range(200):
        c = rng.uniform(0, 4, 3)
        d = rng.normal(size=3)
        d[2] = abs(d[2]) + 0.05
        d /= np.linalg.norm(d)
        np_, flag = oracle.next_point(c, d)
        t = (np_ - c) @ d
        assert t > 0
        if flag:
            assert np_[2] == round(np_[2])
        else:
            on = [abs(np_[q] - round(np_[q])) < 1e-4 for q in range(2)]
            assert any(on)


def test_line_seg_on_iso_plane_has_unit_factor():
    # geom.cu:239-250: both ends on the isocentre plane -> no divergence scaling
    cfg = phantoms.config1()
    bund = make_bundle(cfg["isocenter"], cfg["angles"][0], fluence_dim=10)
    _, b = oracle.beamlet_init(bund, 4, 4, cfg["phantom"].volume)
    z = (float(b["sad"]) - float(b["lim_min"])) / float(b["long_spacing"])
    s = np.array([3.2, 7.9, z])
    e = np.array([5.5, 1.25, z])
    diff = (e - s) * np.array([b["beamlet_size"][0], b["beamlet_size"][1], b["long_spacing"]])
    assert oracle.calc_line_seg(s, e, b) == pytest.approx(float(np.linalg.norm(diff)), rel=1e-5)


def test_sub_beam_fluence_is_centred_square():
    bund = make_bundle((0, 0, 0), (0, 0, 0), fluence_dim=4, sub_fluence_dim=16, sub_fluence_on=4)
    f = api.beamlet_fluence(bund).reshape(16, 16)
    assert f.sum() == 16
    assert f[6:10, 6:10].all()
    np.testing.assert_array_equal(f.ravel(), oracle.beamlet_fluence(bund))


def test_bundles_beamlets_equals_one_call_per_pixel():
    """The batched, multi-threaded beamlet initialisation gives the same bytes
    as one beamlet_init call per flagged pixel, for bundles of different
    fluence dimensions, including empty flag maps."""
    import numpy as np

    from fastdose_b200 import api, phantoms
    from fastdose_b200.types import make_bundle

    cfg = phantoms.config2(12)
    ph = cfg["phantom"]
    rng = np.random.default_rng(3)
    bundles, flags = [], []
    for k, a in enumerate(cfg["angles"]):
        fd = (8, 16, 11)[k % 3]
        bundles.append(make_bundle(cfg["isocenter"], a, sad=100.0, fluence_dim=fd, beamlet_size=0.5,
                                   sub_fluence_dim=16, sub_fluence_on=4, long_spacing=0.25))
        f = (rng.random(fd * fd) < 0.4).astype(np.uint8)
        if k == 5:
            f[:] = 0
        flags.append(f)
    bundles = np.array(bundles)
    ref = [api.bundle_beamlets(b, f, ph.volume) for b, f in zip(bundles, flags)]
    for threads in (1, 4, 0):
        got = api.bundles_beamlets(bundles, flags, ph.volume, threads=threads)
        assert len(got) == len(ref)
        for a, b in zip(ref, got):
            assert a.tobytes() == b.tobytes()
