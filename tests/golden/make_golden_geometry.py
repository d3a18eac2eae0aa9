"""Generates tests/golden/geometry_*.npz from the REFERENCE's own host code.

Runs here (CPU only): loads oracle/_ref/libfdref.so, the reference sources
compiled by oracle/build_ref.sh, and records
  * rotateAroundAxisAtOriginRHS / (inverse)RotateBeamAtOriginRHS on seeded inputs
    (FastDoseLib/src/geom.cu:11-56),
  * BEAM_h::calc_range (FastDoseLib/src/beam.cu:134-222) and
    BeamBundle::beamletInit (IMRTOpt/src/IMRTBeamBundle.cu:341-569) for the
    single-beam slab case and a subset of the 4pi torso case.
Usage: python tests/golden/make_golden_geometry.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from fastdose_b200 import phantoms  # noqa: E402
from fastdose_b200.types import BUNDLE_DTYPE, make_bundle  # noqa: E402
from oracle import ref  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def rotations():
    rng = np.random.default_rng(7)
    v = rng.uniform(-50, 50, (64, 3)).astype(np.float32)
    ang = rng.uniform(-np.pi, np.pi, (64, 3)).astype(np.float32)
    axes = rng.normal(size=(64, 3))
    axes = (axes / np.linalg.norm(axes, axis=1, keepdims=True)).astype(np.float32)
    t = rng.uniform(-np.pi, np.pi, 64).astype(np.float32)
    rot_axis = np.stack([ref.rotate_axis(v[i], axes[i], float(t[i])) for i in range(64)])
    fwd = np.stack([ref.rotate_beam(v[i], *map(float, ang[i])) for i in range(64)])
    inv = np.stack([ref.rotate_beam(v[i], *map(float, ang[i]), inverse=True) for i in range(64)])
    return dict(rot_v=v, rot_angles=ang, rot_axes=axes, rot_t=t, rot_axis_out=rot_axis, rot_fwd_out=fwd,
                rot_inv_out=inv)


def beamlets(cfg, beam_stride, picks):
    ph = cfg["phantom"]
    bundles, ixy, beams, status = [], [], [], []
    for ang in cfg["angles"][::beam_stride]:
        bb = make_bundle(cfg["isocenter"], ang, sad=cfg["sad"], fluence_dim=cfg["fluence_dim"],
                         beamlet_size=cfg["beamlet_size"], sub_fluence_dim=cfg["sub_fluence_dim"],
                         sub_fluence_on=cfg["sub_fluence_on"], long_spacing=cfg["long_spacing"])
        n = cfg["fluence_dim"]
        for (ix, iy) in (picks if picks is not None else [(i % n, i // n) for i in range(n * n)]):
            st, b = ref.beamlet_init(bb, ix, iy, ph.volume)
            bundles.append(bb)
            ixy.append((ix, iy))
            beams.append(b)
            status.append(st)
    return dict(bundles=np.array(bundles, BUNDLE_DTYPE), ixy=np.array(ixy, np.int32),
                beams=np.array(beams), status=np.array(status, np.int32), volume=np.array(ph.volume))


def main():
    if not ref.available():
        raise SystemExit("oracle/_ref/libfdref.so missing: run oracle/build_ref.sh")
    c1 = phantoms.config1()
    np.savez_compressed(os.path.join(OUT, "geometry_c1.npz"), **rotations(), **beamlets(c1, 1, None))
    c2 = phantoms.config2()
    picks = [(0, 0), (15, 15), (7, 8), (3, 12), (12, 3), (8, 7), (0, 15), (15, 0)]
    np.savez_compressed(os.path.join(OUT, "geometry_c2.npz"), **beamlets(c2, 7, picks))
    print("wrote geometry_c1.npz, geometry_c2.npz")


if __name__ == "__main__":
    main()
