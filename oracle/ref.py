"""ctypes bindings of oracle/_ref/libfdref.so -- the REFERENCE's own sources
compiled by oracle/build_ref.sh with the harness oracle/ref/ref_harness.cu.

Test infrastructure: used to pin the oracle and to make golden fixtures.  The
geometry entry points are host-only; the dose entry points need a GPU.
"""
import ctypes as C
import os

import numpy as np

from fastdose_b200.types import BEAM_DTYPE, BUNDLE_DTYPE, VOLUME_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
PATH = os.path.join(HERE, "_ref", "libfdref.so")
_L = None


def available():
    return os.path.exists(PATH)


def lib():
    global _L
    if _L is None:
        _L = C.CDLL(PATH)
        _L.ref_rotate_axis.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_void_p]
        _L.ref_rotate_beam.argtypes = [C.c_void_p, C.c_float, C.c_float, C.c_float, C.c_int, C.c_void_p]
        _L.ref_calc_range.argtypes = [C.c_void_p, C.c_void_p]
        _L.ref_beamlet_init.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        _L.ref_bev2pvcs.argtypes = [C.c_void_p] * 4
    return _L


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def rotate_axis(p, r, t):
    p = np.ascontiguousarray(p, np.float32)
    r = np.ascontiguousarray(r, np.float32)
    o = np.zeros(3, np.float32)
    lib().ref_rotate_axis(_p(p), _p(r), t, _p(o))
    return o


def rotate_beam(v, th, ph, co, inverse=False):
    v = np.ascontiguousarray(v, np.float32)
    o = np.zeros(3, np.float32)
    lib().ref_rotate_beam(_p(v), th, ph, co, int(inverse), _p(o))
    return o


def calc_range(beam, volume):
    b = np.array(beam, BEAM_DTYPE).copy()
    v = np.array(volume, VOLUME_DTYPE)
    st = lib().ref_calc_range(_p(b), _p(v))
    return st, b


def beamlet_init(bundle, ix, iy, volume):
    out = np.zeros((), BEAM_DTYPE)
    bb = np.array(bundle, BUNDLE_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    st = lib().ref_beamlet_init(_p(bb), ix, iy, _p(v), _p(out))
    return st, out


def beamlet_flags(bundles, ptv_mask, volume, density):
    bb = np.ascontiguousarray(bundles, BUNDLE_DTYPE)
    m = np.ascontiguousarray(ptv_mask, np.uint8)
    v = np.array(volume, VOLUME_DTYPE)
    P = int(bb[0]["fluence_dim"][0]) * int(bb[0]["fluence_dim"][1])
    out = np.zeros(bb.size * P, np.uint8)
    st = lib().ref_beamlet_flags(C.c_int(bb.size), _p(bb), _p(m), _p(v),
                                 _p(np.ascontiguousarray(density, np.float32)), _p(out))
    return st, out.reshape(bb.size, P)


def dose_batch(beams, fluence, density, volume, spectrum, kernel, extent=2.0, dense=False, repeats=1):
    """Reference Terma + CCCS (+ batched interpolation) of one batch of beamlets.
    Returns dict with terma/dens/dose [n][maxL][fy][fx], dense [n][nvox], times."""
    beams = np.ascontiguousarray(beams, BEAM_DTYPE)
    n = beams.size
    fx, fy = (int(t) for t in beams[0]["fmap_size"])
    maxL = int(beams["long_dim"].max())
    v = np.array(volume, VOLUME_DTYPE)
    nv = int(np.prod(v["dim"].astype(np.int64)))
    T = np.zeros((n, maxL, fy, fx), np.float32)
    R = np.zeros_like(T)
    D = np.zeros_like(T)
    dn = np.zeros((n, nv), np.float32) if dense else None
    tm = np.zeros(3, np.float32)
    s, k = spectrum, kernel
    st = lib().ref_dose_batch(
        C.c_int(n), _p(beams), _p(np.ascontiguousarray(fluence, np.float32)),
        _p(np.ascontiguousarray(density, np.float32)), _p(v), C.c_int(s.n), _p(s.energy), _p(s.fluence),
        _p(s.mu), _p(s.mu_en), C.c_int(k.n_theta), _p(k.theta), _p(k.A), _p(k.a), _p(k.B), _p(k.b),
        C.c_int(k.n_phi), _p(k.phi), C.c_float(extent), _p(T), _p(R), _p(D),
        _p(dn) if dense else None, _p(tm), C.c_int(repeats))
    return dict(status=st, terma=T, dens=R, dose=D, dense=dn, times_ms=tm)


def bev2pvcs(beam, bev, volume):
    b = np.array(beam, BEAM_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    nx, ny, nz = (int(t) for t in v["dim"])
    out = np.zeros((nz, ny, nx), np.float32)
    st = lib().ref_bev2pvcs(_p(b), _p(np.ascontiguousarray(bev, np.float32)), _p(v), _p(out))
    return st, out
