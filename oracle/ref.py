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


def bev2pvcs_ss(beam, bev, volume, ssfactor=5, extent=2.0):
    """fd::BEV2PVCS_SuperSampling (geom.cu:343-474) through a linear-filter texture."""
    b = np.array(beam, BEAM_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    nx, ny, nz = (int(t) for t in v["dim"])
    out = np.zeros((nz, ny, nx), np.float32)
    L = lib()
    L.ref_bev2pvcs_ss.argtypes = [C.c_void_p] * 3 + [C.c_int, C.c_float, C.c_void_p]
    st = L.ref_bev2pvcs_ss(_p(b), _p(np.ascontiguousarray(bev, np.float32)), _p(v), ssfactor, extent, _p(out))
    return st, out


def dose_mat_steps(bundles, flags, density, volume, spectrum, kernel, extent=2.0, est_nnz_per_mat=6_000_000):
    """IMRT::DoseMatConstruction's per-beam steps (Terma, CCCS, BEV2PVCSInterp,
    addMat) over whole bundles; see ref_dose_mat_steps in ref_harness.cu.
    Returns status, per-bundle nnz, the step times in ms and the beamlet count."""
    bb = np.ascontiguousarray(bundles, BUNDLE_DTYPE)
    fl = np.ascontiguousarray(flags, np.uint8)
    v = np.array(volume, VOLUME_DTYPE)
    nnz = np.zeros(bb.size, np.uint64)
    tm = np.zeros(5, np.float32)
    nb = C.c_int64(0)
    s, k = spectrum, kernel
    L = lib()
    L.ref_dose_mat_steps.argtypes = [C.c_int] + [C.c_void_p] * 4 + [C.c_int] + [C.c_void_p] * 4 + \
        [C.c_int] + [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_float, C.c_uint64] + [C.c_void_p] * 3
    st = L.ref_dose_mat_steps(bb.size, _p(bb), _p(fl), _p(np.ascontiguousarray(density, np.float32)), _p(v),
                              s.n, _p(s.energy), _p(s.fluence), _p(s.mu), _p(s.mu_en), k.n_theta, _p(k.theta),
                              _p(k.A), _p(k.a), _p(k.B), _p(k.b), k.n_phi, _p(k.phi), extent, est_nnz_per_mat,
                              _p(nnz), _p(tm), C.byref(nb))
    return dict(status=st, nnz=nnz, times_ms=tm, beamlets=nb.value)


# ---------------------------------------------------------------- optimizer
# The reference's GPU optimizer (IMRTOptUtils.cu, IMRTOptimize_var1.cu and the
# solver bodies of IMRTOptimize.cu) through oracle/ref/opt_harness.cu.  CSR
# matrices are (offsets, columns, values, n_cols) tuples as the oracle takes.

class _RefCsr(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("nnz", C.c_int64), ("offsets", C.c_void_p),
                ("columns", C.c_void_p), ("values", C.c_void_p)]


def _csr(m, keep):
    off = np.ascontiguousarray(m[0], np.int64)
    col = np.ascontiguousarray(m[1], np.int64)
    val = np.ascontiguousarray(m[2], np.float32)
    keep += [off, col, val]
    return _RefCsr(len(off) - 1, int(m[3]), len(col), _p(off), _p(col), _p(val))


def _transpose(m):
    off, col, val, ncols = m
    rows = np.repeat(np.arange(len(off) - 1, dtype=np.int64), np.diff(off))
    order = np.lexsort((rows, col))
    t_off = np.zeros(ncols + 1, np.int64)
    np.cumsum(np.bincount(col, minlength=ncols), out=t_off[1:])
    return t_off, rows[order], np.asarray(val, np.float32)[order], len(off) - 1


def _opt_lib():
    L = lib()
    if not getattr(L, "_opt_ready", False):
        L.ref_opt_problem_create.restype = C.c_void_p
        L.ref_opt_problem_create.argtypes = [C.c_void_p] * 4 + [C.c_int64, C.c_int64] + [C.c_void_p] * 5 + \
            [C.c_float, C.c_float]
        L.ref_opt_problem_destroy.argtypes = [C.c_void_p]
        L.ref_opt_eval_g.argtypes = [C.c_void_p] * 3
        L.ref_opt_eval_grad.argtypes = [C.c_void_p] * 4
        L.ref_opt_prox.argtypes = [C.c_int64, C.c_int64] + [C.c_void_p] * 5
        L.ref_opt_beam_weights.argtypes = [C.c_int64, C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p]
        L.ref_opt_boo.argtypes = [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                  C.c_int, C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 9
        L.ref_opt_polish.argtypes = [C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 6
        L.ref_opt_dim_reduction.argtypes = [C.c_int, C.c_void_p, C.c_int] + [C.c_void_p] * 4 + \
            [C.c_int64, C.c_void_p, C.c_int] + [C.c_void_p] * 4
        L.ref_opt_rand01.argtypes = [C.c_uint, C.c_int, C.c_int64, C.c_void_p]
        L._opt_ready = True
    return L


class OptProblem:
    """A, D (CSR tuples) and the weights on the device as the reference holds
    them: MatCSR64 with 64-bit indices for A, Aᵀ, D, Dᵀ (Aᵀ and Dᵀ formed here
    as IMRTEigenLoad's transposes do)."""

    def __init__(self, A, D, n_ptv, n_oar, max_dose, max_weights, min_dose, min_weights, oar_weights, gamma, eta,
                 AT=None, DT=None):
        self.L = _opt_lib()
        self.keep = []
        self.n = int(A[3])
        arrs = [np.ascontiguousarray(a, np.float32) for a in (max_dose, max_weights, min_dose, min_weights,
                                                               oar_weights)]
        self.keep += arrs
        AT = _transpose(A) if AT is None else AT
        DT = _transpose(D) if DT is None else DT
        cs = [_csr(m, self.keep) for m in (A, AT, D, DT)]
        self.keep += cs
        self.h = self.L.ref_opt_problem_create(*(C.byref(c) for c in cs), n_ptv, n_oar, *(_p(a) for a in arrs),
                                               gamma, eta)
        if not self.h:
            raise RuntimeError("ref_opt_problem_create failed")

    def close(self):
        if self.h:
            self.L.ref_opt_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def eval_g(self, x):
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(1, np.float32)
        assert self.L.ref_opt_eval_g(self.h, _p(x), _p(out)) == 0
        return float(out[0])

    def eval_grad(self, x):
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(1, np.float32)
        g = np.zeros(self.n, np.float32)
        assert self.L.ref_opt_eval_grad(self.h, _p(x), _p(out), _p(g)) == 0
        return float(out[0]), g

    def boo(self, masks, beam_weights, x0, v0, step_size, iters, prune=(), want=0, change_trigger=100,
            show_trigger=1 << 30, state=None, loss=None):
        """One call of BOO_IMRT_L2OneHalf_gpu_QL.  masks: [n_beams][pixels]
        fluence maps of the phase's beams; state: (k_global, theta_km1, tkm1)."""
        masks = np.ascontiguousarray(masks, np.uint8)
        w = np.ascontiguousarray(beam_weights, np.float32).copy()
        x = np.ascontiguousarray(x0, np.float32).copy()
        v = np.ascontiguousarray(v0, np.float32).copy()
        loss = np.zeros(iters, np.float32) if loss is None else loss
        nrm = np.zeros(masks.shape[0], np.float32)
        k0, th0, t0 = (0, 0.0, step_size) if state is None else state
        k, th, t = C.c_int(k0), C.c_float(th0), C.c_float(t0)
        act, stop = C.c_float(0), C.c_int(0)
        pr = np.ascontiguousarray(prune, np.int32)
        rc = self.L.ref_opt_boo(self.h, masks.shape[0], masks.shape[1], _p(masks), _p(w), show_trigger,
                                change_trigger, iters, _p(pr) if pr.size else None, pr.size, want, C.byref(k),
                                C.byref(th), C.byref(t), _p(x), _p(v), _p(loss), _p(nrm), C.byref(act),
                                C.byref(stop))
        assert rc == 0, rc
        return dict(x=x, v=v, weights=w, loss=loss, nrm=nrm, k=k.value, theta=th.value, t=t.value,
                    active=act.value, stop=bool(stop.value))

    def polish(self, x0, v0, step_size, iters, state=None, loss=None):
        x = np.ascontiguousarray(x0, np.float32).copy()
        v = np.ascontiguousarray(v0, np.float32).copy()
        loss = np.zeros(iters, np.float32) if loss is None else loss
        k0, th0, t0 = (0, 0.0, step_size) if state is None else state
        k, th, t = C.c_int(k0), C.c_float(th0), C.c_float(t0)
        assert self.L.ref_opt_polish(self.h, iters, iters, C.byref(k), C.byref(th), C.byref(t), _p(x), _p(v),
                                     _p(loss)) == 0
        return dict(x=x, v=v, loss=loss, k=k.value, theta=th.value, t=t.value)


def opt_prox(masks, g0, tau):
    """proxL2Onehalf_QL_gpu on the beam x pixel operator of masks."""
    L = _opt_lib()
    masks = np.ascontiguousarray(masks, np.uint8)
    g0 = np.ascontiguousarray(g0, np.float32)
    tau = np.ascontiguousarray(tau, np.float32)
    prox = np.zeros_like(g0)
    nrm = np.zeros(masks.shape[0], np.float32)
    assert L.ref_opt_prox(masks.shape[0], masks.shape[1], _p(masks), _p(g0), _p(tau), _p(prox), _p(nrm)) == 0
    return prox, nrm


def opt_beam_weights(blocks, n_ptv, n_oar):
    """beamWeightsInit_func, host (Eigen) form and cuSPARSE form."""
    L = _opt_lib()
    keep = []
    arr = (_RefCsr * len(blocks))(*[_csr(m, keep) for m in blocks])
    host = np.zeros(len(blocks), np.float32)
    gpu = np.zeros(len(blocks), np.float32)
    assert L.ref_opt_beam_weights(len(blocks), arr, n_ptv, n_oar, _p(host), _p(gpu)) == 0
    return host, gpu


def opt_dim_reduction(active, beam_cols, weights, x, v, nrm, n_keep):
    """DimReduction: the kept beams (strongest first), their weights, x and v."""
    L = _opt_lib()
    act = np.ascontiguousarray(active, np.int32).copy()
    bc = np.ascontiguousarray(beam_cols, np.int64)
    w = np.ascontiguousarray(weights, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    v = np.ascontiguousarray(v, np.float32)
    nrm = np.ascontiguousarray(nrm, np.float32)
    w_out = np.zeros(len(act), np.float32)
    x_out = np.zeros(len(x), np.float32)
    v_out = np.zeros(len(x), np.float32)
    kept = C.c_int(0)
    assert L.ref_opt_dim_reduction(len(act), _p(act), len(bc), _p(bc), _p(w), _p(x), _p(v), len(x), _p(nrm),
                                   int(n_keep), _p(w_out), _p(x_out), _p(v_out), C.byref(kept)) == 0
    k = kept.value
    nx = int(sum(bc[b] for b in act[:k]))
    return act[:k].copy(), w_out[:k].copy(), x_out[:nx].copy(), v_out[:nx].copy()


def opt_rand01(n, seed=10086, reseed=True):
    """(float)rand() / RAND_MAX from this host's C library, after srand(seed)."""
    out = np.zeros(n, np.float32)
    _opt_lib().ref_opt_rand01(seed, int(reseed), n, _p(out))
    return out
