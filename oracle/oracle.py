"""ctypes bindings of the C oracle (fd_oracle.c) plus numpy conveniences.

Test infrastructure only (see __init__.py).  `lib(precision)` loads the double
build (parity) or the float build (timed CPU baseline); both are built by
oracle/Makefile (`build()` below runs it).
"""
import ctypes as C
import os
import subprocess
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from fastdose_b200.types import BEAM_DTYPE, BUNDLE_DTYPE, VOLUME_DTYPE

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

_fp = C.POINTER(C.c_float)
_vp = C.c_void_p
_i64p = C.POINTER(C.c_int64)


def build():
    """Compile both oracle builds with make (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(precision="double"):
    name = "liboracle64.so" if precision == "double" else "liboracle32.so"
    if name not in _LIBS:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.or_calc_range.restype = C.c_int
        L.or_beamlet_init.restype = C.c_int
        L.or_calc_line_seg.restype = C.c_double
        L.or_eval_g.restype = C.c_double
        L.or_eval_grad.restype = C.c_double
        L.or_that.restype = C.c_double
        L.or_that.argtypes = [C.c_double, C.c_double]
        L.or_rotate_axis_f.argtypes = [_fp, _fp, C.c_float, _fp]
        L.or_rotate_beam_f.argtypes = [_fp, C.c_float, C.c_float, C.c_float, _fp]
        L.or_inv_rotate_beam_f.argtypes = [_fp, C.c_float, C.c_float, C.c_float, _fp]
        _LIBS[name] = L
    return _LIBS[name]


def _p(a):
    return a.ctypes.data_as(_vp)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


# ------------------------------------------------------------------ geometry
def rotate_axis(p, r, t):
    p, r = _f32(p), _f32(r)
    o = np.zeros(3, np.float32)
    lib().or_rotate_axis_f(p.ctypes.data_as(_fp), r.ctypes.data_as(_fp), C.c_float(t), o.ctypes.data_as(_fp))
    return o


def rotate_beam(v, theta, phi, coll):
    v = _f32(v)
    o = np.zeros(3, np.float32)
    lib().or_rotate_beam_f(v.ctypes.data_as(_fp), theta, phi, coll, o.ctypes.data_as(_fp))
    return o


def inv_rotate_beam(v, theta, phi, coll):
    v = _f32(v)
    o = np.zeros(3, np.float32)
    lib().or_inv_rotate_beam_f(v.ctypes.data_as(_fp), theta, phi, coll, o.ctypes.data_as(_fp))
    return o


def calc_range(beam, volume):
    b = np.array(beam, BEAM_DTYPE).copy()
    v = np.array(volume, VOLUME_DTYPE)
    st = lib().or_calc_range(_p(b), _p(v))
    return st, b


def beamlet_init(bundle, ix, iy, volume):
    out = np.zeros((), BEAM_DTYPE)
    bb = np.array(bundle, BUNDLE_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    st = lib().or_beamlet_init(_p(bb), C.c_int(ix), C.c_int(iy), _p(v), _p(out))
    return st, out


def beamlet_fluence(bundle):
    bb = np.array(bundle, BUNDLE_DTYPE)
    fx, fy = (int(v) for v in bb["sub_fluence_dim"])
    out = np.zeros(fx * fy, np.float32)
    lib().or_beamlet_fluence(_p(bb), _p(out))
    return out


def next_point(c, d):
    c = np.ascontiguousarray(c, np.float64)
    d = np.ascontiguousarray(d, np.float64)
    o = np.zeros(3, np.float64)
    f = C.c_int(0)
    lib().or_next_point(_p(c), _p(d), _p(o), C.byref(f))
    return o, bool(f.value)


def calc_line_seg(s, e, beam):
    s = np.ascontiguousarray(s, np.float64)
    e = np.ascontiguousarray(e, np.float64)
    b = np.array(beam, BEAM_DTYPE)
    return lib().or_calc_line_seg(_p(s), _p(e), _p(b))


def beamlet_flags(beams, ptv_mask, volume, super_sampling=3, tex_mode=0, precision="double"):
    beams = np.ascontiguousarray(beams, BEAM_DTYPE)
    m = np.ascontiguousarray(ptv_mask, np.uint8)
    v = np.array(volume, VOLUME_DTYPE)
    P = int(beams[0]["fmap_size"][0]) * int(beams[0]["fmap_size"][1])
    out = np.zeros(beams.size * P, np.uint8)
    lib(precision).or_beamlet_flags(C.c_size_t(beams.size), _p(beams), _p(m), _p(v), C.c_int(super_sampling),
                                    C.c_int(tex_mode), _p(out))
    return out.reshape(beams.size, P)


# ------------------------------------------------------------------ dose calc
def _bev_shape(beam):
    fx, fy = (int(v) for v in beam["fmap_size"])
    return int(beam["long_dim"]), fy, fx


def terma(beam, fluence, density, volume, spectrum, tex_mode=0, precision="double"):
    b = np.array(beam, BEAM_DTYPE).copy()
    L, fy, fx = _bev_shape(b)
    b["TermaBEV_pitch"] = b["DensityBEV_pitch"] = fx * fy * 4
    T = np.zeros((L, fy, fx), np.float32)
    R = np.zeros((L, fy, fx), np.float32)
    dens = np.ascontiguousarray(density, np.float32)
    v = np.array(volume, VOLUME_DTYPE)
    lib(precision).or_terma(_p(b), _p(_f32(fluence)), _p(dens), _p(v), C.c_int(spectrum.n),
                            _p(spectrum.energy), _p(spectrum.fluence), _p(spectrum.mu), C.c_int(tex_mode),
                            _p(T), _p(R))
    return T, R


def cccs(beam, terma_bev, dens_bev, kernel, dose=None, precision="double", dirs=None):
    """CCCS of one beam.  `dirs` (optional, float32 [n_fwd][n_phi][4]) supplies
    the cone directions; by default they are evaluated in double precision."""
    b = np.array(beam, BEAM_DTYPE).copy()
    L, fy, fx = _bev_shape(b)
    b["TermaBEV_pitch"] = b["DensityBEV_pitch"] = fx * fy * 4
    D = np.zeros((L, fy, fx), np.float32) if dose is None else np.ascontiguousarray(dose, np.float32).copy()
    k = kernel
    dp = _p(np.ascontiguousarray(dirs, np.float32)) if dirs is not None else None
    lib(precision).or_cccs_dirs(_p(b), _p(_f32(terma_bev)), _p(_f32(dens_bev)), C.c_int(k.n_theta), _p(k.theta),
                                _p(k.A), _p(k.a), _p(k.B), _p(k.b), C.c_int(k.n_phi), _p(k.phi), dp, _p(D))
    return D


def bev2pvcs(beam, bev, volume, tex_mode=0, precision="double"):
    b = np.array(beam, BEAM_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    nx, ny, nz = (int(t) for t in v["dim"])
    out = np.zeros((nz, ny, nx), np.float32)
    lib(precision).or_bev2pvcs(_p(b), _p(_f32(bev)), _p(v), C.c_int(tex_mode), _p(out))
    return out


def bev2pvcs_ss(beam, bev, volume, ssfactor=5, extent=2.0, tex_mode=0, out=None, precision="double"):
    b = np.array(beam, BEAM_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    nx, ny, nz = (int(t) for t in v["dim"])
    o = np.zeros((nz, ny, nx), np.float32) if out is None else np.ascontiguousarray(out, np.float32).copy()
    lib(precision).or_bev2pvcs_ss(_p(b), _p(_f32(bev)), _p(v), C.c_int(ssfactor), C.c_float(extent),
                                  C.c_int(tex_mode), _p(o))
    return o


def beamlet_column(beam, dose_bev, volume, ssfactor=5, extent=2.0, precision="double"):
    b = np.array(beam, BEAM_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    nx, ny, nz = (int(t) for t in v["dim"])
    row = np.zeros(nx * ny * nz, np.float32)
    lib(precision).or_beamlet_column(_p(b), _p(_f32(dose_bev)), _p(v), C.c_int(ssfactor), C.c_float(extent),
                                     _p(row))
    return row


def beamlet_pipeline(beam, fluence, density, volume, spectrum, kernel, ssfactor=5, extent=2.0,
                     precision="double"):
    """Terma -> CCCS -> column of one beamlet, returns the dense row."""
    b = np.array(beam, BEAM_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    nx, ny, nz = (int(t) for t in v["dim"])
    row = np.zeros(nx * ny * nz, np.float32)
    s, k = spectrum, kernel
    lib(precision).or_beamlet_pipeline(
        _p(b), _p(_f32(fluence)), _p(np.ascontiguousarray(density, np.float32)), _p(v), C.c_int(s.n),
        _p(s.energy), _p(s.fluence), _p(s.mu), C.c_int(k.n_theta), _p(k.theta), _p(k.A), _p(k.a), _p(k.B),
        _p(k.b), C.c_int(k.n_phi), _p(k.phi), C.c_int(ssfactor), C.c_float(extent), _p(row))
    return row


def dose_rows(beams, fluence, density, volume, spectrum, kernel, ssfactor=5, extent=2.0,
              precision="double", threads=1):
    """Dense [n_beamlets][n_voxels] dose matrix of a beamlet list; beamlets run
    on `threads` host threads (ctypes releases the GIL during the C call)."""
    beams = np.ascontiguousarray(beams, BEAM_DTYPE)
    dens = np.ascontiguousarray(density, np.float32)

    def one(i):
        return beamlet_pipeline(beams[i], fluence, dens, volume, spectrum, kernel, ssfactor, extent, precision)

    if threads <= 1:
        rows = [one(i) for i in range(beams.size)]
    else:
        with ThreadPoolExecutor(threads) as ex:
            rows = list(ex.map(one, range(beams.size)))
    return np.stack(rows)


def dense_to_csr(dense):
    """cusparseDenseToSparse semantics on a row-major matrix: entries != 0 in
    row-major order (IMRTOpt/src/IMRTSparseMatEns.cu:66-165)."""
    dense = np.asarray(dense)
    nz = dense != 0
    counts = nz.sum(axis=1)
    offsets = np.zeros(dense.shape[0] + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    r, c = np.nonzero(nz)
    return offsets, c.astype(np.int64), dense[r, c].astype(np.float32)


# ------------------------------------------------------------------ optimizer
class _CSR(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("nnz", C.c_int64), ("offsets", _vp),
                ("columns", _vp), ("values", _vp)]


class _Problem(C.Structure):
    _fields_ = [("A", _CSR), ("AT", _CSR), ("D", _CSR), ("DT", _CSR), ("n_ptv", C.c_int64), ("n_oar", C.c_int64),
                ("max_dose", _vp), ("max_weights", _vp), ("min_dose", _vp), ("min_weights", _vp),
                ("oar_weights", _vp), ("gamma", C.c_float), ("eta", C.c_float)]


class _State(C.Structure):
    _fields_ = [("k_global", C.c_int), ("theta_km1", C.c_float), ("tkm1", C.c_float), ("xkm1", _vp),
                ("vkm1", _vp), ("loss", _vp), ("nrm", _vp), ("num_active", C.c_float), ("stop", C.c_int),
                ("trials", C.c_int)]


def _csr_struct(m, keep):
    off = np.ascontiguousarray(m[0], np.int64)
    col = np.ascontiguousarray(m[1], np.int64)
    val = np.ascontiguousarray(m[2], np.float32)
    keep += [off, col, val]
    return _CSR(len(off) - 1, int(m[3]), len(col), _p(off), _p(col), _p(val))


def csr_transpose(m):
    """Transpose of (offsets, columns, values, n_cols) with sorted columns."""
    off, col, val, ncols = m
    rows = np.repeat(np.arange(len(off) - 1, dtype=np.int64), np.diff(off))
    order = np.lexsort((rows, col))
    t_off = np.zeros(ncols + 1, np.int64)
    np.cumsum(np.bincount(col, minlength=ncols), out=t_off[1:])
    return t_off, rows[order], val[order].astype(np.float32), len(off) - 1


class Problem:
    """Optimizer inputs: A (VOI x beamlets), D (fluence-gradient rows), weights."""

    def __init__(self, A, D, n_ptv, n_oar, max_dose, max_weights, min_dose, min_weights, oar_weights,
                 gamma, eta, precision="double", AT=None):
        self.keep = []
        self.A, self.D = A, D
        AT = csr_transpose(A) if AT is None else AT
        DT = csr_transpose(D)
        self.n = A[3]
        arrs = [np.ascontiguousarray(a, np.float32) for a in (max_dose, max_weights, min_dose, min_weights,
                                                               oar_weights)]
        self.keep += arrs
        self.s = _Problem(_csr_struct(A, self.keep), _csr_struct(AT, self.keep), _csr_struct(D, self.keep),
                          _csr_struct(DT, self.keep), n_ptv, n_oar, *(_p(a) for a in arrs), gamma, eta)
        self.L = lib(precision)

    def eval_g(self, x):
        x = _f32(x)
        return self.L.or_eval_g(C.byref(self.s), _p(x))

    def eval_grad(self, x):
        x = _f32(x)
        g = np.zeros(self.n, np.float32)
        v = self.L.or_eval_grad(C.byref(self.s), _p(x), _p(g))
        return v, g

    def boo(self, group_offsets, beam_weights, x0, step_size, iters, prune=(), want=0,
            change_trigger=100, show=100, state=None, loss=None):
        """state: (k_global, theta_km1, tkm1, v) carried from an earlier call;
        loss: the [iters] cost array to fill at the iterations run."""
        go = np.ascontiguousarray(group_offsets, np.int64)
        w = _f32(beam_weights).copy()
        x = _f32(x0).copy()
        v = x.copy() if state is None else _f32(state[3]).copy()
        loss = np.zeros(iters, np.float32) if loss is None else loss
        nrm = np.zeros(len(go) - 1, np.float32)
        k0, th0, t0 = (0, 0.0, step_size) if state is None else state[:3]
        st = _State(k0, th0, t0, _p(x), _p(v), _p(loss), _p(nrm), 0.0, 0, 0)
        pr = np.ascontiguousarray(prune, np.int32)
        self.L.or_boo_l2onehalf(C.byref(self.s), C.c_int64(len(go) - 1), _p(go), _p(w), C.c_int(show),
                                C.c_int(change_trigger), C.c_int(iters), _p(pr), C.c_int(pr.size), C.c_int(want),
                                C.byref(st))
        return dict(x=x, v=v, loss=loss[: st.k_global + (0 if st.stop and st.k_global < iters else 0)],
                    nrm=nrm, weights=w, k=st.k_global, theta=st.theta_km1, t=st.tkm1, active=st.num_active,
                    stop=bool(st.stop), trials=st.trials, loss_full=loss)

    def polish(self, x0, step_size, iters):
        x = _f32(x0).copy()
        v = x.copy()
        loss = np.zeros(iters, np.float32)
        st = _State(0, 0.0, step_size, _p(x), _p(v), _p(loss), None, 0.0, 0, 0)
        self.L.or_polish(C.byref(self.s), C.c_int(iters), C.c_int(iters), C.byref(st))
        return dict(x=x, v=v, loss=loss, k=st.k_global, theta=st.theta_km1, t=st.tkm1, trials=st.trials)


def prox_l2onehalf(group_offsets, g0, tau, precision="double"):
    go = np.ascontiguousarray(group_offsets, np.int64)
    g0 = _f32(g0)
    tau = _f32(tau)
    prox = np.zeros_like(g0)
    nrm = np.zeros(len(go) - 1, np.float32)
    lib(precision).or_prox_l2onehalf(C.c_int64(len(go) - 1), _p(go), _p(g0), _p(tau), _p(prox), _p(nrm))
    return prox, nrm


def that(nrm2, tau):
    return lib().or_that(float(nrm2), float(tau))


def fluence_grad(fluence_dim, active):
    a = np.ascontiguousarray(active, np.uint8)
    n = fluence_dim
    off = np.zeros(2 * n * n + 1, np.int64)
    col = np.zeros(4 * n * n, np.int64)
    val = np.zeros(4 * n * n, np.float32)
    rows, nnz = C.c_int64(0), C.c_int64(0)
    lib().or_fluence_grad(C.c_int(n), _p(a), C.byref(rows), C.byref(nnz), _p(off), _p(col), _p(val))
    r, z = rows.value, nnz.value
    return off[: r + 1].copy(), col[:z].copy(), val[:z].copy(), int(a.astype(bool).sum())


def beam_weights_init(A_blocks, n_ptv):
    keep = []
    arr = (_CSR * len(A_blocks))(*[_csr_struct(m, keep) for m in A_blocks])
    out = np.zeros(len(A_blocks), np.float32)
    lib().or_beam_weights_init(C.c_int64(len(A_blocks)), arr, C.c_int64(n_ptv), _p(out))
    return out
