"""Python mirror of the reference's fluence-optimizer interface over the C ABI.

Reference names: ``IMRT::MatCSR64`` (IMRTOpt/include/IMRTDoseMat.cuh:29-69),
``eval_g`` / ``eval_grad`` (IMRTOpt/src/IMRTOptUtils.cu:74, 512),
``proxL2Onehalf_QL_gpu`` (IMRTOpt/src/IMRTOptimize_var1.cu:457-570),
``beamWeightsInit_func`` (IMRTOptimize_var1.cu:125-161),
``BOO_IMRT_L2OneHalf_gpu_QL`` and ``polish_BOO_IMRT_gpu``
(IMRTOpt/src/IMRTOptimize.cu:16-194, 391-476), ``fluenceGradInit``
(IMRTOpt/src/IMRTOptimize_var.cpp:59-180).  Vectors are torch CUDA float32
tensors; matrices are device handles.  Errors raise ``FD2Error``.
"""
import ctypes as C

import numpy as np

from . import _lib
from .api import VALUE_TYPES, _p, _stream_ptr, _torch

SCALE_AXES = {0: "none", 1: "rows", 2: "cols"}
INDEX_FORMATS = {"i32": 0, "packed16": 1}


class _MatInfo(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("nnz", C.c_int64), ("value_type", C.c_int32),
                ("scale_axis", C.c_int32), ("device_bytes", C.c_int64), ("index_format", C.c_int32),
                ("x_in_shared", C.c_int32), ("exception_chunks", C.c_int64)]


class _State(C.Structure):
    _fields_ = [("k_global", C.c_int32), ("theta_km1", C.c_float), ("tkm1", C.c_float), ("trials", C.c_int32),
                ("d_xkm1", C.c_void_p), ("d_vkm1", C.c_void_p), ("h_loss", C.c_void_p), ("h_nrm", C.c_void_p),
                ("num_active", C.c_float), ("stop", C.c_int32)]


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def _join_torch():
    """The library works on the context's own stream: let torch's pending work
    on the caller's tensors finish first."""
    _torch().cuda.current_stream().synchronize()


def _dev_f32(x):
    torch = _torch()
    if isinstance(x, torch.Tensor):
        assert x.is_cuda and x.dtype == torch.float32 and x.is_contiguous()
        return x
    return torch.as_tensor(np.ascontiguousarray(x, np.float32)).cuda()


class Matrix:
    """Device CSR (IMRT::MatCSR64): int64 offsets, int32 columns, f32/f16/bf16
    values with a per-column (or, transposed, per-row) scale for 16-bit."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    @classmethod
    def from_csr(cls, ctx, offsets, columns, values, n_cols, value_type="f32", index_format="i32"):
        off = np.ascontiguousarray(offsets, np.int64)
        col = np.ascontiguousarray(columns, np.int64)
        val = np.ascontiguousarray(values, np.float32)
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_matrix_create(ctx.h, len(off) - 1, int(n_cols), len(col), _p(off), _p(col), _p(val),
                                             VALUE_TYPES[value_type], INDEX_FORMATS[index_format], C.byref(h)),
                   "matrix_create")
        return cls(ctx, h)

    @classmethod
    def synthetic(cls, ctx, rows, cols, window, density, seed=1, value_type="f32", index_format="i32"):
        """Seeded synthetic VOI pair (A, AT) built on the device."""
        a, at = C.c_void_p(), C.c_void_p()
        _lib.check(ctx.lib.fd2_matrix_synthetic(ctx.h, rows, cols, window, density, seed, VALUE_TYPES[value_type],
                                                INDEX_FORMATS[index_format], C.byref(a), C.byref(at)),
                   "matrix_synthetic")
        return cls(ctx, a), cls(ctx, at)

    @classmethod
    def voi(cls, ctx, ensemble, voxel_row, n_voi, value_type="f32", index_format="i32"):
        """getStructFilter + parallelSpGEMM: (A, AT) of the VOI rows of a dose matrix."""
        vr = np.ascontiguousarray(voxel_row, np.int32)
        a, at = C.c_void_p(), C.c_void_p()
        _lib.check(ctx.lib.fd2_voi_matrices(ensemble.h, _p(vr), vr.size, int(n_voi), VALUE_TYPES[value_type],
                                            INDEX_FORMATS[index_format], C.byref(a), C.byref(at)), "voi_matrices")
        return cls(ctx, a), cls(ctx, at)

    def info(self):
        i = _MatInfo()
        _lib.check(self.ctx.lib.fd2_matrix_info(self.h, C.byref(i)), "matrix_info")
        fmt = {v: k for k, v in INDEX_FORMATS.items()}[i.index_format]
        return dict(rows=i.rows, cols=i.cols, nnz=i.nnz, value_type=i.value_type,
                    scale_axis=SCALE_AXES[i.scale_axis], device_bytes=i.device_bytes, index_format=fmt,
                    exception_chunks=i.exception_chunks, x_in_shared=bool(i.x_in_shared))

    @property
    def shape(self):
        i = self.info()
        return i["rows"], i["cols"]

    def to_host(self):
        i = self.info()
        off = np.zeros(i["rows"] + 1, np.int64)
        col = np.zeros(i["nnz"], np.int32)
        val = np.zeros(i["nnz"], np.float32)
        _lib.check(self.ctx.lib.fd2_matrix_to_host(self.h, _p(off), _p(col), _p(val)), "matrix_to_host")
        return off, col, val

    def transpose(self):
        h = C.c_void_p()
        _lib.check(self.ctx.lib.fd2_matrix_transpose(self.h, C.byref(h)), "matrix_transpose")
        return Matrix(self.ctx, h)

    def select_blocks(self, block_rows, order, block_cols=None):
        """Row blocks `order` of this matrix, in that order (fd2_matrix_select_blocks);
        with block_cols the columns are renumbered block by block (block-diagonal)."""
        br = np.ascontiguousarray(block_rows, np.int64)
        od = np.ascontiguousarray(order, np.int64)
        bc = None if block_cols is None else np.ascontiguousarray(block_cols, np.int64)
        h = C.c_void_p()
        _lib.check(self.ctx.lib.fd2_matrix_select_blocks(self.h, len(br) - 1, _p(br), _p(bc) if bc is not None else None,
                                                         len(od), _p(od) if od.size else None, C.byref(h)),
                   "matrix_select_blocks")
        return Matrix(self.ctx, h)

    def spmv(self, x, y=None, stream=None):
        torch = _torch()
        rows, _ = self.shape
        x = _dev_f32(x)
        if y is None:
            y = torch.empty(rows, dtype=torch.float32, device=x.device)
        _lib.check(self.ctx.lib.fd2_matrix_spmv(self.h, _ptr(x), _ptr(y), _stream_ptr(stream)), "matrix_spmv")
        return y

    def close(self):
        if self.h:
            self.ctx.lib.fd2_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fluence_grad(fluence_dim, active):
    """fluenceGradInit for one beam: (offsets, columns, values, n_active) of D_b."""
    a = np.ascontiguousarray(active, np.uint8).reshape(-1)
    n = int(fluence_dim)
    assert a.size == n * n
    off = np.zeros(2 * n * n + 1, np.int64)
    col = np.zeros(4 * n * n, np.int64)
    val = np.zeros(4 * n * n, np.float32)
    rows, nnz = C.c_int64(0), C.c_int64(0)
    _lib.check(_lib.get().fd2_fluence_grad(n, _p(a), C.byref(rows), C.byref(nnz), _p(off), _p(col), _p(val)),
               "fluence_grad")
    r, z = rows.value, nnz.value
    return off[: r + 1].copy(), col[:z].copy(), val[:z].copy(), int(a.astype(bool).sum())


def block_diag(blocks):
    """Block-diagonal CSR of (offsets, columns, values, n_cols) blocks (diagBlock,
    IMRTOpt/src/IMRTOptimize_var.cpp:317-359)."""
    offs, cols, vals = [np.zeros(1, np.int64)], [], []
    base_nnz = base_col = 0
    for off, col, val, nc in blocks:
        offs.append(np.asarray(off[1:], np.int64) + base_nnz)
        cols.append(np.asarray(col, np.int64) + base_col)
        vals.append(np.asarray(val, np.float32))
        base_nnz += len(col)
        base_col += nc
    return (np.concatenate(offs), np.concatenate(cols) if cols else np.zeros(0, np.int64),
            np.concatenate(vals) if vals else np.zeros(0, np.float32), base_col)


class Problem:
    """eval_g / eval_grad state over device matrices A (VOI x beamlets, PTV rows
    first), AT, D (fluence-gradient rows) and DT."""

    def __init__(self, ctx, A, AT, D, DT, n_ptv, n_oar, max_dose, max_weights, min_dose, min_weights, oar_weights,
                 gamma=1.0, eta=0.1):
        self.ctx = ctx
        self.mats = (A, AT, D, DT)  # kept alive with the problem
        arrs = [np.ascontiguousarray(a, np.float32) for a in (max_dose, max_weights, min_dose, min_weights,
                                                               oar_weights)]
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_opt_problem_create(ctx.h, A.h, AT.h, D.h, DT.h, int(n_ptv), int(n_oar),
                                                  *(_p(a) for a in arrs), float(gamma), float(eta), C.byref(h)),
                   "opt_problem_create")
        self.h = h
        self.n = A.shape[1]

    def eval_g(self, x):
        x = _dev_f32(x)
        _join_torch()
        v = C.c_double(0)
        _lib.check(self.ctx.lib.fd2_eval_g(self.h, _ptr(x), C.byref(v)), "eval_g")
        return v.value

    def eval_grad(self, x):
        torch = _torch()
        x = _dev_f32(x)
        g = torch.empty(self.n, dtype=torch.float32, device=x.device)
        _join_torch()
        v = C.c_double(0)
        _lib.check(self.ctx.lib.fd2_eval_grad(self.h, _ptr(x), _ptr(g), C.byref(v)), "eval_grad")
        return v.value, g

    def beam_weights_init(self, group_offsets):
        go = np.ascontiguousarray(group_offsets, np.int64)
        w = np.zeros(len(go) - 1, np.float32)
        _join_torch()
        _lib.check(self.ctx.lib.fd2_beam_weights_init(self.h, len(go) - 1, _p(go), _p(w)), "beam_weights_init")
        return w

    def _state(self, x0, step_size, iters, n_groups, state):
        torch = _torch()
        x = _dev_f32(x0).clone()
        v = x.clone() if state is None else state["v"]
        loss = np.zeros(iters, np.float32)
        nrm = np.zeros(max(n_groups, 1), np.float32)
        st = _State(0, 0.0, float(step_size), 0, x.data_ptr(), v.data_ptr(), loss.ctypes.data,
                    nrm.ctypes.data if n_groups else None, 0.0, 0)
        if state is not None:
            st.k_global, st.theta_km1, st.tkm1 = state["k"], state["theta"], state["t"]
        _join_torch()
        return st, x, v, loss, nrm

    _REDUCE = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p)

    def set_reducer(self, fn):
        """Row-sharded problem: fn(t) must replace the CUDA float64 tensor t by
        its sum over the ranks (e.g. torch.distributed.all_reduce) before it
        returns.  None restores the single-GPU problem."""
        if fn is None:
            self._reducer = None
            _lib.check(self.ctx.lib.fd2_opt_problem_set_reducer(self.h, None, None), "opt_problem_set_reducer")
            return
        torch = _torch()

        class _View:
            def __init__(self, ptr, n):
                self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                                 "version": 3, "strides": None}

        def cb(_user, ptr, n, _stream):
            try:
                fn(torch.as_tensor(_View(ptr, int(n)), device="cuda"))
                torch.cuda.current_stream().synchronize()
                return 0
            except Exception:  # reported to the solver as a failed reduction
                return 1

        self._reducer = Problem._REDUCE(cb)  # kept alive with the problem
        _lib.check(self.ctx.lib.fd2_opt_problem_set_reducer(self.h, C.cast(self._reducer, C.c_void_p), None),
                   "opt_problem_set_reducer")

    def set_graph(self, on):
        """Trials replayed from one captured CUDA graph (default) or launched one by one."""
        _lib.check(self.ctx.lib.fd2_opt_problem_set_graph(self.h, int(on)), "opt_problem_set_graph")

    def boo(self, group_offsets, beam_weights, x0, step_size, iters, prune=(), want=0, change_trigger=100,
            show=100, state=None):
        """BOO_IMRT_L2OneHalf_gpu_QL; returns the solver state and outputs."""
        go = np.ascontiguousarray(group_offsets, np.int64)
        w = np.ascontiguousarray(beam_weights, np.float32).copy()
        st, x, v, loss, nrm = self._state(x0, step_size, iters, len(go) - 1, state)
        pr = np.ascontiguousarray(prune, np.int32)
        _lib.check(self.ctx.lib.fd2_boo_l2onehalf(self.h, len(go) - 1, _p(go), _p(w), show, change_trigger, iters,
                                                  _p(pr) if pr.size else None, pr.size, want, C.byref(st)),
                   "boo_l2onehalf")
        return dict(x=x, v=v, loss=loss, nrm=nrm[: len(go) - 1], weights=w, k=st.k_global, theta=st.theta_km1,
                    t=st.tkm1, active=st.num_active, stop=bool(st.stop), trials=st.trials)

    def polish(self, x0, step_size, iters, state=None):
        """polish_BOO_IMRT_gpu."""
        st, x, v, loss, _ = self._state(x0, step_size, iters, 0, state)
        _lib.check(self.ctx.lib.fd2_polish(self.h, iters, iters, C.byref(st)), "polish")
        return dict(x=x, v=v, loss=loss, k=st.k_global, theta=st.theta_km1, t=st.tkm1, trials=st.trials)

    def close(self):
        if self.h:
            self.ctx.lib.fd2_opt_problem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def reference_x0(n, seed=10086):
    """The reference's initial fluence for the beam-orientation loop:
    std::srand(10086) then (float)std::rand() / RAND_MAX per beamlet
    (IMRTOptimize.cu:240-243), with glibc's rand() restated -- the additive
    feedback generator r[i] = r[i-3] + r[i-31] (mod 2^32) seeded through
    16807 * r mod (2^31 - 1), whose first 344 outputs are discarded and which
    returns r >> 1."""
    r = [0] * (n + 344)
    r[0] = seed & 0xFFFFFFFF
    for i in range(1, 31):
        hi, lo = divmod(int(np.int32(np.uint32(r[i - 1]))), 127773)
        word = 16807 * lo - 2836 * hi
        if word < 0:
            word += 2147483647
        r[i] = word
    for i in range(31, 34):
        r[i] = r[i - 31]
    for i in range(34, n + 344):
        r[i] = (r[i - 31] + r[i - 3]) & 0xFFFFFFFF
    out = np.array([r[i] >> 1 for i in range(344, n + 344)], np.int64)
    return (out.astype(np.float32) / np.float32(2147483647)).astype(np.float32)


class _BooParams(C.Structure):
    _fields_ = [("beam_weight", C.c_float), ("step_size", C.c_float), ("gamma", C.c_float), ("eta", C.c_float),
                ("max_iter", C.c_int32), ("change_weights_trigger", C.c_int32), ("show_trigger", C.c_int32),
                ("n_beams_want", C.c_int32), ("prune_trigger", C.c_void_p), ("n_prune", C.c_int32),
                ("reserved", C.c_int32)]


class _BooResult(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("n_active", C.c_int32), ("phases", C.c_int32), ("trials", C.c_int32)]


def beam_orientation_optimization(ctx, AT, D, beam_rows, d_rows, n_ptv, n_oar, max_dose, max_weights, min_dose,
                                  min_weights, oar_weights, x0, beam_weight=1.0, step_size=1e-3, gamma=1.0, eta=0.1,
                                  max_iter=1000, change_weights_trigger=100, show_trigger=100, n_beams_want=20,
                                  prune_trigger=()):
    """IMRT::BeamOrientationOptimization with DimReduction, on the device.

    AT: Matrix, beamlets x VOI rows of all candidate beams (beam b = rows
    beam_rows[b]:beam_rows[b+1]); D: Matrix, the block-diagonal fluence
    gradient (beam b = rows d_rows[b]:d_rows[b+1], its beamlets as columns);
    x0: initial fluence of all beamlets.  Returns the kept beams in their final
    order, their group norms and fluence, and the cost of every iteration."""
    torch = _torch()
    br = np.ascontiguousarray(beam_rows, np.int64)
    dr = np.ascontiguousarray(d_rows, np.int64)
    n_beams = len(br) - 1
    arrs = [np.ascontiguousarray(a, np.float32) for a in (max_dose, max_weights, min_dose, min_weights, oar_weights)]
    pr = np.ascontiguousarray(prune_trigger, np.int32)
    prm = _BooParams(beam_weight, step_size, gamma, eta, max_iter, change_weights_trigger, show_trigger, n_beams_want,
                     pr.ctypes.data if pr.size else None, pr.size, 0)
    x0 = _dev_f32(x0)
    x = torch.zeros_like(x0)
    costs = np.zeros(max_iter, np.float32)
    active = np.zeros(n_beams, np.int32)
    norms = np.zeros(n_beams, np.float32)
    res = _BooResult()
    _join_torch()
    _lib.check(ctx.lib.fd2_beam_orientation_optimization(
        ctx.h, AT.h, D.h, n_beams, _p(br), _p(dr), n_ptv, n_oar, *(_p(a) for a in arrs), C.byref(prm), _ptr(x0),
        _p(costs), _p(active), _p(norms), _ptr(x), C.byref(res)), "beam_orientation_optimization")
    k = res.n_active
    nx = int(sum(br[b + 1] - br[b] for b in active[:k]))
    return dict(active=active[:k].copy(), norms=norms[:k].copy(), x=x[:nx], costs=costs[:min(res.iterations + 1, max_iter)],
                costs_full=costs, iterations=res.iterations, phases=res.phases, trials=res.trials)


def final_dose(A_full, beam_rows, active, x):
    """resultDoseCalc (IMRTOptimize.cu:604-625): the dose of the kept beams'
    fluence x (concatenated in the order `active`) through the all-beam matrix
    A_full (voxels x beamlets, beam b = columns beam_rows[b]:beam_rows[b+1]);
    the pruned beams' beamlets carry zero fluence."""
    torch = _torch()
    br = np.asarray(beam_rows, np.int64)
    x = _dev_f32(x)
    full = torch.zeros(int(br[-1]), dtype=torch.float32, device=x.device)
    o = 0
    for b in np.asarray(active, np.int64):
        n = int(br[b + 1] - br[b])
        full[br[b]:br[b + 1]] = x[o:o + n]
        o += n
    assert o == x.numel(), "x does not match the kept beams"
    return A_full.spmv(full)


def dvh(ctx, dose, structures, n_bins, bin_width, stream=None):
    """Cumulative DVHs (fd2_dvh): `structures` is a list of voxel-index arrays;
    returns uint64 counts [n_structs, n_bins] of voxels receiving at least
    k * bin_width, and the same as volume fractions."""
    torch = _torch()
    dose = _dev_f32(dose)
    sizes = [len(s) for s in structures]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    vox = torch.as_tensor(np.concatenate([np.asarray(s, np.int32) for s in structures]) if structures
                          else np.zeros(0, np.int32)).to(dose.device)
    out = torch.empty((len(structures), n_bins), dtype=torch.int64, device=dose.device)
    _join_torch()
    _lib.check(ctx.lib.fd2_dvh(ctx.h, _ptr(dose), dose.numel(), len(structures), _p(off), _ptr(vox), int(n_bins),
                               float(bin_width), _ptr(out), _stream_ptr(stream)), "dvh")
    counts = out.cpu().numpy().astype(np.uint64)
    frac = counts / np.maximum(np.asarray(sizes, np.float64), 1.0)[:, None]
    return counts, frac


def prox_l2onehalf(ctx, group_offsets, g0, tau, stream=None):
    """proxL2Onehalf_QL_gpu::evaluate: (prox, new group norms) as tensors."""
    torch = _torch()
    go = torch.as_tensor(np.ascontiguousarray(group_offsets, np.int64)).cuda()
    g0 = _dev_f32(g0)
    tau = _dev_f32(tau)
    prox = torch.empty_like(g0)
    nrm = torch.empty(len(go) - 1, dtype=torch.float32, device=g0.device)
    _lib.check(ctx.lib.fd2_prox_l2onehalf(ctx.h, len(go) - 1, _ptr(go), _ptr(g0), _ptr(tau), _ptr(prox), _ptr(nrm),
                                          _stream_ptr(stream)), "prox_l2onehalf")
    return prox, nrm
