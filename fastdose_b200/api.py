"""Python mirror of the reference's planning interface over the C ABI.

Names follow the reference: ``TermaComputeCollective`` / ``DoseComputeCollective``
(FastDoseLib/src/TermaComp.cu:153, DoseComp.cu:179), ``BEV2PVCS``
(TermaComp.cu:97), ``DoseMatConstruction`` (IMRTOpt/src/IMRTDoseMat.cu:14),
``beamletFlagInit`` (IMRTOpt/src/IMRTBeamBundle.cu:130) and
``MatCSREnsemble.tofile/fromfile`` (IMRTOpt/src/IMRTSparseMatEns.cu:168,242).
Errors raise ``FD2Error`` (the reference returns 1 or exits).  Device memory is
allocated with torch; streams are torch streams.
"""
import ctypes as C

import numpy as np

from . import _lib
from .types import BEAM_DTYPE, BUNDLE_DTYPE, VOLUME_DTYPE

_p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731


def _torch():
    import torch

    return torch


def _stream_ptr(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


# ------------------------------------------------------------------ geometry
def calc_range(beam, volume):
    """BEAM_h::calc_range (FastDoseLib/src/beam.cu:134): returns an updated copy."""
    b = np.array(beam, BEAM_DTYPE).copy()
    v = np.array(volume, VOLUME_DTYPE)
    _lib.check(_lib.get().fd2_beam_calc_range(_p(b), _p(v)), "calc_range")
    return b


def beamlet_init(bundle, ix, iy, volume):
    """BeamBundle::beamletInit (IMRTOpt/src/IMRTBeamBundle.cu:341)."""
    out = np.zeros((), BEAM_DTYPE)
    bb = np.array(bundle, BUNDLE_DTYPE)
    v = np.array(volume, VOLUME_DTYPE)
    _lib.check(_lib.get().fd2_beamlet_init(_p(bb), ix, iy, _p(v), _p(out)), "beamlet_init")
    return out


def beamlet_fluence(bundle):
    bb = np.array(bundle, BUNDLE_DTYPE)
    n = int(bb["sub_fluence_dim"][0]) * int(bb["sub_fluence_dim"][1])
    out = np.zeros(n, np.float32)
    _lib.check(_lib.get().fd2_beamlet_fluence(_p(bb), _p(out), n), "beamlet_fluence")
    return out


def bundle_beamlets(bundle, flags, volume):
    """BeamBundle::beamletsInit (IMRTBeamBundle.cu:319): canonical sub-beams of
    the flagged pixels in raster order (y outer, x inner)."""
    bb = np.array(bundle, BUNDLE_DTYPE)
    fx, fy = (int(v) for v in bb["fluence_dim"])
    flags = np.asarray(flags).reshape(fy, fx)
    out = [beamlet_init(bb, ix, iy, volume) for iy in range(fy) for ix in range(fx) if flags[iy, ix]]
    return np.array(out, BEAM_DTYPE)


def bundles_beamlets(bundles, flags, volume, threads=0):
    """bundle_beamlets for many bundles in one native call over host threads:
    a list of BEAM_DTYPE arrays, one per bundle (the same beams, bit for bit)."""
    bb = np.ascontiguousarray(bundles, BUNDLE_DTYPE).reshape(-1)
    fl = np.ascontiguousarray(np.concatenate([np.asarray(f, np.uint8).reshape(-1) for f in flags])
                              if len(flags) else np.zeros(0, np.uint8))
    total = int(np.count_nonzero(fl))
    out = np.zeros(max(total, 1), BEAM_DTYPE)
    counts = np.zeros(max(bb.size, 1), np.uint32)
    v = np.array(volume, VOLUME_DTYPE)
    _lib.check(_lib.get().fd2_bundles_beamlets(bb.size, _p(bb), _p(fl), _p(v), int(threads), out.size, _p(out),
                                               _p(counts)), "bundles_beamlets")
    res, o = [], 0
    for c in counts[:bb.size]:
        res.append(out[o:o + int(c)].copy())
        o += int(c)
    return res


# ------------------------------------------------------------------ handles
class Context:
    def __init__(self, device=0):
        self.lib = _lib.get()
        h = C.c_void_p()
        _lib.check(self.lib.fd2_context_create(device, C.byref(h)), "context_create")
        self.h = h
        self.device = device

    def synchronize(self):
        _lib.check(self.lib.fd2_context_synchronize(self.h), "context_synchronize")

    def release(self):
        """Return the context's idle device memory (fd2_context_release)."""
        _lib.check(self.lib.fd2_context_release(self.h), "context_release")

    STAGES = ("terma", "cccs", "columns", "opt_spmv", "opt_other")

    def tuned_schedules(self):
        """The CCCS schedules the construction tuned: ({shape key: schedule}, tuning runs)."""
        cap = 256
        keys = (C.c_uint64 * cap)()
        sch = (C.c_int32 * cap)()
        n, runs = C.c_size_t(0), C.c_uint64(0)
        _lib.check(self.lib.fd2_context_tuned_schedules(self.h, cap, keys, sch, C.byref(n), C.byref(runs)),
                   "tuned_schedules")
        return {int(keys[i]): int(sch[i]) for i in range(min(n.value, cap))}, int(runs.value)

    def set_timing(self, on=True):
        _lib.check(self.lib.fd2_context_set_timing(self.h, int(on)), "set_timing")

    def stage_times(self):
        """Accumulated device ms per stage since the last call (then reset)."""
        out = np.zeros(len(self.STAGES), np.float64)
        _lib.check(self.lib.fd2_context_stage_times(self.h, _p(out), len(out)), "stage_times")
        return dict(zip(self.STAGES, out.tolist()))

    def launch_count(self):
        return int(self.lib.fd2_context_launch_count(self.h))

    def graph_counts(self):
        """Graph-captured construction: (batches launched as graphs, executable
        graphs instantiated, in-place updates)."""
        v = [C.c_uint64(0) for _ in range(3)]
        _lib.check(self.lib.fd2_context_graph_counts(self.h, *(C.byref(x) for x in v)), "graph_counts")
        return tuple(int(x.value) for x in v)

    def close(self):
        if self.h:
            self.lib.fd2_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Density:
    """density_h2d (FastDoseLib/src/density.cu:23): device copy of the volume."""

    def __init__(self, ctx, density, volume):
        self.ctx = ctx
        self.volume = np.array(volume, VOLUME_DTYPE)
        d = np.ascontiguousarray(density, np.float32)
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_density_create(ctx.h, _p(d), _p(self.volume), C.byref(h)), "density_create")
        self.h = h

    def close(self):
        if self.h:
            self.ctx.lib.fd2_density_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Spectrum:
    """SPECTRUM_h::bind_spectrum (FastDoseLib/src/TermaComp.cu:67)."""

    def __init__(self, ctx, spectrum):
        self.ctx = ctx
        self.src = spectrum
        a = [np.ascontiguousarray(x, np.float32) for x in (spectrum.energy, spectrum.fluence, spectrum.mu,
                                                           spectrum.mu_en)]
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_spectrum_create(ctx.h, spectrum.n, *(_p(x) for x in a), C.byref(h)),
                   "spectrum_create")
        self.h = h

    def close(self):
        if self.h:
            self.ctx.lib.fd2_spectrum_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Kernel:
    """KERNEL_h::bind_kernel (FastDoseLib/src/DoseComp.cu:25)."""

    def __init__(self, ctx, kernel):
        self.ctx = ctx
        self.src = kernel
        k = kernel
        arrs = [np.ascontiguousarray(x, np.float32) for x in (k.theta, k.A, k.a, k.B, k.b, k.phi)]
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_kernel_create(ctx.h, k.n_theta, *(_p(x) for x in arrs[:5]), k.n_phi, _p(arrs[5]),
                                             C.byref(h)), "kernel_create")
        self.h = h

    def close(self):
        if self.h:
            self.ctx.lib.fd2_kernel_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ BEV stages
class BEVBatch:
    """Device BEV buffers of a batch of beams: Terma, density and dose, each
    [beam][long_dim][fy][fx] packed with pitch fy*fx floats (the IMRT layout)."""

    def __init__(self, beams, device="cuda"):
        torch = _torch()
        self.beams = np.ascontiguousarray(beams, BEAM_DTYPE).copy()
        fx, fy = (int(v) for v in self.beams[0]["fmap_size"])
        self.P = fx * fy
        self.shape2 = (fy, fx)
        self.beams["TermaBEV_pitch"] = self.P * 4
        self.beams["DensityBEV_pitch"] = self.P * 4
        L = self.beams["long_dim"].astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(L * self.P)])
        n = int(self.offsets[-1])
        self.terma = torch.zeros(n, dtype=torch.float32, device=device)
        self.dens = torch.zeros(n, dtype=torch.float32, device=device)
        self.dose = torch.zeros(n, dtype=torch.float32, device=device)
        self.d_beams = torch.from_numpy(self.beams.view(np.uint8).copy()).to(device)
        self._ptrs = {}
        for name in ("terma", "dens", "dose"):
            base = getattr(self, name).data_ptr()
            arr = np.array([base + 4 * int(o) for o in self.offsets[:-1]], np.uint64)
            self._ptrs[name] = torch.from_numpy(arr.view(np.int64)).to(device)

    def ptrs(self, name):
        return C.c_void_p(self._ptrs[name].data_ptr())

    def fluence_ptrs(self, fluence):
        torch = _torch()
        f = fluence if isinstance(fluence, torch.Tensor) else torch.as_tensor(np.asarray(fluence, np.float32))
        f = f.to(self.terma.device).float().contiguous()
        self._fluence = f
        if f.numel() == self.P:
            arr = np.full(len(self.beams), f.data_ptr(), np.uint64)
        else:
            arr = np.array([f.data_ptr() + 4 * self.P * i for i in range(len(self.beams))], np.uint64)
        self._fptr = torch.from_numpy(arr.view(np.int64)).to(self.terma.device)
        return C.c_void_p(self._fptr.data_ptr())

    def get(self, name, i):
        L = int(self.beams[i]["long_dim"])
        t = getattr(self, name)[int(self.offsets[i]):int(self.offsets[i + 1])]
        return t.view(L, *self.shape2)


def TermaComputeCollective(ctx, batch, fluence, density, spectrum, stream=None):
    """fastdose::TermaComputeCollective over the batch's beams."""
    fp = batch.fluence_ptrs(fluence)
    _lib.check(ctx.lib.fd2_terma_compute(ctx.h, batch.P, len(batch.beams), C.c_void_p(batch.d_beams.data_ptr()), fp,
                                         batch.ptrs("terma"), batch.ptrs("dens"), density.h, spectrum.h,
                                         _stream_ptr(stream)), "terma_compute")


def DoseComputeCollective(ctx, batch, kernel, stream=None):
    """fastdose::DoseComputeCollective: accumulates into batch.dose."""
    _lib.check(ctx.lib.fd2_dose_compute(ctx.h, batch.P, len(batch.beams), C.c_void_p(batch.d_beams.data_ptr()),
                                        batch.ptrs("terma"), batch.ptrs("dens"), batch.ptrs("dose"), kernel.h,
                                        _stream_ptr(stream)), "dose_compute")


def cone_directions(ctx, kernel, beams):
    """The CCCS cone directions the device uses, float32 [n][n_fwd][n_phi][4]."""
    b = np.ascontiguousarray(beams, BEAM_DTYPE).reshape(-1)
    k = kernel.src
    n_fwd = int(np.sum(k.theta.astype(np.float64) <= np.pi / 2))
    out = np.zeros((b.size, n_fwd, k.n_phi, 4), np.float32)
    _lib.check(ctx.lib.fd2_cccs_cone_directions(ctx.h, kernel.h, b.size, _p(b), _p(out), out.size),
               "cone_directions")
    return out


def BEV2PVCSInterp(ctx, batch, beamlets_per_beam, density, extent=2.0, ss_factor=5, value_type="f32", stream=None):
    """IMRT::BEV2PVCSInterp + MatCSREnsemble::addMat on the dose already in
    `batch` (a BEVBatch whose beams are the concatenation of beamlets_per_beam)."""
    counts = np.array(beamlets_per_beam, np.uint32)
    assert counts.sum() == len(batch.beams)
    prm = _Params(extent, ss_factor, VALUE_TYPES[value_type], -1, 0, 0, 0, None)
    h = C.c_void_p()
    _lib.check(ctx.lib.fd2_bev2pvcs_interp(ctx.h, len(counts), _p(counts), _p(batch.beams), batch.ptrs("dose"),
                                           density.h, C.byref(prm), C.byref(h),
                                           _stream_ptr(stream) if stream is not None else None), "bev2pvcs_interp")
    return MatCSREnsemble(ctx, h)


def BEV2PVCS(ctx, beam, density, bev, ssfactor=0, extent=2.0, out=None, stream=None):
    """fastdose::BEV2PVCS (ssfactor=0) or BEV2PVCS_SuperSampling (ssfactor>0)."""
    torch = _torch()
    b = np.array(beam, BEAM_DTYPE)
    nx, ny, nz = (int(v) for v in density.volume["dim"])
    if out is None:
        out = torch.zeros((nz, ny, nx), dtype=torch.float32, device="cuda")
    bev = bev.contiguous()
    if ssfactor <= 0:
        st = ctx.lib.fd2_bev2pvcs(ctx.h, _p(b), density.h, C.c_void_p(bev.data_ptr()), C.c_void_p(out.data_ptr()),
                                  nx * 4, _stream_ptr(stream))
    else:
        st = ctx.lib.fd2_bev2pvcs_supersampling(ctx.h, _p(b), density.h, C.c_void_p(bev.data_ptr()),
                                                C.c_void_p(out.data_ptr()), nx * 4, ssfactor, extent,
                                                _stream_ptr(stream))
    _lib.check(st, "bev2pvcs")
    return out


def beamletFlagInit(ctx, bundles, ptv_mask, volume, super_sampling=3):
    """IMRT::beamletFlagInit: uint8 [n_bundles][fy*fx]."""
    bb = np.ascontiguousarray(bundles, BUNDLE_DTYPE)
    m = np.ascontiguousarray(ptv_mask, np.uint8)
    v = np.array(volume, VOLUME_DTYPE)
    P = int(bb[0]["fluence_dim"][0]) * int(bb[0]["fluence_dim"][1])
    out = np.zeros(bb.size * P, np.uint8)
    _lib.check(ctx.lib.fd2_beamlet_flags(ctx.h, bb.size, _p(bb), _p(m), _p(v), super_sampling, _p(out)),
               "beamlet_flags")
    return out.reshape(bb.size, P)


# ------------------------------------------------------------------ dose matrix
class _Params(C.Structure):
    _fields_ = [("extent", C.c_float), ("ss_factor", C.c_int), ("value_type", C.c_int), ("cccs_schedule", C.c_int),
                ("batch_beamlets", C.c_uint64), ("memory_budget", C.c_uint64), ("verbose", C.c_int),
                ("host_out", C.c_void_p), ("graph", C.c_int), ("overlap", C.c_int)]


class _HostCSR(C.Structure):
    _fields_ = [("row_off", C.c_void_p), ("col", C.c_void_p), ("val", C.c_void_p), ("scale", C.c_void_p),
                ("cap_nnz", C.c_uint64), ("nnz", C.c_uint64)]


class HostCSR:
    """Pinned host buffers a dose matrix is copied into while it is built
    (fd2_host_csr_t): DoseMatConstruction(..., host_out=this) copies each
    finished batch of rows on a copy stream while the device computes the next
    batch.  Reusable across constructions of up to `n_rows` rows and `cap_nnz`
    nonzeros."""

    def __init__(self, n_rows, cap_nnz, value_type="f32"):
        torch = _torch()
        self.value_type = value_type
        vt = torch.float32 if value_type == "f32" else torch.int16
        self.row_off = torch.empty(int(n_rows) + 1, dtype=torch.int64, pin_memory=True)
        self.col = torch.empty(max(1, int(cap_nnz)), dtype=torch.int32, pin_memory=True)
        self.val = torch.empty(max(1, int(cap_nnz)), dtype=vt, pin_memory=True)
        self.scale = torch.empty(max(1, int(n_rows)), dtype=torch.float32, pin_memory=True)
        self.cap_nnz = int(cap_nnz)
        self.n_rows = 0
        self.nnz = 0

    def _struct(self):
        return _HostCSR(self.row_off.data_ptr(), self.col.data_ptr(), self.val.data_ptr(), self.scale.data_ptr(),
                        self.cap_nnz, 0)

    def arrays(self):
        """(row_off, col, val) of the last matrix copied in, as numpy views
        (val: float32, or the raw 16-bit words of an f16/bf16 matrix), plus the
        row scales for 16-bit values (None for f32)."""
        ro = self.row_off.numpy()[: self.n_rows + 1]
        col = self.col.numpy()[: self.nnz]
        val = self.val.numpy()[: self.nnz]
        sc = None if self.value_type == "f32" else self.scale.numpy()[: self.n_rows]
        return ro, col, val, sc

    def nbytes(self):
        vb = 4 if self.value_type == "f32" else 2
        n = (self.n_rows + 1) * 8 + self.nnz * (4 + vb)
        return n + (self.n_rows * 4 if self.value_type != "f32" else 0)


class _Info(C.Structure):
    _fields_ = [("n_mats", C.c_uint64), ("n_rows", C.c_uint64), ("n_cols", C.c_uint64), ("nnz", C.c_uint64),
                ("value_type", C.c_int)]


VALUE_TYPES = {"f32": 0, "f16": 1, "bf16": 2}


class MatCSREnsemble:
    """Device CSR of a dose-loading matrix (rows = beamlets, columns = voxels),
    one matrix per beam, as IMRT::MatCSREnsemble."""

    def __init__(self, ctx, handle):
        self.ctx = ctx
        self.h = handle

    def info(self):
        i = _Info()
        _lib.check(self.ctx.lib.fd2_csr_ensemble_info(self.h, C.byref(i)), "ensemble_info")
        return dict(n_mats=i.n_mats, n_rows=i.n_rows, n_cols=i.n_cols, nnz=i.nnz, value_type=i.value_type)

    def to_host(self):
        inf = self.info()
        ro = np.zeros(inf["n_rows"] + 1, np.int64)
        col = np.zeros(inf["nnz"], np.int32)
        val = np.zeros(inf["nnz"], np.float32)
        _lib.check(self.ctx.lib.fd2_csr_ensemble_to_host(self.h, _p(ro), _p(col), _p(val)), "ensemble_to_host")
        return ro, col, val

    def mat_rows(self):
        inf = self.info()
        ptr = C.POINTER(C.c_uint64)()
        _lib.check(self.ctx.lib.fd2_csr_ensemble_device(self.h, None, None, None, None, C.byref(ptr)),
                   "ensemble_device")
        return np.array([ptr[i] for i in range(inf["n_mats"] + 1)], np.uint64)

    def device_views(self):
        ro, col, val, sc = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_void_p()
        _lib.check(self.ctx.lib.fd2_csr_ensemble_device(self.h, C.byref(ro), C.byref(col), C.byref(val),
                                                        C.byref(sc), None), "ensemble_device")
        return ro.value, col.value, val.value, sc.value

    def tofile(self, folder):
        _lib.check(self.ctx.lib.fd2_csr_ensemble_tofile(self.h, str(folder).encode()), "ensemble_tofile")

    @classmethod
    def fromfile(cls, ctx, folder, n_cols, value_type="f32"):
        """f32 reads the reference's valuesBuffer.bin; f16/bf16 read the sidecars
        a 16-bit ensemble's tofile wrote."""
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_csr_ensemble_fromfile(ctx.h, str(folder).encode(), n_cols, VALUE_TYPES[value_type],
                                                     C.byref(h)), "ensemble_fromfile")
        return cls(ctx, h)

    @classmethod
    def concat(cls, ctx, parts):
        """The matrices of several ensembles as one, in order (fd2_csr_ensemble_concat)."""
        arr = (C.c_void_p * len(parts))(*[p.h for p in parts])
        h = C.c_void_p()
        _lib.check(ctx.lib.fd2_csr_ensemble_concat(ctx.h, len(parts), arr, C.byref(h)), "ensemble_concat")
        return cls(ctx, h)

    def close(self):
        if self.h:
            self.ctx.lib.fd2_csr_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def DoseMatConstruction(ctx, beamlets_per_beam, fluence, density, spectrum, kernel, extent=2.0, ss_factor=5,
                        value_type="f32", cccs_schedule=-1, memory_budget=0, batch_beamlets=0, verbose=False,
                        stream=None, host_out=None, graph=False, overlap=True):
    """IMRT::DoseMatConstruction: `beamlets_per_beam` is a list of BEAM_DTYPE
    arrays (one per beam).  Returns a MatCSREnsemble.  host_out: a HostCSR
    (of this value type) that receives a host copy of the matrix, batch by
    batch while it is built.  graph: each batch launched as one CUDA graph
    (kept per batch shape in the context and updated in place).  overlap: each
    batch's column stage runs on a second stream beside the next batch's
    Terma and CCCS (up to twice the BEV scratch); the matrix is the same."""
    counts = np.array([len(b) for b in beamlets_per_beam], np.uint32)
    allb = np.ascontiguousarray(np.concatenate([np.asarray(b, BEAM_DTYPE).reshape(-1) for b in beamlets_per_beam]),
                                BEAM_DTYPE) if len(beamlets_per_beam) else np.zeros(0, BEAM_DTYPE)
    fl = np.ascontiguousarray(fluence, np.float32)
    hs = None
    if host_out is not None:
        if host_out.value_type != value_type:
            raise ValueError(f"host_out holds {host_out.value_type} values, the matrix is {value_type}")
        if host_out.row_off.numel() < allb.size + 1:
            raise ValueError(f"host_out holds {host_out.row_off.numel() - 1} rows, the plan has {allb.size}")
        hs = host_out._struct()
    prm = _Params(extent, ss_factor, VALUE_TYPES[value_type], cccs_schedule, batch_beamlets, memory_budget,
                  int(verbose), C.cast(C.pointer(hs), C.c_void_p) if hs is not None else None, int(bool(graph)),
                  int(bool(overlap)))
    h = C.c_void_p()
    st = ctx.lib.fd2_dose_mat_construct(ctx.h, len(counts), _p(counts), _p(allb), _p(fl), density.h, spectrum.h,
                                        kernel.h, C.byref(prm), C.byref(h),
                                        _stream_ptr(stream) if stream is not None else None)
    _lib.check(st, "dose_mat_construct")
    if host_out is not None:
        host_out.n_rows = int(allb.size)
        host_out.nnz = int(hs.nnz)
    return MatCSREnsemble(ctx, h)
