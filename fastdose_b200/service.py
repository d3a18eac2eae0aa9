"""Python mirror of the served dose calculation (include/fd2_service.h).

A Service takes plan requests from any thread, admits them in arrival order
under an HBM budget, and builds each plan's dose-loading matrix on one of its
worker contexts; `wait` returns the matrix and the request's timing on the
service clock (submit, start, end) for latency reports.
"""
import ctypes as C

import numpy as np

from . import _lib
from .api import VALUE_TYPES, MatCSREnsemble, _p, _Params
from .types import BEAM_DTYPE, VOLUME_DTYPE


class _Volume(C.Structure):
    _fields_ = [("dim", C.c_uint32 * 3), ("voxel_size", C.c_float * 3), ("bbox_start", C.c_uint32 * 3),
                ("bbox_dim", C.c_uint32 * 3)]


class _ServiceParams(C.Structure):
    _fields_ = [("device", C.c_int), ("workers", C.c_int), ("reserved", C.c_int32), ("hbm_budget", C.c_uint64),
                ("bev_budget", C.c_uint64)]


_vp = C.c_void_p


class _Request(C.Structure):
    _fields_ = [("density", _vp), ("volume", _Volume), ("n_beams", C.c_size_t), ("n_beamlets_per_beam", _vp),
                ("beamlets", _vp), ("fluence", _vp), ("n_spectrum", C.c_int), ("energy", _vp),
                ("spectrum_fluence", _vp), ("mu", _vp), ("mu_en", _vp), ("n_theta", C.c_int), ("theta", _vp),
                ("A", _vp), ("a", _vp), ("B", _vp), ("b", _vp), ("n_phi", C.c_int), ("phi", _vp),
                ("params", _Params)]


class _Stats(C.Structure):
    _fields_ = [("submit_ms", C.c_double), ("start_ms", C.c_double), ("end_ms", C.c_double),
                ("beamlets", C.c_uint64), ("nnz", C.c_uint64), ("est_bytes", C.c_uint64), ("status", C.c_int32),
                ("worker", C.c_int32)]


class _LibOnly:
    """Stand-in context for results: MatCSREnsemble needs only the library."""

    def __init__(self):
        self.lib = _lib.get()


class Service:
    def __init__(self, device=0, workers=2, hbm_budget=0, bev_budget=0):
        lib = _lib.get()
        prm = _ServiceParams(device, workers, 0, int(hbm_budget), int(bev_budget))
        h = C.c_void_p()
        _lib.check(lib.fd2_service_create(C.byref(prm), C.byref(h)), "service_create")
        self.h = h
        self.lib = lib

    def clock_ms(self):
        return self.lib.fd2_service_clock_ms(self.h)

    def submit(self, phantom, beamlets_per_beam, fluence, spectrum, kernel, extent=2.0, ss_factor=5,
               value_type="f32", graph=False):
        """Queues one plan; returns its ticket.  The inputs are copied.  graph:
        the worker launches each construction batch as one CUDA graph (kept
        per batch shape on the worker's context and updated in place)."""
        keep = []

        def arr(x, dt):
            a = np.ascontiguousarray(x, dt)
            keep.append(a)
            return a

        dens = arr(phantom.density, np.float32)
        vol = np.asarray(phantom.volume, VOLUME_DTYPE).reshape(())
        counts = arr([len(b) for b in beamlets_per_beam], np.uint32)
        allb = arr(np.concatenate([np.asarray(b, BEAM_DTYPE).reshape(-1) for b in beamlets_per_beam]), BEAM_DTYPE)
        fl = arr(fluence, np.float32)
        sp = [arr(x, np.float32) for x in (spectrum.energy, spectrum.fluence, spectrum.mu, spectrum.mu_en)]
        kn = [arr(x, np.float32) for x in (kernel.theta, kernel.A, kernel.a, kernel.B, kernel.b)]
        phi = arr(kernel.phi, np.float32)
        v = _Volume((C.c_uint32 * 3)(*vol["dim"]), (C.c_float * 3)(*vol["voxel_size"]),
                    (C.c_uint32 * 3)(*vol["bbox_start"]), (C.c_uint32 * 3)(*vol["bbox_dim"]))
        req = _Request(_p(dens), v, len(counts), _p(counts), _p(allb), _p(fl), spectrum.n, *(_p(x) for x in sp),
                       kernel.n_theta, *(_p(x) for x in kn), kernel.n_phi, _p(phi),
                       _Params(extent, ss_factor, VALUE_TYPES[value_type], -1, 0, 0, 0, None, int(bool(graph))))
        t = C.c_uint64()
        _lib.check(self.lib.fd2_service_submit(self.h, C.byref(req), C.byref(t)), "service_submit")
        return t.value

    def wait(self, ticket):
        """(MatCSREnsemble or None, stats dict) of a submitted plan."""
        h = C.c_void_p()
        st = _Stats()
        rc = self.lib.fd2_service_wait(self.h, C.c_uint64(ticket), C.byref(h), C.byref(st))
        stats = {k: getattr(st, k) for k, _ in _Stats._fields_}
        if rc:
            raise _lib.FD2Error(rc, "service_wait")
        return (MatCSREnsemble(_LibOnly(), h) if h.value else None), stats

    def close(self):
        if self.h:
            self.lib.fd2_service_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
