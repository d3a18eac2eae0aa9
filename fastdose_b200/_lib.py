"""Loads libfd2.so (built in-tree by fastdose_b200.build) and declares its C ABI.

There is no fallback: if the library is missing or fails to load, every entry
point raises.  Call `fastdose_b200.build.build()` (or `__graft_entry__.build()`)
first.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfd2.so")

_vp = C.c_void_p
_i = C.c_int
_sz = C.c_size_t
_f = C.c_float
_u64 = C.c_uint64
_i64 = C.c_int64

_PROTOS = {
    "fd2_status_string": (C.c_char_p, [_i]),
    "fd2_version": (_i, []),
    "fd2_last_error": (C.c_char_p, []),
    "fd2_beam_calc_range": (_i, [_vp, _vp]),
    "fd2_beamlet_init": (_i, [_vp, _i, _i, _vp, _vp]),
    "fd2_beamlet_fluence": (_i, [_vp, _vp, _sz]),
    "fd2_context_create": (_i, [_i, _vp]),
    "fd2_context_destroy": (_i, [_vp]),
    "fd2_context_synchronize": (_i, [_vp]),
    "fd2_context_release": (_i, [_vp]),
    "fd2_density_create": (_i, [_vp, _vp, _vp, _vp]),
    "fd2_density_destroy": (_i, [_vp]),
    "fd2_density_device_ptr": (_vp, [_vp]),
    "fd2_spectrum_create": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp]),
    "fd2_spectrum_destroy": (_i, [_vp]),
    "fd2_kernel_create": (_i, [_vp, _i, _vp, _vp, _vp, _vp, _vp, _i, _vp, _vp]),
    "fd2_kernel_destroy": (_i, [_vp]),
    "fd2_terma_compute": (_i, [_vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_dose_compute": (_i, [_vp, _sz, _sz, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_bev2pvcs": (_i, [_vp, _vp, _vp, _vp, _vp, _sz, _vp]),
    "fd2_bev2pvcs_supersampling": (_i, [_vp, _vp, _vp, _vp, _vp, _sz, _i, _f, _vp]),
    "fd2_beamlet_flags": (_i, [_vp, _sz, _vp, _vp, _vp, _i, _vp]),
    "fd2_dosemat_params_default": (None, [_vp]),
    "fd2_dose_mat_construct": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_csr_ensemble_info": (_i, [_vp, _vp]),
    "fd2_csr_ensemble_device": (_i, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_csr_ensemble_to_host": (_i, [_vp, _vp, _vp, _vp]),
    "fd2_csr_ensemble_tofile": (_i, [_vp, C.c_char_p]),
    "fd2_csr_ensemble_fromfile": (_i, [_vp, C.c_char_p, _u64, _i, _vp]),
    "fd2_csr_ensemble_destroy": (_i, [_vp]),
    "fd2_beamlet_flags_save": (_i, [_vp, _sz, C.c_char_p]),
    "fd2_cccs_cone_directions": (_i, [_vp, _vp, _sz, _vp, _vp, _sz]),
    "fd2_context_set_timing": (_i, [_vp, _i]),
    "fd2_context_stage_times": (_i, [_vp, _vp, _i]),
    "fd2_context_launch_count": (C.c_uint64, [_vp]),
    "fd2_bev2pvcs_interp": (_i, [_vp, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_dose_compute_static": (_i, [_sz, _sz, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    # optimizer (fd2_opt.h)
    "fd2_matrix_create": (_i, [_vp, _i64, _i64, _i64, _vp, _vp, _vp, _i, _i, _vp]),
    "fd2_matrix_destroy": (_i, [_vp]),
    "fd2_matrix_info": (_i, [_vp, _vp]),
    "fd2_matrix_to_host": (_i, [_vp, _vp, _vp, _vp]),
    "fd2_matrix_transpose": (_i, [_vp, _vp]),
    "fd2_matrix_spmv": (_i, [_vp, _vp, _vp, _vp]),
    "fd2_voi_matrices": (_i, [_vp, _vp, _i64, _i64, _i, _i, _vp, _vp]),
    "fd2_matrix_synthetic": (_i, [_vp, _i64, _i64, _i64, _f, _u64, _i, _i, _vp, _vp]),
    "fd2_fluence_grad": (_i, [_i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_opt_problem_create": (_i, [_vp, _vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _f, _f, _vp]),
    "fd2_opt_problem_destroy": (_i, [_vp]),
    "fd2_eval_g": (_i, [_vp, _vp, _vp]),
    "fd2_eval_grad": (_i, [_vp, _vp, _vp, _vp]),
    "fd2_prox_l2onehalf": (_i, [_vp, _i64, _vp, _vp, _vp, _vp, _vp, _vp]),
    "fd2_beam_weights_init": (_i, [_vp, _i64, _vp, _vp]),
    "fd2_boo_l2onehalf": (_i, [_vp, _i64, _vp, _vp, _i, _i, _i, _vp, _i, _i, _vp]),
    "fd2_polish": (_i, [_vp, _i, _i, _vp]),
    "fd2_matrix_select_blocks": (_i, [_vp, _i64, _vp, _vp, _i64, _vp, _vp]),
    "fd2_dvh": (_i, [_vp, _vp, _i64, _i64, _vp, _vp, _i, _f, _vp, _vp]),
    "fd2_csr_ensemble_concat": (_i, [_vp, _sz, _vp, _vp]),
    "fd2_context_tuned_schedules": (_i, [_vp, _sz, _vp, _vp, _vp, _vp]),
    "fd2_context_graph_counts": (_i, [_vp, _vp, _vp, _vp]),
    "fd2_opt_problem_set_graph": (_i, [_vp, _i]),
    "fd2_opt_problem_set_reducer": (_i, [_vp, _vp, _vp]),
    "fd2_bundles_beamlets": (_i, [_sz, _vp, _vp, _vp, _i, _sz, _vp, _vp]),
    "fd2_beam_orientation_optimization": (_i, [_vp, _vp, _vp, _i64, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp,
                                                _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    # served dose calculation (fd2_service.h)
    "fd2_service_create": (_i, [_vp, _vp]),
    "fd2_service_destroy": (_i, [_vp]),
    "fd2_service_submit": (_i, [_vp, _vp, _vp]),
    "fd2_service_wait": (_i, [_vp, _u64, _vp, _vp]),
    "fd2_service_clock_ms": (C.c_double, [_vp]),
}

_LIB = None


class FD2Error(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        lib = get()
        msg = lib.fd2_last_error().decode(errors="replace")
        super().__init__(f"{where}: {lib.fd2_status_string(status).decode()} ({status}): {msg}")


def get():
    """The loaded library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m fastdose_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def declare(name, restype, argtypes):
    """Declares an additional entry point (used by modules that add ABI)."""
    _PROTOS[name] = (restype, argtypes)
    if _LIB is not None:
        fn = getattr(_LIB, name)
        fn.restype = restype
        fn.argtypes = argtypes


def check(status, where):
    if status != 0:
        raise FD2Error(status, where)
    return status
