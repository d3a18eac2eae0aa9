"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares (no compute calls)."""
import ctypes as C
import os
import re

from fastdose_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:int|void|double|int64_t|uint64_t|const char\s*\*)\s+(fd2_\w+)\s*\(", re.M)


def _declared():
    names = set()
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            with open(os.path.join(ROOT, "include", fn)) as f:
                names |= set(DECL.findall(f.read()))
    return names


def test_headers_declare_the_interface():
    names = _declared()
    for required in ("fd2_dose_compute", "fd2_terma_compute", "fd2_dose_mat_construct", "fd2_matrix_spmv",
                     "fd2_boo_l2onehalf", "fd2_polish", "fd2_eval_grad", "fd2_dose_compute_static"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(lib, n)]
    assert not missing, missing


def test_ctypes_prototypes_cover_the_headers():
    assert _declared() <= set(_lib._PROTOS), sorted(_declared() - set(_lib._PROTOS))


def test_status_strings_without_gpu():
    lib = _lib.get()
    assert lib.fd2_status_string(0)
    assert lib.fd2_version() > 0
