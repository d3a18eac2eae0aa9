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


def test_cpp_shim_compiles_links_and_runs(tmp_path):
    """A C++ caller using the reference's names (fd2_compat.hpp) builds against
    the library and runs its device-free calls."""
    import shutil
    import subprocess

    if not shutil.which("g++"):
        import pytest

        pytest.skip("no g++")
    src = tmp_path / "caller.cpp"
    src.write_text(
        '#include "fd2_compat.hpp"\n#include <cstdio>\n'
        "int main() {\n"
        "  auto f = &fastdose::DoseComputeCollective; auto g = &IMRT::DoseMatConstruction; (void)f; (void)g;\n"
        '  std::printf("%d %s\\n", fd2_version(), fd2_status_string(FD2_ERR_ADMISSION));\n'
        "  return 0;\n}\n")
    exe = tmp_path / "caller"
    libdir = os.path.dirname(_lib.LIB_PATH)
    subprocess.run(["g++", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", "/usr/local/cuda/include",
                    str(src), "-L", libdir, "-lfd2", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split(maxsplit=1)
    assert int(out[0]) == _lib.get().fd2_version() and out[1].strip()


def test_status_strings_without_gpu():
    lib = _lib.get()
    assert lib.fd2_status_string(0)
    assert lib.fd2_version() > 0
