"""The C ABI library loads and exports every function include/*.h declares
(no GPU needed: only symbols are resolved)."""
import ctypes
import glob
import os
import re

from conftest import ROOT


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(sa_[a-z0-9_]+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    names = declared()
    assert {"sa_ctx_create", "sa_plan_forward_adjoint", "sa_eik_fwd_field",
            "sa_surfdisp_columns", "sa_combine_kernels_vs"} <= names


def test_library_exports_declared_symbols():
    from surfattpp_b200 import _capi, build
    if not os.path.exists(_capi.LIB_PATH):
        build.build()
    lib = ctypes.CDLL(_capi.LIB_PATH)
    missing = [n for n in sorted(declared()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_capi.EXPORTED) == declared()


def test_cpp_adapters_compile_and_link():
    """tests/cpp/adapters_test.cpp: C++20 adapters in the reference's layouts
    compile against include/surfatt_gpu.h and link to the library (run on a
    GPU by test_gpu_cpp_adapters.py)."""
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    subprocess.run(["make", "-s", "-B", "-C", os.path.join(here, "cpp")], check=True)
    assert os.access(os.path.join(here, "_build", "adapters_test"), os.X_OK)
