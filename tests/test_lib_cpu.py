"""CPU: the C-ABI library builds, loads and exports every symbol the header declares.
No compute entry point is called here (there is no GPU)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "pyfantom_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|size_t|const char\*|unsigned long long)\s+(pf_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ["pf_matvec_f64", "pf_mg_solve", "pf_filter_fwd_f64", "pf_oc_update_f64", "pf_sensitivity_f64"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    from pyfantom_b200 import _lib
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s), s
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_status_strings_and_version():
    from pyfantom_b200 import _lib
    lib = _lib.load()
    assert lib.pf_version() >= 100
    for code, name in _lib.STATUS_NAMES.items():
        assert lib.pf_status_string(code).decode() == name


def test_bad_arguments_fail_before_touching_the_device():
    from pyfantom_b200 import _lib
    lib = _lib.load()
    g = _lib.make_grid((4, 4, 0))
    g.dim = 5
    h = ctypes.c_void_p()
    K0 = (ctypes.c_double * 576)()
    assert lib.pf_op_create(ctypes.byref(g), K0, ctypes.byref(h)) == _lib.PF_BAD_ARG
    assert b"dim" in lib.pf_last_error()
    assert lib.pf_matvec_f64(None, None, None, None, None, None) == _lib.PF_BAD_ARG
    assert lib.pf_mg_solve(None, None, None, 0, 1e-8, 10, None, None) == _lib.PF_BAD_ARG
    assert lib.pf_oc_update_f64(0, None, None, None, 0.5, 0.2, None, None, None, None) == _lib.PF_BAD_ARG


def test_package_imports_without_gpu():
    import pyfantom_b200.CUDA as C
    for name in C.__all__:
        assert hasattr(C, name)


def test_product_has_no_oracle_dependency():
    pkg = os.path.join(ROOT, "pyfantom_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh")):
                src = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in src.replace("oracle/", ""), f
