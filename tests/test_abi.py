"""The C-ABI library loads without a GPU and exports every symbol include/sht.h declares."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "sht.h")
LIB = os.path.join(ROOT, "speedyweather.jl_b200", "libsht.so")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^SHT_API\s+[\w\s\*]+?\b(sht_\w+)\s*\(", text, flags=re.M)))


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "speedyweather.jl_b200", "csrc")])
    return ctypes.CDLL(LIB)


def test_header_declares_entry_points():
    syms = declared_symbols()
    for s in ("sht_plan_create", "sht_synthesize", "sht_analyze", "sht_curl", "sht_divergence",
              "sht_uv_from_vordiv", "sht_laplace", "sht_gradient", "sht_plan_destroy"):
        assert s in syms


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, f"libsht.so lacks {missing}"


def test_python_binding_covers_header():
    import speedytransforms._lib as L
    assert sorted(L.SIGNATURES) == declared_symbols()


def test_errors_without_gpu_are_statuses(lib):
    # host-side argument checks answer before any CUDA call
    import speedytransforms._lib as L
    h = ctypes.c_void_p()
    d = L.ShtDesc(7, 24, 32, 32, 8, 0, 0, 0)      # unknown grid kind
    assert L.lib.sht_plan_create(ctypes.byref(d), ctypes.byref(h)) == L.SHT_EUNSUPPORTED
    d = L.ShtDesc(0, 24, 16, 32, 8, 0, 0, 0)      # lmax < mmax
    assert L.lib.sht_plan_create(ctypes.byref(d), ctypes.byref(h)) == L.SHT_EINVAL
    assert b"lmax" in L.lib.sht_last_error()
    assert L.lib.sht_synthesize(None, None, 0, None, 0, 1, 0, None) == L.SHT_EINVAL
    assert L.lib.sht_version().startswith(b"libsht")
