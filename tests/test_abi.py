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


def test_argument_checks_of_the_newer_entry_points(lib):
    """Host-side checks of the host-buffer transforms, batches, dense-matrix transforms,
    column physics and the MLP answer with statuses before any CUDA call."""
    import speedytransforms._lib as L
    E = L.SHT_EINVAL
    f = L.lib
    assert f.sht_synthesize_host(None, None, 0, None, 0, 1, 0, None) == E
    assert f.sht_analyze_host(None, None, 0, None, 0, 1, 0, None) == E
    assert f.sht_plan_set_host_chunk(None, 8) == E
    assert f.sht_host_wait(None, None) == E
    assert f.sht_diag_wait_expiry(None, 1000, None) == E
    assert f.sht_column_physics(None, None, None, 10, 10, 7, 1200.0, None, None, 0, None) == E   # nlayers
    assert b"nlayers" in f.sht_last_error()
    assert f.sht_column_physics(None, None, None, 5, 10, 8, 1200.0, None, None, 0, None) == E    # ld < ncol
    assert f.sht_column_physics(None, None, None, 10, 10, 8, 1200.0, None, None, 0, None) == E   # NULL
    h = ctypes.c_void_p()
    assert f.sht_mlp_create(0, 0, 0, ctypes.byref(h)) == E
    assert f.sht_mlp_train_step(None, None, None, 16, 1e-3, None) == E
    assert f.sht_mlp_backward(None, None, None, 16, None) == E
    assert f.sht_mlp_infer(None, None, None, 16, None) == E
    assert f.sht_mlp_params(None, 0, None, None, 0) == E
    assert f.sht_column_emulate(None, None, None, None, None, None, 10, 10, 1200.0, 4.0, None, None, 0, None,
                                None) == E
    err = (ctypes.c_int32 * 1)()
    assert f.sht_bf16_gemm(None, 8, 0, None, 8, 0, None, 8, 1, 1, 1, err, None) == E
    assert f.sht_bf16_gemm(1, 7, 0, 1, 8, 0, 1, 8, 1, 1, 1, err, None) == E           # lda % 8
    assert f.sht_batch_create(None, 0, ctypes.byref(h)) == E
    assert f.sht_matrix_create(None, ctypes.byref(h)) == E
