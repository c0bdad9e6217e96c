"""ctypes wrapper of the oracle's C restatement (oracle/sht_cpu.c).

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU baseline and
--impl reference arm; never by the product.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "_build", "libsht_cpu.so")


def _load():
    if not os.path.exists(_LIB):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    lib = C.CDLL(_LIB)
    lib.cpu_plan_create.restype = C.c_void_p
    lib.cpu_plan_create.argtypes = [C.c_int] * 5
    lib.cpu_plan_destroy.argtypes = [C.c_void_p]
    lib.cpu_npoints.restype = C.c_int64
    lib.cpu_npoints.argtypes = [C.c_void_p]
    lib.cpu_nlm.restype = C.c_int64
    lib.cpu_nlm.argtypes = [C.c_void_p]
    lib.cpu_synthesize.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
    lib.cpu_analyze.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    lib.cpu_max_threads.restype = C.c_int
    return lib


lib = _load()


class CpuTransform:
    """FP32 CPU transform with the reference's loop structure; grid 0 = full, 1 = octahedral."""

    def __init__(self, grid, nlat_half, lmax, mmax, nlayers):
        self.h = lib.cpu_plan_create(grid, nlat_half, lmax, mmax, nlayers)
        self.npoints = lib.cpu_npoints(self.h)
        self.nlm = lib.cpu_nlm(self.h)

    def __del__(self):
        if getattr(self, "h", None):
            lib.cpu_plan_destroy(self.h)
            self.h = None

    def synthesize(self, coeffs_kl, out=None, unscale=False):
        """coeffs (K, nlm) complex64 -> grid (K, npoints) float32."""
        c = np.ascontiguousarray(coeffs_kl, dtype=np.complex64)
        K = c.shape[0]
        out = np.empty((K, self.npoints), np.float32) if out is None else out
        lib.cpu_synthesize(self.h, c.ctypes.data, out.ctypes.data, K, int(unscale))
        return out

    def analyze(self, grid_kp, out=None):
        g = np.ascontiguousarray(grid_kp, dtype=np.float32)
        K = g.shape[0]
        out = np.empty((K, self.nlm), np.complex64) if out is None else out
        lib.cpu_analyze(self.h, g.ctypes.data, out.ctypes.data, K)
        return out


def max_threads():
    return lib.cpu_max_threads()
