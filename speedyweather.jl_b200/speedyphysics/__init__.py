"""speedyphysics: column physics of SpeedyWeather's wet primitive-equation model on B200.

* ``column_physics_(dtemp, dhumid, temp, humid, surface_pressure; dt, add)`` -- the plain
  large-scale condensation + simplified Betts-Miller convection
  (SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178,
  convection.jl:33-253), one CUDA thread per column.
* ``ColumnEmulator`` -- the MLP that stands in for both, with hand-written BF16 training and
  inference kernels on the tensor cores, used as a parameterization with the plain
  schemes as fallback for columns outside its training range (``parameterization_``).

Fields are layer-major like a Field{npoints, nlayers}: torch tensors [8, ncol] float32 on
the GPU, surface pressure [ncol]. Every compute call runs libsht's kernels.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from speedytransforms import _lib
from speedytransforms._lib import check, lib

NLAYERS = 8
NIN, NOUT = 4 * NLAYERS + 1, 2 * NLAYERS


def _stream(t):
    return torch.cuda.current_stream(t.device).cuda_stream


def _f32(t, name, shape=None):
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float32):
        raise TypeError(f"{name} must be a float32 CUDA tensor")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise _lib.DimensionMismatch(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


def column_physics_(dtemp, dhumid, temp, humid, surface_pressure, *, dt=1200.0, add=False):
    """Tendencies of the plain condensation + convection for every column (in place)."""
    ncol = temp.shape[1]
    for n, t in (("temp", temp), ("humid", humid), ("dtemp", dtemp), ("dhumid", dhumid)):
        _f32(t, n, (NLAYERS, ncol))
    _f32(surface_pressure, "surface_pressure", (ncol,))
    check(lib.sht_column_physics(temp.data_ptr(), humid.data_ptr(), surface_pressure.data_ptr(), ncol, ncol, NLAYERS,
                                 float(dt), dtemp.data_ptr(), dhumid.data_ptr(), _lib.ADD if add else 0,
                                 _stream(temp)))
    return dtemp, dhumid


def columns_as_rows(temp, humid, u, v, surface_pressure):
    """[ncol, 33] network inputs: temp, humid, u, v on the 8 layers, then log ps (torch)."""
    return torch.cat([temp.T, humid.T, u.T, v.T, torch.log(surface_pressure)[:, None]], dim=1).contiguous()


class ColumnEmulator:
    """MLP 33 -> 256 -> 256 -> 256 -> 16 (GELU) on the tensor cores (sht_mlp_*)."""

    def __init__(self, capacity: int, seed: int = 0, device=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        h = C.c_void_p()
        self._m = None
        check(lib.sht_mlp_create(int(capacity), int(seed), self.device.index or 0, C.byref(h)))
        self._m = h
        self.capacity = int(capacity)
        self.x_mean = self.x_std = self.y_mean = self.y_std = None

    def set_normalization(self, x_mean, x_std, y_mean, y_std):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (x_mean, x_std, y_mean, y_std)]
        ptr = [a.ctypes.data_as(C.c_void_p) for a in arrs]
        check(lib.sht_mlp_set_normalization(self._m, *ptr))
        self.x_mean, self.x_std, self.y_mean, self.y_std = arrs

    def fit_normalization(self, x, y):
        """Mean and standard deviation of training inputs [N, 33] and targets [N, 16]."""
        xm, xs = x.mean(0).double().cpu().numpy(), x.std(0).double().cpu().numpy()
        ym, ys = y.mean(0).double().cpu().numpy(), y.std(0).double().cpu().numpy()
        self.set_normalization(xm, np.maximum(xs, 1e-12), ym, np.maximum(ys, 1e-30))

    def train_step(self, x, y, lr=1e-3):
        _f32(x, "x", (x.shape[0], NIN))
        _f32(y, "y", (x.shape[0], NOUT))
        check(lib.sht_mlp_train_step(self._m, x.data_ptr(), y.data_ptr(), x.shape[0], float(lr), _stream(x)))

    def loss(self) -> float:
        v = C.c_float(0)
        check(lib.sht_mlp_loss(self._m, C.byref(v)))
        return float(v.value)

    def train(self, x, y, *, epochs=4, batch=4096, lr=1e-3, seed=0):
        """Minibatch Adam over (x, y) [N, 33], [N, 16] on the GPU; returns the mean loss per epoch."""
        g = torch.Generator(device=x.device).manual_seed(seed)
        losses = []
        n = x.shape[0]
        for ep in range(epochs):
            perm = torch.randperm(n, device=x.device, generator=g)
            tot, cnt = 0.0, 0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                self.train_step(x[idx].contiguous(), y[idx].contiguous(), lr * (0.5 ** ep))
                if (i // batch) % 16 == 0:
                    tot += self.loss()
                    cnt += 1
            losses.append(tot / max(cnt, 1))
        return losses

    def infer(self, x):
        _f32(x, "x", (x.shape[0], NIN))
        y = torch.empty((x.shape[0], NOUT), device=x.device, dtype=torch.float32)
        check(lib.sht_mlp_infer(self._m, x.data_ptr(), y.data_ptr(), x.shape[0], _stream(x)))
        return y

    def params(self, layer):
        fo = [256, 256, 256, NOUT][layer]
        fi = [64, 256, 256, 256][layer]
        w = np.zeros((fo, fi), np.float32)
        b = np.zeros(fo, np.float32)
        check(lib.sht_mlp_params(self._m, layer, w.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), 0))
        return w, b

    def parameterization_(self, dtemp, dhumid, temp, humid, u, v, surface_pressure, *, dt=1200.0, z_max=4.0,
                          add=False) -> int:
        """The emulator as the column parameterization (fallback to the plain schemes outside
        z_max standard deviations of the training inputs); returns the fallback count."""
        ncol = temp.shape[1]
        for n, t in (("temp", temp), ("humid", humid), ("u", u), ("v", v), ("dtemp", dtemp), ("dhumid", dhumid)):
            _f32(t, n, (NLAYERS, ncol))
        _f32(surface_pressure, "surface_pressure", (ncol,))
        nf = C.c_int32(0)
        check(lib.sht_column_emulate(self._m, temp.data_ptr(), humid.data_ptr(), u.data_ptr(), v.data_ptr(),
                                     surface_pressure.data_ptr(), ncol, ncol, float(dt), float(z_max),
                                     dtemp.data_ptr(), dhumid.data_ptr(), _lib.ADD if add else 0, C.byref(nf),
                                     _stream(temp)))
        return int(nf.value)

    def device_status(self) -> int:
        v = C.c_int32(0)
        check(lib.sht_mlp_device_status(self._m, C.byref(v)))
        return int(v.value)

    def __del__(self):
        if getattr(self, "_m", None) is not None:
            lib.sht_mlp_destroy(self._m)
            self._m = None


def bf16_gemm(A, a_mn, B, b_mn, M, N, K):
    """C [M, N] float32 = A B on the tensor cores (the network's matrix product); A, B
    bfloat16 CUDA tensors stored as described for sht_bf16_gemm."""
    err = torch.zeros(1, dtype=torch.int32, device=A.device)
    Cm = torch.empty((M, N), dtype=torch.float32, device=A.device)
    check(lib.sht_bf16_gemm(A.data_ptr(), A.shape[1], int(a_mn), B.data_ptr(), B.shape[1], int(b_mn), Cm.data_ptr(),
                            N, M, N, K, err.data_ptr(), _stream(A)))
    return Cm, err
