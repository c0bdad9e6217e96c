"""speedyphysics: column physics of SpeedyWeather's wet primitive-equation model on B200.

* ``column_physics_(dtemp, dhumid, temp, humid, surface_pressure; dt, add)`` -- the plain
  large-scale condensation + simplified Betts-Miller convection
  (SpeedyWeather/src/parameterizations/large_scale_condensation.jl:55-178,
  convection.jl:33-253), one CUDA thread per column.
* ``ColumnEmulator`` -- the MLP that stands in for both, with hand-written BF16 training and
  inference kernels on the tensor cores, used as a parameterization with the plain
  schemes as fallback for columns outside its training range (``parameterization_``).
* ``ModelStates`` -- columns of the wet model's own states at T63 (the reference's initial
  state with seeded variations, through this library's transforms) to train it on.

Fields are layer-major like a Field{npoints, nlayers}: torch tensors [8, ncol] float32 on
the GPU, surface pressure [ncol]. Every compute call runs libsht's kernels.
"""
from __future__ import annotations

import ctypes as C
import math

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


def synthetic_columns(ncol: int, seed: int = 0, device=None):
    """Seeded columns standing in for model-generated states (there is no dynamical core
    here), generated on the GPU: latitude-dependent surface temperature with a
    tropospheric lapse rate, relative humidity 0.2 .. 1.05 decreasing upward, a zonal jet
    with noise, log surface pressure near 1e5 Pa. Returns temp, humid, u, v [8, ncol] and
    surface_pressure [ncol], float32 (the same distribution as the tests' numpy columns).
    Saturation humidity by Clausius-Clapeyron (SpeedyWeather/src/dynamics/atmosphere.jl:138-157)."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev).manual_seed(seed)
    f64 = torch.float64
    half = torch.linspace(0, 1, NLAYERS + 1, dtype=f64, device=dev)
    full = (0.5 * (half[1:] + half[:-1]))[:, None]
    U = lambda *shape: torch.rand(*shape, generator=g, device=dev, dtype=f64)      # noqa: E731
    N = lambda *shape: torch.randn(*shape, generator=g, device=dev, dtype=f64)     # noqa: E731
    r_dry, r_vap = 1000 * 8.3145 / 28.9649, 1000 * 8.3145 / 18.0153
    lat = torch.asin(2 * U(ncol) - 1)
    ps = 1e5 * torch.exp(0.02 * N(ncol))
    Ts = 302 - 45 * torch.sin(lat) ** 2 + 3 * N(ncol)
    T = Ts[None, :] * full ** (r_dry * 0.0065 / 9.81) + 1.5 * N(NLAYERS, ncol)
    T = torch.maximum(T, 195.0 + 2 * N(NLAYERS, ncol))
    rh = (0.5 + 0.55 * U(ncol))[None, :] * (0.25 + 0.75 * full ** 1.5) * (0.85 + 0.3 * U(NLAYERS, ncol))
    qsat = (r_dry / r_vap) * 610.78 * torch.exp(2501.0e3 / r_vap * (1 / 273.15 - 1 / T)) / (ps[None, :] * full)
    q = torch.clamp(rh, 0.02, 1.08) * qsat
    u = 30 * torch.sin(2 * lat)[None, :] * (1.2 - full) + 5 * N(NLAYERS, ncol)
    v = 4 * N(NLAYERS, ncol)
    return tuple(a.float().contiguous() for a in (T, q, u, v, ps))


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

    def backward(self, x, y):
        """Loss and gradients over (x, y) without an update; returns the loss."""
        _f32(x, "x", (x.shape[0], NIN))
        _f32(y, "y", (x.shape[0], NOUT))
        check(lib.sht_mlp_backward(self._m, x.data_ptr(), y.data_ptr(), x.shape[0], _stream(x)))
        return self.loss()

    def gradients(self, layer):
        """(dW [out][in], db [out]) of the last backward pass, FP32 numpy."""
        w, b = self._layer_arrays(layer)
        check(lib.sht_mlp_params(self._m, layer, w.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), 2))
        return w, b

    def _layer_arrays(self, layer):
        fo = [256, 256, 256, NOUT][layer]
        fi = [64, 256, 256, 256][layer]
        return np.zeros((fo, fi), np.float32), np.zeros(fo, np.float32)

    def set_params(self, layer, w, b):
        """Upload FP32 parameters of one layer (w [out][in], b [out])."""
        w0, b0 = self._layer_arrays(layer)
        w = np.ascontiguousarray(w, dtype=np.float32).reshape(w0.shape)
        b = np.ascontiguousarray(b, dtype=np.float32).reshape(b0.shape)
        check(lib.sht_mlp_params(self._m, layer, w.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), 1))

    def loss(self) -> float:
        v = C.c_float(0)
        check(lib.sht_mlp_loss(self._m, C.byref(v)))
        return float(v.value)

    def train(self, x, y, *, epochs=4, batch=4096, lr=1e-3, seed=0, schedule="halve"):
        """Minibatch Adam over (x, y) [N, 33], [N, 16] on the GPU; returns the mean loss per
        epoch. schedule: "halve" (lr / 2 per epoch) or "cosine" (cosine decay over all steps
        to lr / 100)."""
        g = torch.Generator(device=x.device).manual_seed(seed)
        losses = []
        n = x.shape[0]
        steps = max(1, epochs * (n // batch))
        k = 0
        for ep in range(epochs):
            perm = torch.randperm(n, device=x.device, generator=g)
            tot, cnt = 0.0, 0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                if schedule == "cosine":
                    rate = lr * (0.01 + 0.99 * 0.5 * (1 + math.cos(math.pi * k / steps)))
                else:
                    rate = lr * (0.5 ** ep)
                self.train_step(x[idx].contiguous(), y[idx].contiguous(), rate)
                k += 1
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
        """(w [out][in], b [out]) FP32 master parameters of one layer, numpy."""
        w, b = self._layer_arrays(layer)
        check(lib.sht_mlp_params(self._m, layer, w.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), 0))
        return w, b

    def parameterization_(self, dtemp, dhumid, temp, humid, u, v, surface_pressure, *, dt=1200.0, z_max=4.0,
                          add=False, count=True):
        """The emulator as the column parameterization (fallback to the plain schemes outside
        z_max standard deviations of the training inputs); returns the fallback count
        (count=True synchronises the stream), or None."""
        ncol = temp.shape[1]
        for n, t in (("temp", temp), ("humid", humid), ("u", u), ("v", v), ("dtemp", dtemp), ("dhumid", dhumid)):
            _f32(t, n, (NLAYERS, ncol))
        _f32(surface_pressure, "surface_pressure", (ncol,))
        nf = C.c_int32(0)
        check(lib.sht_column_emulate(self._m, temp.data_ptr(), humid.data_ptr(), u.data_ptr(), v.data_ptr(),
                                     surface_pressure.data_ptr(), ncol, ncol, float(dt), float(z_max),
                                     dtemp.data_ptr(), dhumid.data_ptr(), _lib.ADD if add else 0,
                                     C.byref(nf) if count else None, _stream(temp)))
        return int(nf.value) if count else None

    def device_status(self) -> int:
        v = C.c_int32(0)
        check(lib.sht_mlp_device_status(self._m, C.byref(v)))
        return int(v.value)

    def __del__(self):
        if getattr(self, "_m", None) is not None and lib is not None:   # lib is None at interpreter exit
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


from .model_states import ModelStates  # noqa: E402,F401
