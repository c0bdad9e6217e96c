"""SpectralTransform, transform!/transform and the spectral operators over libsht.

Reference: SpeedyTransforms/src/spectral_transform.jl (constructor :118-302,
``transform!`` :515-631, allocating ``transform`` :638-682),
SpeedyTransforms/src/spectral_gradients.jl (operators), RingGrids (grids, Field)
and LowerTriangularArrays (Spectrum, LowerTriangularArray).

Layouts. torch tensors are row-major, the reference's arrays column-major, so a
field with K layers is a float32 tensor of shape ``(K, npoints)`` (layer k is row
k, which is exactly the reference's ``field.data[:, k]``) and coefficients are a
complex64 tensor of shape ``(K, nlm)``. One-dimensional tensors are single
layers. Rows may be strided (views into a larger parent, as the reference's fused
"mega-batch" parents); the innermost dimension must be contiguous.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import _lib
from ._lib import DimensionMismatch, check, lib

__all__ = []


# ------------------------------------------------------------------------------------------
# sizes (SpeedyTransforms/src/aliasing.jl)
# ------------------------------------------------------------------------------------------
def _roundup_fft(n: int, small_primes=(2, 3, 5)) -> int:
    n += n % 2
    while True:
        m = n
        for p in small_primes:
            while m % p == 0:
                m //= p
        if m == 1:
            return n
        n += 2


def get_nlat_half(truncation: int, dealiasing: float = 2.0) -> int:
    """aliasing.jl:9-15."""
    return _roundup_fft(math.ceil(((1 + dealiasing) * (truncation - 1) + 1) / 4))


def get_truncation(nlat_half: int, dealiasing: float = 2.0) -> int:
    """aliasing.jl:24-30."""
    return int(math.floor((4 * nlat_half - 1) / (dealiasing + 1))) + 1


# ------------------------------------------------------------------------------------------
# spectrum and grids
# ------------------------------------------------------------------------------------------
class Spectrum:
    """Spectrum(lmax, mmax): 1-based sizes of the packed lower triangle (spectrum.jl:37-62)."""

    def __init__(self, lmax: int, mmax: int | None = None):
        mmax = lmax if mmax is None else mmax
        if mmax < 1 or lmax < mmax:
            raise ValueError(f"Spectrum(lmax={lmax}, mmax={mmax}) needs 1 <= mmax <= lmax")
        self.lmax, self.mmax = int(lmax), int(mmax)
        self.nlm = self.lmax * self.mmax - self.mmax * (self.mmax - 1) // 2

    def offset(self, m: int) -> int:
        return m * self.lmax - m * (m - 1) // 2

    def lm(self, l: int, m: int) -> int:
        """0-based packed index of 0-based degree l and order m."""
        if not (0 <= m < self.mmax and m <= l < self.lmax):
            raise IndexError(f"(l={l}, m={m}) outside {self}")
        return self.offset(m) + l - m

    @property
    def l_indices(self):
        return np.concatenate([np.arange(m, self.lmax) for m in range(self.mmax)])

    @property
    def m_indices(self):
        return np.concatenate([np.full(self.lmax - m, m) for m in range(self.mmax)])

    def __eq__(self, o):
        return isinstance(o, Spectrum) and (self.lmax, self.mmax) == (o.lmax, o.mmax)

    def __hash__(self):
        return hash((self.lmax, self.mmax))

    def __repr__(self):
        return f"Spectrum({self.lmax}, {self.mmax})"


class _GaussianGrid:
    kind: int
    name: str

    def __init__(self, nlat_half: int):
        if nlat_half < 1:
            raise ValueError("nlat_half must be >= 1")
        self.nlat_half = int(nlat_half)
        self.nlat = 2 * self.nlat_half
        half = self._nlons_half()
        self.nlons = np.concatenate([half, half[::-1]])
        self.npoints = int(self.nlons.sum())
        self.nlon_max = int(self.nlons.max())
        self.ring_start = np.concatenate([[0], np.cumsum(self.nlons)[:-1]])

    def eachring(self):
        return [range(int(s), int(s + n)) for s, n in zip(self.ring_start, self.nlons)]

    def __eq__(self, o):
        return type(self) is type(o) and self.nlat_half == o.nlat_half

    def __hash__(self):
        return hash((self.kind, self.nlat_half))

    def __repr__(self):
        return f"{self.name}({self.nlat_half})"


class FullGaussianGrid(_GaussianGrid):
    """4 nlat_half points on every ring (RingGrids/src/grids/full_gaussian.jl:43-45)."""

    kind = _lib.GRID_FULL_GAUSSIAN
    name = "FullGaussianGrid"

    def _nlons_half(self):
        return np.full(self.nlat_half, 4 * self.nlat_half, dtype=np.int64)


class OctahedralGaussianGrid(_GaussianGrid):
    """16 + 4j points on ring j (RingGrids/src/grids/octahedral_gaussian.jl:50-70)."""

    kind = _lib.GRID_OCTAHEDRAL_GAUSSIAN
    name = "OctahedralGaussianGrid"

    def _nlons_half(self):
        return 16 + 4 * np.arange(1, self.nlat_half + 1, dtype=np.int64)


# ------------------------------------------------------------------------------------------
# data containers
# ------------------------------------------------------------------------------------------
def _default_device():
    if not torch.cuda.is_available():
        raise RuntimeError("speedytransforms needs a CUDA device (libsht has no CPU path)")
    return torch.device("cuda", torch.cuda.current_device())


class Field:
    """Gridded data on a ring grid: float32 tensor (K, npoints) or (npoints,)."""

    def __init__(self, data: torch.Tensor, grid: _GaussianGrid):
        if data.shape[-1] != grid.npoints:
            raise DimensionMismatch(f"field of {tuple(data.shape)} does not fit {grid} ({grid.npoints} points)")
        self.data, self.grid = data, grid

    @classmethod
    def zeros(cls, grid, nlayers: int | None = None, device=None):
        shape = (grid.npoints,) if nlayers is None else (nlayers, grid.npoints)
        return cls(torch.zeros(shape, dtype=torch.float32, device=device or _default_device()), grid)

    @property
    def nlayers(self):
        return 1 if self.data.dim() == 1 else self.data.shape[0]

    def __repr__(self):
        return f"Field({self.grid}, K={self.nlayers})"


class LowerTriangularArray:
    """Packed spectral coefficients: complex64 tensor (K, nlm) or (nlm,)."""

    def __init__(self, data: torch.Tensor, spectrum: Spectrum):
        if data.shape[-1] != spectrum.nlm:
            raise DimensionMismatch(f"coefficients of {tuple(data.shape)} do not fit {spectrum} (nlm={spectrum.nlm})")
        self.data, self.spectrum = data, spectrum

    @classmethod
    def zeros(cls, spectrum, nlayers: int | None = None, device=None):
        shape = (spectrum.nlm,) if nlayers is None else (nlayers, spectrum.nlm)
        return cls(torch.zeros(shape, dtype=torch.complex64, device=device or _default_device()), spectrum)

    @property
    def nlayers(self):
        return 1 if self.data.dim() == 1 else self.data.shape[0]

    def similar(self):
        return LowerTriangularArray(torch.empty_like(self.data), self.spectrum)

    def __repr__(self):
        return f"LowerTriangularArray({self.spectrum}, K={self.nlayers})"


def _ld_and_k(t: torch.Tensor, width: int, what: str, host: bool = False):
    if host:
        if t.is_cuda:
            raise ValueError(f"{what} must live in host memory")
    elif not t.is_cuda:
        raise ValueError(f"{what} must live on a CUDA device")
    if t.dim() == 1:
        if t.stride(0) != 1:
            raise ValueError(f"{what} must be contiguous")
        return width, 1
    if t.dim() != 2:
        raise ValueError(f"{what} must be 1-D or 2-D (layers, points)")
    if t.stride(1) != 1:
        raise ValueError(f"{what}: innermost dimension must be contiguous")
    K = t.shape[0]
    return (t.stride(0) if K > 1 else width), K


def _stream_ptr(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _coeff_arg(lta: LowerTriangularArray, S, what, host: bool = False):
    if not isinstance(lta, LowerTriangularArray):
        raise TypeError(f"{what} must be a LowerTriangularArray")
    if lta.data.dtype != torch.complex64:
        raise TypeError(f"{what}: coefficients must be complex64 (NF = Float32)")
    if lta.spectrum != S.spectrum:
        raise DimensionMismatch(f"SpectralTransform for {S.spectrum} and {what} on {lta.spectrum} do not match")
    return _ld_and_k(lta.data, S.spectrum.nlm, what, host)


def _field_arg(f: Field, S, what):
    if not isinstance(f, Field):
        raise TypeError(f"{what} must be a Field")
    if f.data.dtype != torch.float32:
        raise TypeError(f"{what}: field must be float32 (NF = Float32)")
    if f.grid != S.grid:
        raise DimensionMismatch(f"SpectralTransform for {S.grid} and {what} on {f.grid} do not match")
    return _ld_and_k(f.data, S.grid.npoints, what)


# ------------------------------------------------------------------------------------------
# SpectralTransform
# ------------------------------------------------------------------------------------------
_PRECISIONS = {"fp32": _lib.PREC_FP32, "bf16x3": _lib.PREC_BF16X3, "bf16x5": _lib.PREC_BF16X5,
               "fp16x3": _lib.PREC_FP16X3}


class SpectralTransform:
    """Precomputed spectral transform (spectral_transform.jl:118-302) living on one GPU.

    ``SpectralTransform(spectrum, grid, nlayers=K, LegendreShortcut="linear",
    precision="fp32")`` or, as the reference's convenience constructors,
    ``SpectralTransform(grid=..., truncation=..., one_more_degree=...)`` and
    ``SpectralTransform(spectrum, Grid=OctahedralGaussianGrid, nlat_half=0, dealiasing=2)``.
    ``precision`` selects the Legendre arithmetic: "fp32" (CUDA cores), "bf16x3"
    (tensor cores, split BF16, 3 products), "bf16x5" (tensor cores, Legendre
    polynomials in 3 BF16 pieces, 5 products) or "fp16x3" (scaled split FP16).
    """

    def __init__(self, spectrum: Spectrum | None = None, grid: _GaussianGrid | None = None, *, NF=torch.float32,
                 nlayers: int = 1, LegendreShortcut: str = "linear", precision: str = "fp32", Grid=None,
                 nlat_half: int = 0, truncation: int = 0, dealiasing: float = 2.0, one_more_degree: bool = False,
                 device=None):
        if NF not in (torch.float32, "Float32", np.float32):
            raise NotImplementedError("libsht computes in Float32 (the reference's default NF)")
        if spectrum is None:
            if grid is None:
                raise ValueError("give a spectrum, a grid, or both")
            truncation = truncation if truncation > 0 else get_truncation(grid.nlat_half, dealiasing)
            spectrum = Spectrum(truncation + int(one_more_degree), truncation)
        if grid is None:
            Grid = Grid or FullGaussianGrid
            nlat_half = nlat_half if nlat_half > 0 else get_nlat_half(spectrum.mmax, dealiasing)
            grid = Grid(nlat_half)
        if LegendreShortcut not in _lib.SHORTCUTS:
            raise ValueError(f"unknown LegendreShortcut {LegendreShortcut!r}")
        if precision not in _PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        self.spectrum, self.grid = spectrum, grid
        self.nlayers = int(nlayers)
        self.precision = precision
        self.LegendreShortcut = LegendreShortcut
        self.device = torch.device(device) if device is not None else _default_device()
        d = _lib.ShtDesc(grid.kind, grid.nlat_half, spectrum.lmax, spectrum.mmax, self.nlayers,
                         _PRECISIONS[precision], _lib.SHORTCUTS[LegendreShortcut],
                         self.device.index if self.device.index is not None else torch.cuda.current_device())
        h = C.c_void_p()
        self._plan = None
        check(lib.sht_plan_create(C.byref(d), C.byref(h)))
        self._plan = h
        info = _lib.ShtInfo()
        check(lib.sht_plan_info(h, C.byref(info)))
        self.info = info
        nlat, nh = grid.nlat, grid.nlat_half
        latd = np.zeros(nlat)
        w = np.zeros(nlat)
        nl = np.zeros(nlat, dtype=np.int32)
        mt = np.zeros(nh, dtype=np.int32)
        check(lib.sht_plan_tables(h, latd.ctypes.data_as(C.POINTER(C.c_double)),
                                  w.ctypes.data_as(C.POINTER(C.c_double)),
                                  nl.ctypes.data_as(C.POINTER(C.c_int32)), mt.ctypes.data_as(C.POINTER(C.c_int32))))
        self.latd, self.quadrature_weights, self.mmax_truncation = latd, w, mt
        self.coslat = np.cos(np.radians(latd))
        self.norm_sphere = 2 * math.sqrt(math.pi)

    def __del__(self):
        if getattr(self, "_plan", None) is not None and lib is not None:   # lib is None at interpreter exit
            lib.sht_plan_destroy(self._plan)
            self._plan = None

    @property
    def handle(self):
        return self._plan

    def device_status(self) -> int:
        """Synchronise and return (then clear) the plan's device status word (0 = ok)."""
        v = C.c_int32(0)
        check(lib.sht_device_status(self._plan, C.byref(v)))
        return int(v.value)

    def diag_wait_expiry(self, limit_us: int = 20000):
        """Failure-detection check of the tensor-core kernels' bounded waits: one thread
        on the plan's device waits, through the same routine, for an mbarrier phase that
        nothing completes and gives up after ``limit_us`` microseconds, storing
        ``SHT_STATUS_DIAG_EXPIRED`` (9) in the status word that ``device_status`` reads."""
        check(lib.sht_diag_wait_expiry(self._plan, int(limit_us), _stream_ptr(self.device)))

    def host_wait(self):
        """Make the current stream wait for the copies of host-memory coefficients that
        earlier transforms issued (synchronise it afterwards to read them)."""
        check(lib.sht_host_wait(self._plan, _stream_ptr(self.device)))

    def set_host_chunk(self, layers: int):
        """Layers per chunk of the host-memory transforms (allocates the staging slots)."""
        check(lib.sht_plan_set_host_chunk(self._plan, int(layers)))

    def autotune(self, nlayers: int | None = None):
        """Time the Legendre kernels at ``nlayers`` layers for each tile width and keep the
        fastest (results are bitwise independent of the choice): the SIMT tile width per
        direction for "fp32" plans, the tcgen05 column tile width (64 or 128) for the
        tensor-core precisions. Returns the (synthesis, analysis) widths."""
        cols = (C.c_int32 * 2)()
        check(lib.sht_plan_autotune(self._plan, int(nlayers or self.nlayers), _stream_ptr(self.device), cols))
        return int(cols[0]), int(cols[1])

    def set_tile_columns(self, synthesis: int, analysis: int | None = None):
        """Set the Legendre tile widths directly (as autotune's choices)."""
        check(lib.sht_plan_set_tile_columns(self._plan, int(synthesis), int(analysis or synthesis)))

    @property
    def fusion(self) -> bool:
        """True when transforms run fused (FFT and Legendre stage in one launch per
        direction, thread-block clusters passing the Fourier rows through shared memory);
        same bits as the separate kernels. Settable; FP32 plans of small truncations only.
        On by default for full Gaussian grids up to nlat 64, where it measured faster."""
        mode = C.c_int32(0)
        check(lib.sht_plan_get_fusion(self._plan, C.byref(mode), None))
        return bool(mode.value)

    @fusion.setter
    def fusion(self, on: bool):
        check(lib.sht_plan_set_fusion(self._plan, 1 if on else 0))

    @property
    def fusion_available(self) -> bool:
        ok = C.c_int32(0)
        check(lib.sht_plan_get_fusion(self._plan, None, C.byref(ok)))
        return bool(ok.value)

    @property
    def prime_stage(self) -> str:
        """Where the ring FFTs run their first stage when it is a prime radix p >= 64:
        "tensor" (one tcgen05 launch for all such rings, three TF32 products) or "direct"
        (inside the FFT kernel on the FP32 pipes, the default: faster at T511 x 64). Settable.
        The two agree to FP32 rounding, not bit for bit."""
        mode = C.c_int32(0)
        check(lib.sht_plan_get_prime_stage(self._plan, C.byref(mode), None))
        return "tensor" if mode.value else "direct"

    @prime_stage.setter
    def prime_stage(self, where: str):
        if where not in ("tensor", "direct"):
            raise ValueError(f"prime_stage must be 'tensor' or 'direct', not {where!r}")
        check(lib.sht_plan_set_prime_stage(self._plan, 1 if where == "tensor" else 0))

    @property
    def prime_stage_available(self) -> bool:
        """True when some ring's FFT starts with a prime radix p >= 64."""
        ok = C.c_int32(0)
        check(lib.sht_plan_get_prime_stage(self._plan, None, C.byref(ok)))
        return bool(ok.value)

    def __repr__(self):
        return (f"SpectralTransform({self.spectrum}, {self.grid}, nlayers={self.nlayers}, "
                f"precision={self.precision!r})")


class MatrixSpectralTransform:
    """Dense-matrix spectral transform (matrix_transform.jl:56-260):
    ``MatrixSpectralTransform(spectrum, grid, nlayers=K, precision="fp32")``; the
    matrices are the transforms of unit vectors. "fp32" multiplies as three TF32 products
    on the tensor cores (the reference's Float32 mul!, to FP32 rounding), "bf16x3" /
    "fp16x3" / "bf16x5" as split 16-bit products.
    Used through ``transform_`` / ``transform`` like a SpectralTransform (no ``add``)."""

    def __init__(self, spectrum: Spectrum, grid: _GaussianGrid, *, nlayers: int = 1, LegendreShortcut: str = "linear",
                 precision: str = "fp32", device=None):
        if precision not in _PRECISIONS:
            raise ValueError(f"unknown precision {precision!r}")
        self.spectrum, self.grid = spectrum, grid
        self.nlayers = int(nlayers)
        self.precision = precision
        self.device = torch.device(device) if device is not None else _default_device()
        d = _lib.ShtDesc(grid.kind, grid.nlat_half, spectrum.lmax, spectrum.mmax, self.nlayers,
                         _PRECISIONS[precision], _lib.SHORTCUTS[LegendreShortcut],
                         self.device.index if self.device.index is not None else torch.cuda.current_device())
        h = C.c_void_p()
        self._m = None
        check(lib.sht_matrix_create(C.byref(d), C.byref(h)))
        self._m = h

    @property
    def handle(self):
        return self._m

    def device_status(self) -> int:
        v = C.c_int32(0)
        check(lib.sht_matrix_device_status(self._m, C.byref(v)))
        return int(v.value)

    def __del__(self):
        if getattr(self, "_m", None) is not None and lib is not None:
            lib.sht_matrix_destroy(self._m)
            self._m = None

    def __repr__(self):
        return (f"MatrixSpectralTransform({self.spectrum}, {self.grid}, nlayers={self.nlayers}, "
                f"precision={self.precision!r})")


class Batch:
    """Many transforms in one grouped launch per stage (sht_batch_*): all syntheses,
    then all analyses, each item with its own scratch.

    ``Batch([(out, in, S, flags...), ...])`` where each entry is
    ``(Field, LowerTriangularArray, S)`` for a synthesis or
    ``(LowerTriangularArray, Field, S)`` for an analysis, optionally followed by a dict
    ``{"unscale_coslat": bool, "add": bool}``. The arrays are bound at construction.
    ``run()`` launches the grouped kernels, ``run_each()`` the same transforms one call
    each, ``capture()``/``launch()`` a CUDA graph of ``run()``, ``autotune()`` picks the
    Legendre tile width. FP32 plans.
    """

    def __init__(self, entries):
        items = (_lib.ShtBatchItem * len(entries))()
        self._keep = []
        self.device = None
        for i, e in enumerate(entries):
            out, inp, S = e[0], e[1], e[2]
            opts = e[3] if len(e) > 3 else {}
            if isinstance(out, Field) and isinstance(inp, LowerTriangularArray):
                ldg, K = _field_arg(out, S, "field")
                ldc, K2 = _coeff_arg(inp, S, "coeffs")
                _check_k(S, K, K2)
                flags = (_lib.UNSCALE_COSLAT if opts.get("unscale_coslat") else 0) | (_lib.ADD if opts.get("add") else 0)
                items[i] = _lib.ShtBatchItem(S.handle.value, _lib.SYNTHESIS, inp.data.data_ptr(), ldc,
                                             out.data.data_ptr(), ldg, K, flags)
            elif isinstance(out, LowerTriangularArray) and isinstance(inp, Field):
                ldc, K = _coeff_arg(out, S, "coeffs")
                ldg, K2 = _field_arg(inp, S, "field")
                _check_k(S, K, K2)
                items[i] = _lib.ShtBatchItem(S.handle.value, _lib.ANALYSIS, out.data.data_ptr(), ldc,
                                             inp.data.data_ptr(), ldg, K, _lib.ADD if opts.get("add") else 0)
            else:
                raise TypeError("batch entries are (Field, LowerTriangularArray, S) or (LowerTriangularArray, Field, S)")
            self._keep += [out, inp, S]
            self.device = S.device
        h = C.c_void_p()
        self._b = None
        check(lib.sht_batch_create(items, len(entries), C.byref(h)))
        self._b = h

    def run(self):
        check(lib.sht_batch_run(self._b, _stream_ptr(self.device)))

    def run_each(self):
        check(lib.sht_batch_run_each(self._b, _stream_ptr(self.device)))

    def capture(self):
        check(lib.sht_batch_capture(self._b, _stream_ptr(self.device)))

    def launch(self):
        check(lib.sht_batch_launch(self._b, _stream_ptr(self.device)))

    def autotune(self) -> int:
        v = C.c_int32(0)
        check(lib.sht_batch_autotune(self._b, _stream_ptr(self.device), C.byref(v)))
        return int(v.value)

    def __del__(self):
        if getattr(self, "_b", None) is not None and lib is not None:
            lib.sht_batch_destroy(self._b)
            self._b = None


# ------------------------------------------------------------------------------------------
# transforms
# ------------------------------------------------------------------------------------------
def _check_k(S, K, *others):
    if K > S.nlayers:
        raise DimensionMismatch(f"{K} layers exceed the transform's nlayers = {S.nlayers}")
    for o in others:
        if o != K:
            raise DimensionMismatch(f"number of layers differ: {K} vs {o}")


def transform_(out, inp, S: SpectralTransform, *, unscale_coslat: bool = False, add: bool = False):
    """transform!(out, in, S): synthesis if ``out`` is a Field, analysis if it is a
    LowerTriangularArray (spectral_transform.jl:515-531, 579-593). Coefficients may live
    in host memory (page-locked for overlap; the field on the device): the copies then
    run inside the call, pipelined over chunks of layers on the plan's copy streams
    (sht_synthesize_host / sht_analyze_host); host results are complete after
    ``S.host_wait()`` and a synchronisation of the current stream."""
    dev = S.device
    if isinstance(S, MatrixSpectralTransform):
        return _matrix_transform_(out, inp, S, unscale_coslat=unscale_coslat, add=add)
    if isinstance(out, Field) and isinstance(inp, LowerTriangularArray):
        ldg, K = _field_arg(out, S, "field")
        host = isinstance(inp.data, torch.Tensor) and not inp.data.is_cuda
        ldc, K2 = _coeff_arg(inp, S, "coeffs", host)
        _check_k(S, K, K2)
        flags = (_lib.UNSCALE_COSLAT if unscale_coslat else 0) | (_lib.ADD if add else 0)
        fn = lib.sht_synthesize_host if host else lib.sht_synthesize
        check(fn(S.handle, inp.data.data_ptr(), ldc, out.data.data_ptr(), ldg, K, flags, _stream_ptr(dev)))
        return out
    if isinstance(out, LowerTriangularArray) and isinstance(inp, Field):
        if unscale_coslat:
            raise TypeError("unscale_coslat applies to spectral-to-grid transforms only")
        host = isinstance(out.data, torch.Tensor) and not out.data.is_cuda
        ldc, K = _coeff_arg(out, S, "coeffs", host)
        ldg, K2 = _field_arg(inp, S, "field")
        _check_k(S, K, K2)
        if host and add:
            raise TypeError("add=True needs device coefficients")
        fn = lib.sht_analyze_host if host else lib.sht_analyze
        check(fn(S.handle, inp.data.data_ptr(), ldg, out.data.data_ptr(), ldc, K, _lib.ADD if add else 0,
                 _stream_ptr(dev)))
        return out
    raise TypeError("transform_(out, in, S) needs (Field, LowerTriangularArray) or (LowerTriangularArray, Field)")


def _matrix_transform_(out, inp, M, *, unscale_coslat=False, add=False):
    """transform! with a MatrixSpectralTransform (matrix_transform.jl:196-260)."""
    if add:
        raise TypeError("MatrixSpectralTransform has no add option (matrix_transform.jl:228-260)")
    dev = M.device
    if isinstance(out, Field) and isinstance(inp, LowerTriangularArray):
        ldg, K = _field_arg(out, M, "field")
        ldc, K2 = _coeff_arg(inp, M, "coeffs")
        _check_k(M, K, K2)
        check(lib.sht_matrix_synthesize(M.handle, inp.data.data_ptr(), ldc, out.data.data_ptr(), ldg, K,
                                        _lib.UNSCALE_COSLAT if unscale_coslat else 0, _stream_ptr(dev)))
        return out
    if isinstance(out, LowerTriangularArray) and isinstance(inp, Field):
        if unscale_coslat:
            raise TypeError("unscale_coslat applies to spectral-to-grid transforms only")
        ldc, K = _coeff_arg(out, M, "coeffs")
        ldg, K2 = _field_arg(inp, M, "field")
        _check_k(M, K, K2)
        check(lib.sht_matrix_analyze(M.handle, inp.data.data_ptr(), ldg, out.data.data_ptr(), ldc, K, 0,
                                     _stream_ptr(dev)))
        return out
    raise TypeError("transform_(out, in, M) needs (Field, LowerTriangularArray) or (LowerTriangularArray, Field)")


def spec2grid_pullback_(coeffs_bar, field_bar, S: SpectralTransform, *, unscale_coslat: bool = False,
                        add: bool = True):
    """Adjoint of the synthesis ``transform_(field, coeffs, S; unscale_coslat)``:
    ``coeffs_bar (+)= S^T field_bar`` (spec2grid_pullback!,
    SpeedyTransformsEnzymeExt.jl:263-289; accumulates by default, as the reference)."""
    ldc, K = _coeff_arg(coeffs_bar, S, "coeffs_bar")
    ldg, K2 = _field_arg(field_bar, S, "field_bar")
    _check_k(S, K, K2)
    flags = (_lib.UNSCALE_COSLAT if unscale_coslat else 0) | (_lib.ADD if add else 0)
    check(lib.sht_synthesize_adjoint(S.handle, field_bar.data.data_ptr(), ldg, coeffs_bar.data.data_ptr(), ldc, K,
                                     flags, _stream_ptr(S.device)))
    return coeffs_bar


def grid2spec_pullback_(field_bar, coeffs_bar, S: SpectralTransform, *, add: bool = True):
    """Adjoint of the analysis ``transform_(coeffs, field, S)``: ``field_bar (+)= A^T coeffs_bar``
    (grid2spec_pullback!, SpeedyTransformsEnzymeExt.jl:294-323; accumulates by default)."""
    ldg, K = _field_arg(field_bar, S, "field_bar")
    ldc, K2 = _coeff_arg(coeffs_bar, S, "coeffs_bar")
    _check_k(S, K, K2)
    check(lib.sht_analyze_adjoint(S.handle, coeffs_bar.data.data_ptr(), ldc, field_bar.data.data_ptr(), ldg, K,
                                  _lib.ADD if add else 0, _stream_ptr(S.device)))
    return field_bar


def transform(inp, S: SpectralTransform, *, unscale_coslat: bool = False):
    """Allocating transform (spectral_transform.jl:638-661)."""
    K = inp.nlayers if inp.data.dim() == 2 else None
    if isinstance(inp, LowerTriangularArray):
        out = Field.zeros(S.grid, K, device=inp.data.device)
        return transform_(out, inp, S, unscale_coslat=unscale_coslat)
    if isinstance(inp, Field):
        out = LowerTriangularArray.zeros(S.spectrum, K, device=inp.data.device)
        return transform_(out, inp, S)
    raise TypeError("transform(in, S) needs a Field or a LowerTriangularArray")


# ------------------------------------------------------------------------------------------
# operators (spectral_gradients.jl)
# ------------------------------------------------------------------------------------------
def _coeffs(S, *arrs):
    lds, Ks = zip(*[_coeff_arg(a, S, "coefficients") for a in arrs])
    if len(set(lds)) != 1:
        raise DimensionMismatch("operator arguments need equal row strides")
    _check_k(S, Ks[0], *Ks[1:])
    return lds[0], Ks[0]


def _divcurl(fn, out, u, v, S, flipsign, add, radius):
    ld, K = _coeffs(S, out, u, v)
    flags = (_lib.FLIPSIGN if flipsign else 0) | (_lib.ADD if add else 0)
    check(fn(S.handle, out.data.data_ptr(), u.data.data_ptr(), v.data.data_ptr(), ld, K, flags, float(radius),
             _stream_ptr(S.device)))
    return out


class Operators:
    """Several spectral operators run in one kernel launch (sht_operators), each with the
    arguments and the result of its single call (curl_, divergence_, laplace_,
    inverse_laplace_, gradient_, UV_from_vordiv_), applied in the order added, so that
    operators accumulating (add=True) into the same output match the separate calls bit
    for bit. No counterpart in the reference, whose time step calls the operators one by
    one (SpeedyWeather/src/dynamics/tendencies.jl:161-214, 585-594). Inputs must not
    overlap any output of the set; overlapping outputs must be the same array. The set
    keeps references to its arrays and can be run repeatedly (and captured in a graph)."""

    def __init__(self, S):
        self.S = S
        self._ops = []
        self._keep = []

    def _add(self, kind, flags, out, out2, a, b, radius):
        arrs = [x for x in (out, out2, a, b) if x is not None]
        ld, K = _coeffs(self.S, *arrs)
        if len(self._ops) >= _lib.MAX_OPS:
            raise ValueError(f"at most {_lib.MAX_OPS} operators per set")
        ptr = lambda x: x.data.data_ptr() if x is not None else None   # noqa: E731
        self._ops.append(_lib.ShtOp(kind, flags, ptr(out), ptr(out2), ptr(a), ptr(b), ld, K, 0, float(radius)))
        self._keep.extend(arrs)
        return self

    def curl(self, out, u, v, *, flipsign=False, add=False, radius=1.0):
        flags = (_lib.FLIPSIGN if flipsign else 0) | (_lib.ADD if add else 0)
        return self._add(_lib.OP_CURL, flags, out, None, u, v, radius)

    def divergence(self, out, u, v, *, flipsign=False, add=False, radius=1.0):
        flags = (_lib.FLIPSIGN if flipsign else 0) | (_lib.ADD if add else 0)
        return self._add(_lib.OP_DIVERGENCE, flags, out, None, u, v, radius)

    def laplace(self, out, alms, *, add=False, flipsign=False, inverse=False, radius=1.0):
        flags = (_lib.FLIPSIGN if flipsign else 0) | (_lib.ADD if add else 0) | (_lib.INVERSE if inverse else 0)
        return self._add(_lib.OP_LAPLACE, flags, out, None, alms, None, radius)

    def gradient(self, dpdx, dpdy, p, *, radius=1.0):
        return self._add(_lib.OP_GRADIENT, 0, dpdx, dpdy, p, None, radius)

    def UV_from_vordiv(self, U, V, vor, div=None, *, radius=1.0):
        return self._add(_lib.OP_UV_FROM_VORDIV, 0, U, V, vor, div, radius)

    def __len__(self):
        return len(self._ops)

    def __call__(self):
        arr = (_lib.ShtOp * max(1, len(self._ops)))(*self._ops)
        check(lib.sht_operators(self.S.handle, arr, len(self._ops), _stream_ptr(self.S.device)))


def curl_(out, u, v, S, *, flipsign=False, add=False, radius=1.0):
    """curl!(curl, u, v, S; flipsign, add, radius) (spectral_gradients.jl:30-41)."""
    return _divcurl(lib.sht_curl, out, u, v, S, flipsign, add, radius)


def divergence_(out, u, v, S, *, flipsign=False, add=False, radius=1.0):
    """divergence!(div, u, v, S; flipsign, add, radius) (spectral_gradients.jl:51-62)."""
    return _divcurl(lib.sht_divergence, out, u, v, S, flipsign, add, radius)


def curl(u, v, S, **kw):
    return curl_(u.similar(), u, v, S, **kw)


def divergence(u, v, S, **kw):
    return divergence_(u.similar(), u, v, S, **kw)


def UV_from_vordiv_(U, V, vor, div, S, *, radius=1.0):
    """UV_from_vordiv!(U, V, vor, div, S; radius) (spectral_gradients.jl:309-329)."""
    ld, K = _coeffs(S, U, V, vor, div)
    check(lib.sht_uv_from_vordiv(S.handle, U.data.data_ptr(), V.data.data_ptr(), vor.data.data_ptr(),
                                 div.data.data_ptr(), ld, K, float(radius), _stream_ptr(S.device)))
    return U, V


def UV_from_vor_(U, V, vor, S, *, radius=1.0):
    """UV_from_vor!(U, V, vor, S; radius) (spectral_gradients.jl:248-267)."""
    ld, K = _coeffs(S, U, V, vor)
    check(lib.sht_uv_from_vordiv(S.handle, U.data.data_ptr(), V.data.data_ptr(), vor.data.data_ptr(), None, ld, K,
                                 float(radius), _stream_ptr(S.device)))
    return U, V


def UV_from_vordiv(vor, div, S, **kw):
    return UV_from_vordiv_(vor.similar(), vor.similar(), vor, div, S, **kw)


def UV_from_vor(vor, S, **kw):
    return UV_from_vor_(vor.similar(), vor.similar(), vor, S, **kw)


def laplace_(out, alms, S, *, add=False, flipsign=False, inverse=False, radius=1.0):
    """∇²!(out, alms, S; add, flipsign, inverse, radius) (spectral_gradients.jl:386-409)."""
    ld, K = _coeffs(S, out, alms)
    flags = (_lib.ADD if add else 0) | (_lib.FLIPSIGN if flipsign else 0) | (_lib.INVERSE if inverse else 0)
    check(lib.sht_laplace(S.handle, out.data.data_ptr(), alms.data.data_ptr(), ld, K, flags, float(radius),
                          _stream_ptr(S.device)))
    return out


def inverse_laplace_(out, alms, S, *, add=False, flipsign=False, radius=1.0):
    """∇⁻²!(out, alms, S; add, flipsign, radius) (spectral_gradients.jl:468-478)."""
    return laplace_(out, alms, S, add=add, flipsign=flipsign, inverse=True, radius=radius)


def laplace(alms, S, **kw):
    return laplace_(alms.similar(), alms, S, **kw)


def inverse_laplace(alms, S, **kw):
    return inverse_laplace_(alms.similar(), alms, S, **kw)


def gradient_(dpdx, dpdy, p, S, *, radius=1.0):
    """∇!(dpdx, dpdy, p, S; radius) (spectral_gradients.jl:483-507)."""
    ld, K = _coeffs(S, dpdx, dpdy, p)
    check(lib.sht_gradient(S.handle, dpdx.data.data_ptr(), dpdy.data.data_ptr(), p.data.data_ptr(), ld, K,
                           float(radius), _stream_ptr(S.device)))
    return dpdx, dpdy


def gradient(p, S, **kw):
    return gradient_(p.similar(), p.similar(), p, S, **kw)
