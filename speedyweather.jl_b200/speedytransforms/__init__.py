"""speedytransforms: SpeedyTransforms' spectral transform on B200 (sm_100a).

Host-side mirror of the reference interface (SpeedyTransforms/src/spectral_transform.jl,
SpeedyTransforms/src/spectral_gradients.jl) over the C ABI of libsht.so:

* ``Spectrum``, ``FullGaussianGrid``, ``OctahedralGaussianGrid``,
  ``LowerTriangularArray``, ``Field`` -- the reference's data layouts;
* ``SpectralTransform(spectrum, grid; NF, nlayers, LegendreShortcut, precision)``;
* ``transform_(out, in, S)`` is ``transform!`` (direction by argument types),
  ``transform(in, S)`` allocates;
* operators ``curl_``, ``divergence_``, ``UV_from_vor_``, ``UV_from_vordiv_``,
  ``laplace_`` (``∇²!``), ``inverse_laplace_`` (``∇⁻²!``), ``gradient_`` (``∇!``)
  and their allocating forms; ``Operators`` -- several of them in one kernel launch;
* ``MatrixSpectralTransform`` -- the dense-matrix transforms (3xTF32 or split 16-bit, tcgen05);
* ``Batch`` -- many transforms in one grouped launch per stage, CUDA-graph capture;
* ``spec2grid_pullback_``, ``grid2spec_pullback_`` -- the adjoints of the transforms.

Every compute call runs the CUDA kernels of libsht; there is no CPU path.
"""
from ._lib import DimensionMismatch, ShtError  # noqa: F401
from .core import (  # noqa: F401
    Batch,
    Field,
    FullGaussianGrid,
    LowerTriangularArray,
    MatrixSpectralTransform,
    OctahedralGaussianGrid,
    Operators,
    SpectralTransform,
    Spectrum,
    UV_from_vor,
    UV_from_vor_,
    UV_from_vordiv,
    UV_from_vordiv_,
    curl,
    curl_,
    divergence,
    divergence_,
    get_nlat_half,
    get_truncation,
    gradient,
    gradient_,
    grid2spec_pullback_,
    inverse_laplace,
    inverse_laplace_,
    laplace,
    laplace_,
    spec2grid_pullback_,
    transform,
    transform_,
)

__version__ = "0.1.0"
from .dycore_step import DycoreStep  # noqa: F401,E402
