"""Host-side mirror of Inti.jl's operator surface over libinti_b200.

Names, argument meaning and error behaviour follow the reference:

* ``Laplace(dim=)``, ``Helmholtz(k=, dim=)`` (src/kernels.jl:118-128, 310-335);
* ``SingleLayerKernel``, ``DoubleLayerKernel``, ``AdjointDoubleLayerKernel``,
  ``HyperSingularKernel`` (src/kernels.jl:52-112);
* ``IntegralOperator(K, target, source=target)`` whose entries are
  ``K(x_i, y_j)·w_j`` (src/nystrom.jl:67-96), applied on the fly on the GPU,
  and ``assemble_matrix`` (src/nystrom.jl:103-124);
* ``single_double_layer`` / ``adj_double_layer_hypersingular``
  (src/api.jl:65-212) with ``compression=dict(method="b200", precision=...)``
  and ``correction=dict(method="dim"|"none")``; the result is ``S = A + δS``,
  a lazy map like ``LinearMap(Smat) + LinearMap(δS)`` (src/api.jl:179-184)
  whose apply runs the pair kernel and the CSR correction in one pass;
* ``bdim_correction`` (src/bdim.jl:50-196) built on the GPU, on the surface
  (target === source) or for other targets near it (src/api.jl:105-148);
* ``single_double_layer_potential`` / ``IntegralPotential`` (src/api.jl:220-226,
  src/nystrom.jl:20-38);
* ``volume_potential`` with the VDIM correction (src/api.jl:282-378,
  src/vdim.jl:30-130; 2D Laplace);
* ``gmres`` for ``shift·I + Σ c_t·op_t`` (the IterativeSolvers call of
  docs/src/examples/poisson.jl:166-168), plain FP64 or mixed precision.

Arrays cross the boundary as numpy arrays; complex densities are
``complex128`` (interleaved re/im, as ComplexF64).
"""
from __future__ import annotations

import ctypes as C
import numbers
import threading
import warnings
import weakref

import numpy as np

from . import _lib as L
from .geometry import Quadrature

__all__ = [
    "Context",
    "default_context",
    "Laplace",
    "Helmholtz",
    "SingleLayerKernel",
    "DoubleLayerKernel",
    "AdjointDoubleLayerKernel",
    "HyperSingularKernel",
    "GpuOperator",
    "CombinedFieldOperator",
    "BatchOperator",
    "LinearCombination",
    "IntegralOperator",
    "assemble_matrix",
    "CorrectionMatrix",
    "bdim_correction",
    "single_double_layer",
    "adj_double_layer_hypersingular",
    "IntegralPotential",
    "single_double_layer_potential",
    "volume_potential",
    "I",
    "gmres",
    "COMPRESSION_METHODS",
    "CORRECTION_METHODS",
]

COMPRESSION_METHODS = ("none", "b200")
CORRECTION_METHODS = ("none", "dim")


# ----------------------------------------------------------------------------
# context
# ----------------------------------------------------------------------------
class Context:
    """One CUDA device and stream (``inti_ctx``).  All handles created through
    a context live on its device; calls on one context are serialised."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self.lib = L.load()
        h = C.c_void_p()
        st = self.lib.inti_ctx_create(int(device), C.c_void_p(stream) if stream else None, C.byref(h))
        L.check(st, None)
        self.handle = h
        self.device = device
        self._fin = weakref.finalize(self, self.lib.inti_ctx_destroy, h)

    def check(self, status: int) -> None:
        L.check(status, self.handle)

    @property
    def stream(self) -> int:
        return self.lib.inti_ctx_stream(self.handle) or 0

    @property
    def launch_count(self) -> int:
        return int(self.lib.inti_ctx_launch_count(self.handle))

    def set_profiling(self, enable: bool) -> None:
        """Start (clearing earlier records) or stop per-kernel event timing."""
        self.check(self.lib.inti_ctx_set_profiling(self.handle, int(bool(enable))))

    def profile(self, kernel: str) -> tuple[float, int]:
        """(total device ms, launches) recorded for a kernel class."""
        ms, n = C.c_double(), L.I64()
        self.check(self.lib.inti_ctx_profile(self.handle, kernel.encode(), C.byref(ms), C.byref(n)))
        return ms.value, n.value

    def synchronize(self) -> None:
        self.check(self.lib.inti_ctx_synchronize(self.handle))

    def set_autotune(self, enable: bool) -> None:
        """Pick pair-kernel launch shapes of large operators by timing (on by
        default; see ``GpuOperator.tuning``)."""
        self.check(self.lib.inti_ctx_set_autotune(self.handle, int(bool(enable))))

    def set_symmetric(self, enable: bool) -> None:
        """Use the symmetric pair kernel for square operators created
        afterwards (on by default; see ``GpuOperator.tuning``)."""
        self.check(self.lib.inti_ctx_set_symmetric(self.handle, int(bool(enable))))

    def set_single_launch(self, enable: bool) -> None:
        """Apply small FP64 operators (at most 2^20 pairs, 65,536 sources) created afterwards
        in the single-launch form (on by default; see ``GpuOperator.tuning``)."""
        self.check(self.lib.inti_ctx_set_single_launch(self.handle, int(bool(enable))))

    def set_gmres_small(self, max_unknowns: int) -> None:
        """GMRES on systems of at most ``max_unknowns`` unknowns (default
        8192) runs each Arnoldi step in one single-CTA kernel with a host
        check every four steps; 0 turns that form off."""
        self.check(self.lib.inti_ctx_set_gmres_small(self.handle, int(max_unknowns)))

    def set_partial_budget(self, nbytes: float) -> None:
        """Bytes of partial sums a symmetric operator created afterwards may
        hold before its work is split into panels run one after another
        (0 restores the default, 2e9)."""
        self.check(self.lib.inti_ctx_set_partial_budget(self.handle, float(nbytes)))

    def selftest_math(self) -> dict:
        """Accuracy of the device's fast rsqrt / reciprocal / e^{iθ} helpers (see the ABI)."""
        out = (C.c_double * 6)()
        self.check(self.lib.inti_selftest_math(self.handle, out))
        return {"rsqrt_f64_maxrel": out[0], "expi_f64_maxabs_25": out[1], "expi_f64_maxabs_1000": out[2],
                "expi_f32_maxabs_25": out[3], "rsqrt_cube_f64_maxrel": out[4],
                "rcp_f64_maxrel": out[5]}

    def measure_peaks(self) -> dict:
        a, b, c, t = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        self.check(self.lib.inti_measure_peaks(self.handle, C.byref(a), C.byref(b), C.byref(c)))
        self.check(self.lib.inti_measure_peak_tf32(self.handle, C.byref(t)))
        return {"fp64_flops": a.value, "fp32_flops": b.value, "mufu_ops": c.value, "tf32_flops": t.value}


_default = None
_default_lock = threading.Lock()


def default_context() -> Context:
    global _default
    with _default_lock:
        if _default is None:
            _default = Context(0)
        return _default


# ----------------------------------------------------------------------------
# differential operators and kernels
# ----------------------------------------------------------------------------
class Laplace:
    """``-Δu`` in ``dim`` dimensions (src/kernels.jl:118-128)."""

    pde = L.LAPLACE
    k = 0.0

    def __init__(self, *, dim: int):
        if dim not in (2, 3):
            raise L.ArgumentError(L.E_ARG, "dim must be 2 or 3")
        self.dim = dim

    def default_density_eltype(self):
        return np.float64

    def __repr__(self):
        return f"Laplace operator in {self.dim} dimensions: -Δu"


class Helmholtz:
    """``-Δu - k²u`` in ``dim`` dimensions (src/kernels.jl:310-335)."""

    pde = L.HELMHOLTZ

    def __init__(self, *, k, dim: int):
        if dim not in (2, 3):
            raise L.ArgumentError(L.E_ARG, "dim must be 2 or 3")
        if isinstance(k, complex):
            if k.imag < 0:
                raise L.ArgumentError(L.E_ARG, "k must have a non-negative imaginary part")
            if k.imag == 0:
                k = k.real
        self.k = k
        self.dim = dim

    def default_density_eltype(self):
        return np.complex128

    def __repr__(self):
        return f"Helmholtz operator in {self.dim} dimensions: -Δu - k²u"


class _Kernel:
    kind = -1

    def __init__(self, op):
        self.op = op

    def __repr__(self):
        return f"{type(self).__name__}({self.op!r})"


class SingleLayerKernel(_Kernel):
    kind = L.SL


class DoubleLayerKernel(_Kernel):
    kind = L.DL


class AdjointDoubleLayerKernel(_Kernel):
    kind = L.ADL


class HyperSingularKernel(_Kernel):
    kind = L.HS


# ----------------------------------------------------------------------------
# device handles
# ----------------------------------------------------------------------------
def _quad_handle(q: Quadrature, ctx: Context):
    """Device copy of a quadrature, cached on the object per context."""
    cache = q.__dict__.setdefault("_b200", {})
    key = id(ctx)
    if key in cache:
        return cache[key][0]
    h = C.c_void_p()
    nrm = q.normals
    ctx.check(ctx.lib.inti_quad_create(ctx.handle, q.dim, len(q), L.dptr(q.coords), L.dptr(nrm),
                                       L.dptr(q.weights), int(q.nq), C.byref(h)))
    fin = weakref.finalize(q, ctx.lib.inti_quad_destroy, h)
    cache[key] = (h, fin, ctx)
    return h


def _as_density(x, cplx: bool, n: int, name="x") -> np.ndarray:
    x = np.asarray(x)
    if x.shape[0] != n:
        raise L.DimensionMismatch(L.E_SHAPE, f"{name} has {x.shape[0]} rows, expected {n}")
    dt = np.complex128 if cplx else np.float64
    if not cplx and np.iscomplexobj(x):
        raise L.ArgumentError(L.E_ARG, "complex density for a real operator")
    return np.ascontiguousarray(x, dtype=dt)


class CorrectionMatrix:
    """Sparse correction δ on the device (``inti_csr``), the counterpart of
    the ``SparseMatrixCSC`` that ``bdim_correction`` returns
    (src/bdim.jl:193-194).  ``to_scipy()`` gives a CSR copy on the host."""

    def __init__(self, handle, ctx: Context):
        self.handle = handle
        self.ctx = ctx
        m, n, nnz, dt = L.I64(), L.I64(), L.I64(), C.c_int()
        ctx.check(ctx.lib.inti_csr_info(handle, C.byref(m), C.byref(n), C.byref(nnz), C.byref(dt)))
        self.shape = (m.value, n.value)
        self.nnz = nnz.value
        self.dtype = np.complex128 if dt.value == L.C128 else np.float64
        self._fin = weakref.finalize(self, ctx.lib.inti_csr_destroy, handle)

    @classmethod
    def from_csr(cls, indptr, indices, data, shape, ctx: Context | None = None):
        ctx = ctx or default_context()
        indptr = np.ascontiguousarray(indptr, dtype=np.int64)
        indices = np.ascontiguousarray(indices, dtype=np.int32)
        cplx = np.iscomplexobj(data)
        data = np.ascontiguousarray(data, dtype=np.complex128 if cplx else np.float64)
        h = C.c_void_p()
        ctx.check(ctx.lib.inti_csr_create(ctx.handle, shape[0], shape[1], len(indices), L.dptr(indptr),
                                          L.dptr(indices), L.dptr(data), L.C128 if cplx else L.F64,
                                          C.byref(h)))
        return cls(h, ctx)

    @classmethod
    def from_csc_1based(cls, colptr, rowval, nzval, shape, ctx: Context | None = None):
        """From Julia's ``SparseMatrixCSC`` arrays (1-based colptr/rowval)."""
        ctx = ctx or default_context()
        colptr = np.ascontiguousarray(colptr, dtype=np.int64)
        rowval = np.ascontiguousarray(rowval, dtype=np.int64)
        cplx = np.iscomplexobj(nzval)
        nzval = np.ascontiguousarray(nzval, dtype=np.complex128 if cplx else np.float64)
        h = C.c_void_p()
        ctx.check(ctx.lib.inti_csr_create_from_csc(ctx.handle, shape[0], shape[1], len(rowval),
                                                   L.dptr(colptr), L.dptr(rowval), L.dptr(nzval),
                                                   L.C128 if cplx else L.F64, C.byref(h)))
        return cls(h, ctx)

    def arrays(self):
        """(indptr int64, indices int32, data) copied from the device."""
        m, _ = self.shape
        rp = np.empty(m + 1, np.int64)
        col = np.empty(self.nnz, np.int32)
        val = np.empty(self.nnz, self.dtype)
        self.ctx.check(self.ctx.lib.inti_csr_download(self.handle, L.dptr(rp), L.dptr(col), L.dptr(val)))
        return rp, col, val

    def to_scipy(self):
        import scipy.sparse as sp

        rp, col, val = self.arrays()
        return sp.csr_matrix((val, col, rp), shape=self.shape)

    def __matmul__(self, x):
        x = _as_density(x, self.dtype == np.complex128, self.shape[1])
        y = np.zeros(self.shape[0], self.dtype)
        self.ctx.check(self.ctx.lib.inti_csr_apply(self.handle, L.dptr(x), L.dptr(y), None, None, 0))
        return y

    def apply_device(self, x_ptr: int, y_ptr: int, alpha=1.0, beta=0.0) -> None:
        """Stream-ordered ``y = alpha*C*x + beta*y`` on device pointers."""
        self.ctx.check(self.ctx.lib.inti_csr_apply(self.handle, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                                   L.cpair(alpha), L.cpair(beta), 1))


# ----------------------------------------------------------------------------
# lazy linear maps
# ----------------------------------------------------------------------------
class _UniformScaling:
    """``I`` of LinearAlgebra: combine as ``a*I + op``."""

    def __init__(self, s=1.0):
        self.s = s

    def __mul__(self, c):
        return _UniformScaling(self.s * c)

    __rmul__ = __mul__

    def __truediv__(self, c):
        return _UniformScaling(self.s / c)

    def __neg__(self):
        return _UniformScaling(-self.s)

    def __add__(self, other):
        return LinearCombination.of(other) + self

    __radd__ = __add__

    def __sub__(self, other):
        return (-LinearCombination.of(other)) + self

    def __rsub__(self, other):
        return LinearCombination.of(other) + (-self)


I = _UniformScaling(1.0)


class _Map:
    """Common algebra: ``a*A``, ``A + B``, ``A + s*I``, ``A @ x``."""

    def __add__(self, other):
        return LinearCombination.of(self) + other

    __radd__ = __add__

    def __sub__(self, other):
        return LinearCombination.of(self) + (-LinearCombination.of(other)
                                             if not isinstance(other, _UniformScaling) else -other)

    def __rsub__(self, other):
        return (-LinearCombination.of(self)) + other

    def __mul__(self, c):
        if isinstance(c, numbers.Number):
            return LinearCombination(0.0, [(c, self)])
        return NotImplemented

    __rmul__ = __mul__

    def __neg__(self):
        return LinearCombination(0.0, [(-1.0, self)])

    def __matmul__(self, x):
        return self.matvec(x)

    def __mul_vec__(self, x):
        return self.matvec(x)


class LinearCombination(_Map):
    """``shift·I + Σ coef_t·op_t`` over GPU operators sharing one quadrature."""

    def __init__(self, shift, terms):
        self.shift = shift
        self.terms = list(terms)

    @staticmethod
    def of(x):
        if isinstance(x, LinearCombination):
            return x
        if isinstance(x, _UniformScaling):
            return LinearCombination(x.s, [])
        if isinstance(x, GpuOperator):
            return LinearCombination(0.0, [(1.0, x)])
        raise TypeError(f"cannot combine {type(x).__name__}")

    def __add__(self, other):
        if isinstance(other, _UniformScaling):
            return LinearCombination(self.shift + other.s, self.terms)
        o = LinearCombination.of(other)
        return LinearCombination(self.shift + o.shift, self.terms + o.terms)

    def __mul__(self, c):
        if isinstance(c, numbers.Number):
            return LinearCombination(self.shift * c, [(a * c, t) for a, t in self.terms])
        return NotImplemented

    __rmul__ = __mul__

    def __neg__(self):
        return self * -1.0

    @property
    def shape(self):
        return self.terms[0][1].shape

    @property
    def is_complex(self):
        return any(t.is_complex for _, t in self.terms) or any(
            isinstance(c, complex) and c.imag != 0 for c, _ in self.terms) or (
            isinstance(self.shift, complex) and self.shift.imag != 0)

    def matvec(self, x):
        cplx = self.is_complex
        x = np.asarray(x)
        x = x.astype(np.complex128 if cplx else np.float64)
        y = complex(self.shift) * x if cplx else float(np.real(self.shift)) * x
        for c, t in self.terms:
            yt = t.matvec(x)
            y = y + (c * yt)
        return y


class GpuOperator(_Map):
    """A Nyström operator ``A (+ δ)`` resident on the GPU (``inti_op``).

    ``matvec`` (``@``) and ``mul(y, x, alpha, beta)`` (the 5-argument mul! of
    LinearAlgebra) run the on-the-fly pair kernel and, when present, the
    correction SpMV fused in its epilogue.  ``rmatvec`` applies the
    transpose.  Arrays of shape ``(n, nrhs)`` are applied column by column.
    """

    def __init__(self, kernel: _Kernel, target: Quadrature, source: Quadrature,
                 correction: CorrectionMatrix | None = None, precision: str = "fp64",
                 ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.kernel = kernel
        self.target = target
        self.source = source
        self.correction = correction
        self.precision = precision
        op = kernel.op
        if target.dim != op.dim or source.dim != op.dim:
            raise L.DimensionMismatch(L.E_SHAPE, "quadrature dimension differs from the operator's")
        prec = {"fp64": L.FP64, "fp32c": L.FP32C, "mixed": L.FP64}.get(precision)
        if prec is None:
            raise L.ArgumentError(L.E_ARG, f"unknown precision {precision!r}")
        th = _quad_handle(target, self.ctx)
        sh = _quad_handle(source, self.ctx)
        h = C.c_void_p()
        k = complex(getattr(op, "k", 0.0))
        self.ctx.check(self.ctx.lib.inti_op_create(self.ctx.handle, op.pde, kernel.kind, k.real, k.imag, th, sh,
                                                   correction.handle if correction else None, prec,
                                                   C.byref(h)))
        self.handle = h
        self._fin = weakref.finalize(self, self.ctx.lib.inti_op_destroy, h)
        self.shape = (len(target), len(source))
        self.is_complex = op.pde == L.HELMHOLTZ
        self.dtype = np.complex128 if self.is_complex else np.float64

    def _apply(self, x, transpose=False, y=None, alpha=1.0, beta=0.0):
        m, n = self.shape
        if transpose:
            m, n = n, m
        fn = self.ctx.lib.inti_op_apply_transpose if transpose else self.ctx.lib.inti_op_apply
        dt = self.dtype
        if (type(x) is np.ndarray and x.ndim == 1 and x.shape[0] == n and x.dtype == dt and x.flags.c_contiguous
                and (y is None or (type(y) is np.ndarray and y.ndim == 1 and y.shape[0] == m and y.dtype == dt
                                   and y.flags.c_contiguous and y.flags.writeable))):
            # one contiguous column of the operator's type: no conversions
            if y is None:
                y, beta = np.empty(m, dt), 0.0
            self.ctx.check(fn(self.handle, x.ctypes.data, n, y.ctypes.data, m, 1, L.cpair(alpha), L.cpair(beta), 0))
            return y
        x = np.asarray(x)
        single = x.ndim == 1
        if x.shape[0] != n:
            raise L.DimensionMismatch(L.E_SHAPE, f"x has {x.shape[0]} rows, expected {n}")
        X = _as_density(x.reshape(n, -1) if single else x, self.is_complex, n)
        X = np.asfortranarray(X)
        nrhs = X.shape[1]
        if y is None:
            Y = np.zeros((m, nrhs), self.dtype, order="F")
            beta = 0.0
        else:
            Y = np.asfortranarray(np.asarray(y, dtype=self.dtype).reshape(m, -1))
        self.ctx.check(fn(self.handle, L.dptr(X), n, L.dptr(Y), m, nrhs, L.cpair(alpha), L.cpair(beta), 0))
        out = Y[:, 0] if single else Y
        if y is not None:
            np.copyto(y, out.reshape(np.shape(y)))
            return y
        return out

    def matvec(self, x):
        return self._apply(x)

    def rmatvec(self, x):
        """``transpose(A) * x`` (not conjugated)."""
        return self._apply(x, transpose=True)

    def mul(self, y, x, alpha=1.0, beta=0.0):
        """``y = alpha*A*x + beta*y`` in place."""
        return self._apply(x, y=y, alpha=alpha, beta=beta)

    def apply_device(self, x_ptr: int, y_ptr: int, nrhs: int = 1, alpha=1.0, beta=0.0,
                     ldx: int | None = None, ldy: int | None = None) -> None:
        """Stream-ordered apply on device pointers (no copies, no sync)."""
        m, n = self.shape
        self.ctx.check(self.ctx.lib.inti_op_apply(self.handle, C.c_void_p(x_ptr), ldx or n, C.c_void_p(y_ptr),
                                                  ldy or m, nrhs, L.cpair(alpha), L.cpair(beta), 1))

    def grad_sources(self, g, sigma):
        """Gradients of J with dJ/du = g for u = A·sigma (Laplace SL/DL):
        returns dict(sigma, coords, normals, weights)."""
        m, n = self.shape
        g = _as_density(g, False, m, "g")
        sigma = _as_density(sigma, False, n, "sigma")
        dim = self.source.dim
        out = {"sigma": np.empty(n), "coords": np.empty((n, dim)), "normals": np.empty((n, dim)),
               "weights": np.empty(n)}
        self.ctx.check(self.ctx.lib.inti_op_grad_sources(self.handle, L.dptr(g), L.dptr(sigma),
                                                         L.dptr(out["sigma"]), L.dptr(out["coords"]),
                                                         L.dptr(out["normals"]), L.dptr(out["weights"]), 0))
        return out

    @property
    def tuning(self) -> dict:
        """Launch shape of the pair kernel: targets per thread and split."""
        t, s = C.c_int32(), C.c_int32()
        self.ctx.check(self.ctx.lib.inti_op_tuning(self.handle, C.byref(t), C.byref(s)))
        return {"targets_per_thread": t.value, "split": s.value,
                "symmetric": bool(self.ctx.lib.inti_op_symmetric(self.handle) == 1),
                "panels": int(self.ctx.lib.inti_op_panels(self.handle)),
                "single_launch": bool(self.ctx.lib.inti_op_single_launch(self.handle) == 1)}

    def set_shard(self, rank: int, nranks: int) -> None:
        """Compute only rank ``rank``'s share of the node pairs (symmetric
        operators): each apply returns a partial product over all rows, and
        the ranks' partials sum to the whole (one all-reduce).  Rank 0
        carries the correction and ``beta*y``.  ``nranks=1`` restores the
        whole operator."""
        self.ctx.check(self.ctx.lib.inti_op_set_shard(self.handle, int(rank), int(nranks)))

    def grad_sources_device(self, g_ptr: int, sigma_ptr: int, dsigma_ptr: int, dcoords_ptr: int,
                            dnormals_ptr: int, dweights_ptr: int) -> None:
        """Stream-ordered ``grad_sources`` on device pointers (no copies, no
        sync); an output pointer of 0 skips that gradient."""
        v = lambda p: C.c_void_p(p or None)  # noqa: E731
        self.ctx.check(self.ctx.lib.inti_op_grad_sources(self.handle, v(g_ptr), v(sigma_ptr), v(dsigma_ptr),
                                                         v(dcoords_ptr), v(dnormals_ptr), v(dweights_ptr), 1))


class CombinedFieldOperator(GpuOperator):
    """``c_D·D + c_S·S`` of two GPU operators (a double layer and a single
    layer over the same nodes, corrections included), applied in one pass
    over the node pairs.  The lazy sum ``c_D*D + c_S*S`` of the reference's
    LinearMaps (docs/src/examples/helmholtz_scattering.jl:485-486) gives the
    same product with two passes."""

    def __init__(self, D: GpuOperator, S: GpuOperator, c_D=1.0, c_S=1.0, precision: str | None = None):
        if not (isinstance(D.kernel, DoubleLayerKernel) and isinstance(S.kernel, SingleLayerKernel)):
            raise L.ArgumentError(L.E_ARG, "expected a double-layer and a single-layer operator")
        if D.target is not S.target or D.source is not S.source:
            raise L.ArgumentError(L.E_ARG, "both operators must share target and source")
        self.ctx = D.ctx
        self.kernel = D.kernel
        self.target, self.source = D.target, D.source
        self.correction = None
        self.precision = precision or D.precision
        prec = {"fp64": L.FP64, "fp32c": L.FP32C}[self.precision]
        op = D.kernel.op
        k = complex(getattr(op, "k", 0.0))
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.inti_op_create_combined(
            self.ctx.handle, op.pde, k.real, k.imag, _quad_handle(D.target, self.ctx),
            _quad_handle(D.source, self.ctx), D.correction.handle if D.correction else None,
            S.correction.handle if S.correction else None, L.cpair(c_D), L.cpair(c_S), prec, C.byref(h)))
        self.handle = h
        self._keep = (D, S)
        self._fin = weakref.finalize(self, self.ctx.lib.inti_op_destroy, h)
        self.shape = D.shape
        self.is_complex = D.is_complex
        self.dtype = D.dtype


class BatchOperator:
    """Block-diagonal ``diag(A_1 + C_1, …, A_S + C_S)`` over many surfaces,
    applied to many right-hand sides in one launch (``inti_batch``).

    ``kind`` is ``"SL"``, ``"DL"`` or ``"CF"`` (``c_dl·DL + c_sl·SL``).
    ``corrections`` is a list of ``(δS, δD)`` pairs (``bdim_correction``
    output) or None.  Densities are ``(N_total, nrhs)`` arrays over the
    concatenated nodes, surface order as given.
    """

    def __init__(self, op, quads, kind="SL", corrections=None, c_dl=1.0, c_sl=1.0, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        self.op = op
        self.quads = list(quads)
        kinds = {"SL": L.SL, "DL": L.DL, "CF": L.CF}
        if kind not in kinds:
            raise L.ArgumentError(L.E_ARG, f"unknown batch kernel {kind!r}")
        qh = (C.c_void_p * len(self.quads))(*[_quad_handle(q, self.ctx).value for q in self.quads])
        dS = dD = None
        if corrections is not None:
            dS = (C.c_void_p * len(self.quads))(*[(c[0].handle.value if c and c[0] else None) for c in corrections])
            dD = (C.c_void_p * len(self.quads))(*[(c[1].handle.value if c and c[1] else None) for c in corrections])
        k = complex(getattr(op, "k", 0.0))
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.inti_batch_create(self.ctx.handle, len(self.quads), qh, op.pde, kinds[kind],
                                                      k.real, k.imag, L.cpair(c_dl), L.cpair(c_sl), dD, dS,
                                                      C.byref(h)))
        self.handle = h
        self._keep = (corrections,)
        self._fin = weakref.finalize(self, self.ctx.lib.inti_batch_destroy, h)
        self.n = int(self.ctx.lib.inti_batch_size(h))
        self.offsets = np.cumsum([0] + [len(q) for q in self.quads])
        self.is_complex = op.pde == L.HELMHOLTZ
        self.dtype = np.complex128 if self.is_complex else np.float64

    def apply(self, X, precision: str = "fp64", Y=None, alpha=1.0, beta=0.0):
        prec = {"fp64": L.FP64, "tf32": L.TF32}.get(precision)
        if prec is None:
            raise L.ArgumentError(L.E_ARG, f"unknown batch precision {precision!r}")
        X = np.asarray(X)
        single = X.ndim == 1
        X = X.reshape(self.n, -1) if single else X
        if X.shape[0] != self.n:
            raise L.DimensionMismatch(L.E_SHAPE, f"X has {X.shape[0]} rows, expected {self.n}")
        if not self.is_complex and np.iscomplexobj(X):
            raise L.ArgumentError(L.E_ARG, "complex density for a real operator")
        X = np.asfortranarray(X, dtype=self.dtype)  # no copy when already column-major of this dtype
        nrhs = X.shape[1]
        if Y is None:
            Yo = np.zeros((self.n, nrhs), self.dtype, order="F")
            beta = 0.0
        else:
            Yin = np.asarray(Y)
            Yo = Yin if (Yin.dtype == self.dtype and Yin.flags.f_contiguous and Yin.shape == (self.n, nrhs)) else \
                np.asfortranarray(Yin.reshape(self.n, -1), dtype=self.dtype).copy(order="F")
        self.ctx.check(self.ctx.lib.inti_batch_apply(self.handle, prec, L.dptr(X), self.n, L.dptr(Yo), self.n, nrhs,
                                                     L.cpair(alpha), L.cpair(beta), 0))
        return Yo[:, 0] if single else Yo

    def gmres(self, B, *, shift=0.0, X0=None, rtol: float = 1e-10, restart: int = 30, maxiter: int = 300,
              mode: str = "fp64", out=None):
        """Solve ``(shift·I + A_s + C_s) x = b`` for every surface and column
        in lockstep; returns ``(X, stats)`` with ``stats["relres"]`` the
        per-system FP64 relative residuals ``(S, nrhs)``.  ``B`` that is
        already complex128 and column-major is used without a copy; ``out``
        (complex128, column-major, ``(N_total, nrhs)``) receives the solution
        in place (page-locked buffers make the copies fast)."""
        B = np.asarray(B)
        single = B.ndim == 1
        Bm = B.reshape(self.n, -1) if single else B
        if not (Bm.dtype == np.complex128 and Bm.flags.f_contiguous and Bm.shape[0] == self.n):
            Bm = np.asfortranarray(_as_density(Bm, True, self.n))
        nrhs = Bm.shape[1]
        if out is not None:
            X = out
            if not (X.dtype == np.complex128 and X.flags.f_contiguous and X.shape == (self.n, nrhs)):
                raise L.ArgumentError(L.E_ARG, "out must be a column-major complex128 array of shape (N_total, nrhs)")
            if X0 is None:
                X[...] = 0
            else:
                X[...] = np.asarray(X0).reshape(self.n, nrhs)
        else:
            X = np.zeros_like(Bm, order="F") if X0 is None else np.asfortranarray(
                _as_density(np.asarray(X0).reshape(self.n, -1), True, self.n)).copy(order="F")
        rel = np.zeros(len(self.quads) * nrhs)
        st = L.GmresStats()
        m = {"fp64": L.GMRES_FP64, "mixed": L.GMRES_MIXED}[mode]
        self.ctx.check(self.ctx.lib.inti_batch_gmres(self.handle, L.cpair(shift), L.dptr(Bm), L.dptr(X), self.n, nrhs,
                                                     rtol, restart, maxiter, m, 0, L.dptr(rel), C.byref(st)))
        stats = st.as_dict()
        stats["relres_all"] = rel.reshape(len(self.quads), nrhs)
        return (X[:, 0] if single else X), stats

    def apply_device(self, x_ptr: int, y_ptr: int, nrhs: int, precision: str = "fp64", alpha=1.0, beta=0.0):
        prec = {"fp64": L.FP64, "tf32": L.TF32}[precision]
        self.ctx.check(self.ctx.lib.inti_batch_apply(self.handle, prec, C.c_void_p(x_ptr), self.n, C.c_void_p(y_ptr),
                                                     self.n, nrhs, L.cpair(alpha), L.cpair(beta), 1))


class IntegralOperator(GpuOperator):
    """``IntegralOperator(K, target, source=target)`` (src/nystrom.jl:79-89):
    entries ``K(x_i, y_j)·w_j`` applied on the fly, never stored."""

    def __init__(self, kernel: _Kernel, target: Quadrature, source: Quadrature | None = None,
                 precision: str = "fp64", ctx: Context | None = None):
        super().__init__(kernel, target, target if source is None else source, None, precision, ctx)

    def __getitem__(self, idx):
        i, j = idx
        return assemble_matrix(self)[i, j]


def assemble_matrix(iop: GpuOperator) -> np.ndarray:
    """Dense matrix of the (uncorrected) operator, assembled on the GPU
    (src/nystrom.jl:103-124).  Column-major like Julia's ``Matrix``."""
    m, n = iop.shape
    out = np.empty((m, n), iop.dtype, order="F")
    iop.ctx.check(iop.ctx.lib.inti_op_assemble(iop.handle, L.dptr(out), 0))
    return out


# ----------------------------------------------------------------------------
# correction and the high-level constructors
# ----------------------------------------------------------------------------
def bdim_correction(op, target: Quadrature, source: Quadrature, *, green_multiplier=None,
                    derivative: bool = False, maxdist: float = float("inf"), ctx: Context | None = None):
    """``(δS, δD)`` of the density-interpolation method (src/bdim.jl:50-196),
    built on the GPU.  With ``target is source`` each element corrects its own
    nodes (src/quadrature.jl:250-256) and the multiplier defaults to -1/2.
    Otherwise every target within ``maxdist`` of its nearest source node is
    corrected through that node's element (src/quadrature.jl:264-286), and
    ``green_multiplier`` (a scalar or one value per target) is required."""
    ctx = ctx or default_context()
    hsrc = _quad_handle(source, ctx)
    hs, hd = C.c_void_p(), C.c_void_p()
    k = complex(getattr(op, "k", 0.0))
    if target is source:
        gm = None
        if green_multiplier is not None:
            gm = np.ascontiguousarray(np.broadcast_to(np.asarray(green_multiplier, float), (len(source),)))
        ctx.check(ctx.lib.inti_dim_correction(ctx.handle, op.pde, k.real, k.imag, hsrc, int(bool(derivative)),
                                              L.dptr(gm), C.byref(hs), C.byref(hd)))
    else:
        if green_multiplier is None:
            raise L.ArgumentError(L.E_ARG, "off-surface targets need a green multiplier")
        gm = np.ascontiguousarray(np.broadcast_to(np.asarray(green_multiplier, float), (len(target),)))
        htgt = _quad_handle(target, ctx)
        ctx.check(ctx.lib.inti_dim_correction_targets(ctx.handle, op.pde, k.real, k.imag, htgt, hsrc,
                                                      int(bool(derivative)), L.dptr(gm), float(maxdist),
                                                      C.byref(hs), C.byref(hd)))
    return CorrectionMatrix(hs, ctx), CorrectionMatrix(hd, ctx)


def _normalize_compression(compression):
    """src/utils.jl:189-198: validate the method, default tol 1e-8."""
    compression = dict(compression or {"method": "b200"})
    method = str(compression.get("method", "b200")).lstrip(":")
    if method not in COMPRESSION_METHODS:
        raise L.ArgumentError(
            L.E_ARG, f"Unknown compression.method {method}. Available options: {COMPRESSION_METHODS}")
    compression["method"] = method
    compression.setdefault("tol", 1e-8)
    compression.setdefault("precision", "fp64")
    return compression


def _normalize_correction(correction, target, source):
    """src/utils.jl:200-228 for the methods implemented here."""
    correction = dict(correction or {"method": "dim"})
    method = str(correction.get("method", "dim")).lstrip(":")
    if method not in CORRECTION_METHODS:
        raise L.ArgumentError(
            L.E_ARG, f"Unknown correction.method {method}. Available options: {CORRECTION_METHODS}")
    correction["method"] = method
    if method == "dim":
        if "target_location" in correction and target is source and \
                str(correction["target_location"]).lstrip(":") != "on":
            warnings.warn("ignoring target_location field in correction since target === source")
        if target is not source and "target_location" not in correction and "green_multiplier" not in correction:
            raise L.ArgumentError(L.E_ARG, "missing target_location field in correction")
        if "target_location" in correction and "green_multiplier" in correction:
            raise L.ArgumentError(L.E_ARG, "conflicting target_location and green_multiplier fields in correction")
        if "maxdist" not in correction and target is not source:
            warnings.warn("missing maxdist field in correction: setting to Inf")
        correction.setdefault("maxdist", float("inf"))
    return correction


def _green_multiplier(s: str) -> float:
    """src/nystrom.jl:196-207."""
    s = str(s).lstrip(":")
    if s == "inside":
        return -1.0
    if s == "outside":
        return 0.0
    if s == "on":
        return -0.5
    raise L.ArgumentError(L.E_ARG, f"Unknown target location {s}. Expected :inside, :outside, or :on")


def single_double_layer(*, op, target: Quadrature, source: Quadrature, compression=None,
                        correction=None, derivative: bool = False, ctx: Context | None = None):
    """``(S, D)`` (or ``(K, H)`` when ``derivative``) as GPU operators with the
    correction fused (src/api.jl:65-187).  ``compression["precision"]`` is
    ``"fp64"`` or ``"fp32c"`` (FP32 pairs, compensated sums, FP64 SpMV)."""
    ctx = ctx or default_context()
    compression = _normalize_compression(compression)
    correction = _normalize_correction(correction, target, source)
    G = AdjointDoubleLayerKernel(op) if derivative else SingleLayerKernel(op)
    dG = HyperSingularKernel(op) if derivative else DoubleLayerKernel(op)
    prec = compression["precision"]
    dS = dD = None
    if correction["method"] == "dim":
        if "green_multiplier" in correction:
            gm = np.asarray(correction["green_multiplier"], float)
            if gm.shape != (len(target),):
                raise L.DimensionMismatch(L.E_SHAPE, "green_multiplier must have one entry per target")
        else:
            loc = "on" if target is source else correction["target_location"]
            gm = _green_multiplier(loc)
        dS, dD = bdim_correction(op, target, source, green_multiplier=gm, derivative=derivative,
                                 maxdist=correction["maxdist"], ctx=ctx)
    S = GpuOperator(G, target, source, dS, prec, ctx)
    D = GpuOperator(dG, target, source, dD, prec, ctx)
    return S, D


def adj_double_layer_hypersingular(*, op, target: Quadrature, source: Quadrature | None = None,
                                   compression=None, correction=None, ctx: Context | None = None):
    """src/api.jl:197-212."""
    return single_double_layer(op=op, target=target, source=target if source is None else source,
                               compression=compression, correction=correction, derivative=True, ctx=ctx)


def volume_potential(*, op, target: Quadrature, source: Quadrature, compression=None, correction=None,
                     ctx: Context | None = None):
    """``V`` (+ ``δV``) of src/api.jl:282-378: the volume potential of the
    single-layer kernel from a volume quadrature, with the VDIM correction
    (``correction=dict(method="dim", boundary=Q_boundary, [target_location |
    green_multiplier], [maxdist], [interpolation_order])``).  The boundary
    layer operators it needs are built with their own DIM correction (off the
    surface for volume targets); the result is one GPU operator with δV fused
    into its epilogue."""
    from .vdim import vdim_correction

    ctx = ctx or default_context()
    correction = _normalize_correction(correction, target, source)
    compression = _normalize_compression(compression)
    G = SingleLayerKernel(op)
    prec = compression["precision"]
    V = GpuOperator(G, target, source, None, prec, ctx)
    if correction["method"] == "none":
        return V
    if "green_multiplier" in correction:
        gm = np.asarray(correction["green_multiplier"], float)
        loc = None
    else:
        loc = "inside" if target is source else correction["target_location"]
        gm = np.full(len(target), _green_multiplier(loc))
    if "boundary" not in correction:
        raise L.ArgumentError(L.E_ARG, "Missing correction.boundary field for :dim method on a volume potential")
    boundary = correction["boundary"]
    bc = {k: v for k, v in correction.items() if k not in ("boundary", "interpolation_order", "center")}
    if loc is not None:
        bc = dict(bc, target_location=loc)
    bc.setdefault("maxdist", correction.get("maxdist", float("inf")))
    if "S_b2d" in correction and "D_b2d" in correction:
        S, D = correction["S_b2d"], correction["D_b2d"]
    else:
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            S, D = single_double_layer(op=op, target=target, source=boundary, compression=compression,
                                       correction=bc, ctx=ctx)
    dV = vdim_correction(op, target, source, boundary, S, D, V, green_multiplier=gm,
                         interpolation_order=correction.get("interpolation_order"),
                         maxdist=correction.get("maxdist", float("inf")), center=correction.get("center"), ctx=ctx)
    return GpuOperator(G, target, source, dV, prec, ctx)


class IntegralPotential:
    """``IntegralPotential(kernel, quadrature)``; ``pot[σ]`` returns a callable
    that evaluates ``Σ_j K(x, y_j) σ_j w_j`` at an array of points
    (src/nystrom.jl:20-38), batched through one GPU operator."""

    def __init__(self, kernel: _Kernel, source: Quadrature, ctx: Context | None = None):
        self.kernel = kernel
        self.source = source
        self.ctx = ctx or default_context()

    def __getitem__(self, sigma):
        sigma = np.asarray(sigma)

        def evaluate(x):
            from .geometry import points

            pts = np.atleast_2d(np.asarray(x, float))
            op = GpuOperator(self.kernel, points(pts), self.source, None, "fp64", self.ctx)
            u = op.matvec(sigma)
            return u if np.ndim(x) > 1 else u[0]

        return evaluate


def single_double_layer_potential(*, op, source: Quadrature, ctx: Context | None = None):
    """src/api.jl:220-226."""
    return IntegralPotential(SingleLayerKernel(op), source, ctx), IntegralPotential(DoubleLayerKernel(op), source, ctx)


# ----------------------------------------------------------------------------
# solver
# ----------------------------------------------------------------------------
def gmres(L_, b, *, x0=None, rtol: float = 1e-10, restart: int = 100, maxiter: int = 1000,
          mode: str = "fp64", history: bool = False):
    """Solve ``L x = b`` for ``L = shift·I + Σ c_t·op_t`` on the GPU.

    ``mode="fp64"``: restarted GMRES on the FP64 operators.  ``mode="mixed"``:
    FP64 residuals, FP32C inner GMRES, iterative refinement.  Convergence is
    ``‖b − L x‖₂ ≤ rtol·‖b‖₂`` with the residual formed in FP64.  Returns
    ``(x, stats)``; ``stats["history"]`` holds relative residuals when
    requested.
    """
    Lc = LinearCombination.of(L_) if not isinstance(L_, LinearCombination) else L_
    if not Lc.terms:
        raise L.ArgumentError(L.E_ARG, "the operator has no GPU terms")
    ops = [t for _, t in Lc.terms]
    ctx = ops[0].ctx
    cplx = Lc.is_complex
    n = ops[0].shape[1]
    b = _as_density(b, cplx, n, "b")
    x = np.zeros(n, b.dtype) if x0 is None else _as_density(x0, cplx, n, "x0").copy()
    handles = (C.c_void_p * len(ops))(*[o.handle.value for o in ops])
    coefs = (C.c_double * (2 * len(ops)))()
    for i, (c, _) in enumerate(Lc.terms):
        c = complex(c)
        coefs[2 * i], coefs[2 * i + 1] = c.real, c.imag
    sh = L.cpair(Lc.shift)
    hist = np.zeros(maxiter + 1) if history else None
    st = L.GmresStats()
    m = {"fp64": L.GMRES_FP64, "mixed": L.GMRES_MIXED}.get(mode)
    if m is None:
        raise L.ArgumentError(L.E_ARG, f"unknown mode {mode!r}")
    ctx.check(ctx.lib.inti_gmres(ctx.handle, len(ops), handles, coefs, sh, L.dptr(b), L.dptr(x), rtol,
                                 restart, maxiter, m, 0, L.dptr(hist), C.byref(st)))
    stats = st.as_dict()
    if history:
        stats["history"] = hist[: st.iterations + 1]
    return x, stats
