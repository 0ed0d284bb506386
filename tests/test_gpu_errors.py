"""Error behaviour at the boundary: invalid arguments raise (status codes
mapped to ArgumentError / DimensionMismatch / ...), never crash, and leave
the context usable."""
import ctypes as C

import numpy as np
import pytest

import inti_b200 as inti
from inti_b200 import _lib as L

pytestmark = pytest.mark.gpu


def test_shape_and_type_errors(ctx):
    q = inti.ellipsoid_quadrature(2, 5)
    A = inti.IntegralOperator(inti.SingleLayerKernel(inti.Laplace(dim=3)), q, ctx=ctx)
    with pytest.raises(inti.DimensionMismatch):
        A @ np.ones(len(q) + 1)
    with pytest.raises(inti.ArgumentError):
        A @ (np.ones(len(q)) * 1j)
    with pytest.raises(inti.ArgumentError):
        inti.IntegralOperator(inti.SingleLayerKernel(inti.Laplace(dim=3)), q, precision="fp16", ctx=ctx)
    # still usable
    assert np.isfinite(A @ np.ones(len(q))).all()


def test_unsupported_and_missing_normals(ctx):
    c = inti.kite_quadrature(10, 3)
    with pytest.raises(inti.UnsupportedError):
        inti.IntegralOperator(inti.SingleLayerKernel(inti.Helmholtz(k=1.0, dim=2)), c, ctx=ctx)
    q = inti.ellipsoid_quadrature(2, 5)
    with pytest.raises(inti.UnsupportedError):
        inti.IntegralOperator(inti.SingleLayerKernel(inti.Helmholtz(k=1.0 + 0.5j, dim=3)), q, ctx=ctx)
    pts = inti.points(q.coords * 2)
    with pytest.raises(inti.ArgumentError):
        inti.GpuOperator(inti.AdjointDoubleLayerKernel(inti.Laplace(dim=3)), pts, q, ctx=ctx)


def test_nonfinite_inputs_rejected(ctx):
    q = inti.ellipsoid_quadrature(2, 5)
    bad = inti.Quadrature(q.coords.copy(), q.normals, q.weights, q.nq)
    bad.coords[3, 1] = np.nan
    with pytest.raises(inti.NonFiniteError):
        inti.IntegralOperator(inti.SingleLayerKernel(inti.Laplace(dim=3)), bad, ctx=ctx)


def test_csr_validation(ctx):
    with pytest.raises(inti.ArgumentError):  # unsorted columns
        inti.CorrectionMatrix.from_csr([0, 2], [1, 0], [1.0, 2.0], (1, 2), ctx)
    with pytest.raises(inti.ArgumentError):  # column out of range
        inti.CorrectionMatrix.from_csr([0, 1], [5], [1.0], (1, 2), ctx)
    with pytest.raises(inti.DimensionMismatch):
        inti.CorrectionMatrix.from_csr([0, 1], [0], [1.0], (2, 2), ctx)
    # Julia's 1-based CSC converts to the same CSR
    m = inti.CorrectionMatrix.from_csc_1based([1, 2, 4], [2, 1, 2], [5.0, 6.0, 7.0], (2, 2), ctx)
    rp, col, val = m.arrays()
    assert rp.tolist() == [0, 1, 3] and col.tolist() == [1, 0, 1] and val.tolist() == [6.0, 5.0, 7.0]
    assert np.allclose(m @ np.array([1.0, 2.0]), [12.0, 19.0])


def test_correction_shape_and_dtype_checked(ctx):
    q = inti.ellipsoid_quadrature(2, 5)
    wrong = inti.CorrectionMatrix.from_csr([0, 1], [0], [1.0], (1, len(q)), ctx)
    with pytest.raises(inti.DimensionMismatch):
        inti.GpuOperator(inti.SingleLayerKernel(inti.Laplace(dim=3)), q, q, wrong, ctx=ctx)
    dS, _ = inti.bdim_correction(inti.Laplace(dim=3), q, q, ctx=ctx)
    with pytest.raises(inti.ArgumentError):
        inti.GpuOperator(inti.SingleLayerKernel(inti.Helmholtz(k=1.0, dim=3)), q, q, dS, ctx=ctx)


def test_reference_error_messages(ctx):
    q = inti.ellipsoid_quadrature(2, 5)
    op = inti.Laplace(dim=3)
    with pytest.raises(inti.ArgumentError, match="Unknown compression.method"):
        inti.single_double_layer(op=op, target=q, source=q, compression={"method": "fmm"}, ctx=ctx)
    with pytest.raises(inti.ArgumentError, match="Unknown correction.method"):
        inti.single_double_layer(op=op, target=q, source=q, correction={"method": "foo"}, ctx=ctx)
    t = inti.points(q.coords * 2)
    with pytest.raises(inti.ArgumentError, match="missing target_location"):
        inti.single_double_layer(op=op, target=t, source=q, correction={"method": "dim"}, ctx=ctx)


def test_null_handles_through_abi(ctx):
    lib = L.load()
    assert lib.inti_op_apply(None, None, 0, None, 0, 1, None, None, 0) == L.E_ARG
    assert lib.inti_gmres(ctx.handle, 0, None, None, None, None, None, 1e-8, 10, 10, 0, 0, None, None) == L.E_ARG
    assert b"operator" in lib.inti_last_error(ctx.handle)
