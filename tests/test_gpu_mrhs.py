"""Multi-column applies of single operators (inti_op_apply with nrhs >= 8):
the FP64 MMA kernel evaluates each kernel value once for up to 64 columns,
for the single and double layer, the combined field, the adjoint double
layer and the hypersingular kernel.
Checked against the same operator applied one column at a time (itself
checked against the oracle), on-surface with the DIM correction and off the
surface, for 8 columns, and for 70 (two column groups, the second ragged),
with alpha/beta and padded leading dimensions on device pointers."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import relerr

pytestmark = pytest.mark.gpu


def _ops(kind, pde, on_surface, ctx):
    q = inti.ellipsoid_quadrature(5, 5)
    op = inti.Helmholtz(k=4.0, dim=3) if pde == "helmholtz" else inti.Laplace(dim=3)
    deriv = kind in ("ADL", "HS")
    if on_surface:
        S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"},
                                        derivative=deriv, ctx=ctx)
        tq = q
    else:
        r = np.random.default_rng(3)
        d = r.standard_normal((700, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        nt = r.standard_normal((700, 3))
        nt /= np.linalg.norm(nt, axis=1, keepdims=True)
        tq = inti.Quadrature(1.6 * d, nt, np.ones(700), 0)  # off-surface targets with normals
        K1, K2 = ((inti.AdjointDoubleLayerKernel, inti.HyperSingularKernel) if deriv
                  else (inti.SingleLayerKernel, inti.DoubleLayerKernel))
        S = inti.GpuOperator(K1(op), tq, q, None, "fp64", ctx)
        D = inti.GpuOperator(K2(op), tq, q, None, "fp64", ctx)
    if kind in ("SL", "ADL"):
        return S, q, tq
    if kind in ("DL", "HS"):
        return D, q, tq
    cS = -4.0j if pde == "helmholtz" else 0.7
    return inti.CombinedFieldOperator(D, S, 1.0, cS), q, tq


def _cols(A, X):
    return np.stack([A @ X[:, c] for c in range(X.shape[1])], axis=1)


@pytest.mark.parametrize("kind", ["SL", "DL", "CF", "ADL", "HS"])
@pytest.mark.parametrize("pde", ["helmholtz", "laplace"])
@pytest.mark.parametrize("on_surface", [True, False])
@pytest.mark.parametrize("nrhs", [8, 70])
def test_multi_column_apply_matches_columns(ctx, kind, pde, on_surface, nrhs):
    A, q, tq = _ops(kind, pde, on_surface, ctx)
    r = np.random.default_rng(nrhs)
    X = r.standard_normal((len(q), nrhs))
    if pde == "helmholtz":
        X = X + 1j * r.standard_normal((len(q), nrhs))
    before = ctx.launch_count
    Y = A @ X
    launches = ctx.launch_count - before
    assert launches <= 2  # one MMA launch (+ the correction SpMV), not one product per column
    assert relerr(Y, _cols(A, X)) < 1e-12
    if kind in ("SL", "ADL", "HS") and not on_surface:  # and against the oracle directly
        pde_o = O.HELMHOLTZ if pde == "helmholtz" else O.LAPLACE
        k = 4.0 if pde == "helmholtz" else 0.0
        okind = {"SL": O.SL, "ADL": O.ADL, "HS": O.HS}[kind]
        for c in (0, nrhs - 1):
            ref = O.apply(pde_o, okind, k, tq.coords, tq.normals, q.coords, q.normals, q.weights, X[:, c])
            assert relerr(Y[:, c], ref) < 1e-12


@pytest.mark.parametrize("pde", ["helmholtz", "laplace"])
def test_multi_column_device_alpha_beta_leading_dims(ctx, pde):
    import torch

    A, q, tq = _ops("CF", pde, True, ctx)
    m, n = A.shape
    nrhs, ldx, ldy = 20, n + 5, m + 3
    cplx = pde == "helmholtz"
    r = np.random.default_rng(11)
    X = r.standard_normal((n, nrhs)) + (1j * r.standard_normal((n, nrhs)) if cplx else 0)
    Y0 = r.standard_normal((m, nrhs)) + (1j * r.standard_normal((m, nrhs)) if cplx else 0)
    dt = np.complex128 if cplx else np.float64
    Xp = np.zeros((ldx, nrhs), dt, order="F")
    Yp = np.zeros((ldy, nrhs), dt, order="F")
    Xp[:n] = X
    Yp[:m] = Y0
    dev = torch.device("cuda:0")
    xs = torch.from_numpy(np.ascontiguousarray(Xp.T).view(np.float64).copy()).to(dev)
    ys = torch.from_numpy(np.ascontiguousarray(Yp.T).view(np.float64).copy()).to(dev)
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, -1.5)
    torch.cuda.synchronize()
    A.apply_device(xs.data_ptr(), ys.data_ptr(), nrhs, alpha, beta, ldx=ldx, ldy=ldy)
    ctx.synchronize()
    got = ys.cpu().numpy().view(dt).T
    want = alpha * _cols(A, X) + beta * Y0
    assert relerr(got[:m], want) < 1e-12
    assert np.array_equal(got[m:], Yp[m:])  # padding rows untouched
