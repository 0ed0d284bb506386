"""Symmetric pair kernel of square operators (target === source): each
unordered pair is evaluated once for both products.  Checked against the
one-sided kernel (a context with the symmetric form off) and the oracle, on
surfaces of many node blocks with a ragged last block, for the single layer,
double layer, combined field, adjoint double layer and hypersingular kernel,
Laplace (3D and 2D) and Helmholtz, FP64 and FP32C, with the DIM correction,
alpha/beta and repeated applies."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, relerr

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def one_sided():
    c = inti.Context(0)
    c.set_symmetric(False)
    c.set_single_launch(False)  # the tiled one-sided kernel at every size
    return c


@pytest.fixture(scope="module")
def tiled():
    """The symmetric kernel at every size (small FP64 operators otherwise
    take the single-launch form)."""
    c = inti.Context(0)
    c.set_single_launch(False)
    return c


def _op(pde):
    return inti.Laplace(dim=3) if pde == O.LAPLACE else inti.Helmholtz(k=6.0, dim=3)


KERNELS = {"SL": (inti.SingleLayerKernel, O.SL), "DL": (inti.DoubleLayerKernel, O.DL),
           "ADL": (inti.AdjointDoubleLayerKernel, O.ADL), "HS": (inti.HyperSingularKernel, O.HS)}


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
@pytest.mark.parametrize("kname", ["SL", "DL", "ADL", "HS"])
@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32c", 5e-5)])
def test_symmetric_matches_one_sided_and_oracle(ctx, one_sided, pde, kname, prec, tol):
    q = inti.ellipsoid_quadrature(9, 5)  # 4,374 nodes: 9 blocks of 512, the last ragged
    K, okind = KERNELS[kname]
    k = 0.0 if pde == O.LAPLACE else 6.0
    A = inti.GpuOperator(K(_op(pde)), q, q, None, prec, ctx)
    B = inti.GpuOperator(K(_op(pde)), q, q, None, prec, one_sided)
    assert A.tuning["symmetric"] and not B.tuning["symmetric"]
    x = density(len(q), pde == O.HELMHOLTZ, 3)
    ya, yb = A @ x, B @ x
    ref = oracle_apply(pde, okind, k, q, q, x)
    assert relerr(ya, ref) < tol and relerr(yb, ref) < tol
    if prec == "fp64":
        assert relerr(ya, yb) < 1e-13
    assert np.array_equal(A @ x, ya)  # deterministic


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
def test_symmetric_combined_field_with_correction(ctx, one_sided, pde):
    q = inti.ellipsoid_quadrature(8, 5)  # 3,456 nodes
    op = _op(pde)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    cS = -6.0j if pde == O.HELMHOLTZ else 0.7
    CF = inti.CombinedFieldOperator(D, S, 1.0, cS)
    assert CF.tuning["symmetric"]
    cs = inti.CorrectionMatrix.from_csr(*S.correction.arrays(), S.shape, ctx=one_sided)
    cd = inti.CorrectionMatrix.from_csr(*D.correction.arrays(), D.shape, ctx=one_sided)
    S2 = inti.GpuOperator(S.kernel, q, q, cs, "fp64", one_sided)
    D2 = inti.GpuOperator(D.kernel, q, q, cd, "fp64", one_sided)
    cplx = pde == O.HELMHOLTZ
    x = density(len(q), cplx, 4)
    y0 = density(len(q), cplx, 5)
    alpha, beta = (0.5 + 0.5j, -1.0 + 0.25j) if cplx else (0.5, -1.0)
    got = CF.mul(y0.copy(), x, alpha=alpha, beta=beta)
    want = alpha * (D2 @ x + cS * (S2 @ x)) + beta * y0
    assert relerr(got, want) < 1e-12


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
def test_symmetric_adjoint_double_layer_hypersingular_with_correction(ctx, one_sided, pde):
    """adj_double_layer_hypersingular on the surface (DIM correction): the
    symmetric operators against one-sided ones carrying the same corrections,
    with alpha/beta."""
    q = inti.ellipsoid_quadrature(8, 5)
    A, H = inti.adj_double_layer_hypersingular(op=_op(pde), target=q, source=q, correction={"method": "dim"},
                                              ctx=ctx)
    assert A.tuning["symmetric"] and H.tuning["symmetric"]
    cplx = pde == O.HELMHOLTZ
    x, y0 = density(len(q), cplx, 7), density(len(q), cplx, 8)
    alpha, beta = (0.25 - 1.0j, 0.5 + 0.5j) if cplx else (-0.75, 1.5)
    for P in (A, H):
        c = inti.CorrectionMatrix.from_csr(*P.correction.arrays(), P.shape, ctx=one_sided)
        P2 = inti.GpuOperator(P.kernel, q, q, c, "fp64", one_sided)
        assert not P2.tuning["symmetric"]
        got = P.mul(y0.copy(), x, alpha=alpha, beta=beta)
        want = alpha * (P2 @ x) + beta * y0
        assert relerr(got, want) < 1e-12


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
@pytest.mark.parametrize("kname", ["SL", "DL", "ADL", "HS"])
def test_symmetric_transpose_matches_one_sided(ctx, one_sided, pde, kname):
    """A^T of a square operator runs the symmetric product of the swapped
    kernel (DL <-> ADL) with unit weights; against the one-sided transpose
    (itself checked against the oracle's dense transpose) and, on sampled
    columns, against the oracle's rows of the swapped kernel."""
    q = inti.ellipsoid_quadrature(9, 5)
    K, okind = KERNELS[kname]
    A = inti.GpuOperator(K(_op(pde)), q, q, None, "fp64", ctx)
    B = inti.GpuOperator(K(_op(pde)), q, q, None, "fp64", one_sided)
    cplx = pde == O.HELMHOLTZ
    g = density(len(q), cplx, 9)
    ya = A.rmatvec(g)
    assert relerr(ya, B.rmatvec(g)) < 1e-13
    swapped = {O.DL: O.ADL, O.ADL: O.DL}.get(okind, okind)
    k = 0.0 if pde == O.LAPLACE else 6.0
    rows = np.arange(0, len(q), 97)
    ref = O.apply(pde, swapped, k, q.coords, q.normals, q.coords, q.normals, np.ones(len(q)), g, rows=rows)
    assert relerr(ya[rows], q.weights[rows] * ref) < 1e-12


def test_symmetric_gmres_matches_one_sided(ctx, one_sided):
    """The solver's fused combined field and its FP32C twin on the symmetric
    kernel give the same solution as on the one-sided one."""
    q = inti.ellipsoid_quadrature(8, 5)
    op = inti.Laplace(dim=3)
    b = density(len(q), False, 6)
    xs = []
    for c in (ctx, one_sided):
        S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=c)
        for mode in ("fp64", "mixed"):
            x, st = inti.gmres(0.5 * inti.I + D + S, b, rtol=1e-10, restart=50, maxiter=200, mode=mode)
            assert st["converged"] == 1, st
            xs.append(x)
    for x in xs[1:]:
        assert relerr(x, xs[0]) < 1e-8


@pytest.mark.parametrize("n", [1, 7, 511, 512, 513, 1025])
@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
def test_symmetric_edge_sizes(tiled, n, pde):
    """Node counts around the block size (512 or 256 nodes): a single node,
    a partial block, exact blocks and one node past them; points with
    arbitrary normals and weights (no element structure needed)."""
    r = np.random.default_rng(n)
    X = r.standard_normal((n, 3))
    N = r.standard_normal((n, 3))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    W = r.uniform(0.5, 1.5, n)
    q = inti.Quadrature(X, N, W, 0)
    cplx = pde == O.HELMHOLTZ
    k = 0.0 if pde == O.LAPLACE else 3.0
    x = density(n, cplx, 2)
    op = inti.Laplace(dim=3) if pde == O.LAPLACE else inti.Helmholtz(k=3.0, dim=3)
    for K, okind in KERNELS.values():
        A = inti.GpuOperator(K(op), q, q, None, "fp64", tiled)
        assert A.tuning["symmetric"] and not A.tuning["single_launch"]
        ref = oracle_apply(pde, okind, k, q, q, x)
        got = A @ x
        if n == 1:
            assert np.all(got == 0)  # the self pair is excluded
        else:
            assert relerr(got, ref) < 1e-12


# FP32C against the FP64 oracle on the 4,500-node kite: on a curve r.n is
# O(d^2) between neighbouring nodes and cancels in FP32 coordinates, so even
# exact sums of the FP32 pair values (a numpy restatement: FP32 coordinates,
# products and quotients, FP64 sums) are off by 9.6e-4 (DL), 6.9e-4 (ADL),
# 1.4e-4 (HS) and 2.9e-7 (SL); the bounds are about twice those floors.
FP32_2D_TOL = {"SL": 5e-5, "DL": 2e-3, "ADL": 2e-3, "HS": 5e-4}


@pytest.mark.parametrize("kname", ["SL", "DL", "ADL", "HS"])
@pytest.mark.parametrize("prec", ["fp64", "fp32c"])
def test_symmetric_2d_laplace(ctx, one_sided, kname, prec):
    """2D Laplace kernels on the symmetric form (log(d^2) once per unordered
    pair for the single layer): against the one-sided kernel and the oracle,
    and the transposes of the two forms against each other."""
    q = inti.kite_quadrature(900, 9)  # 4,500 nodes: 9 blocks of 512, the last ragged
    K, okind = KERNELS[kname]
    A = inti.GpuOperator(K(inti.Laplace(dim=2)), q, q, None, prec, ctx)
    B = inti.GpuOperator(K(inti.Laplace(dim=2)), q, q, None, prec, one_sided)
    assert A.tuning["symmetric"] and not B.tuning["symmetric"]
    x = density(len(q), False, 21)
    ya, yb = A @ x, B @ x
    ref = oracle_apply(O.LAPLACE, okind, 0.0, q, q, x)
    tol = 1e-12 if prec == "fp64" else FP32_2D_TOL[kname]
    assert relerr(ya, ref) < tol and relerr(yb, ref) < tol
    if prec == "fp64":
        assert relerr(ya, yb) < 1e-13
        assert relerr(A.rmatvec(x), B.rmatvec(x)) < 1e-13
    else:  # the same FP32 pair values (r_ts = -r_st exactly), summed in another order
        assert relerr(ya, yb) < 1e-4
    assert np.array_equal(A @ x, ya)


@pytest.mark.parametrize("n", [1, 7, 257, 513])
def test_symmetric_2d_edge_sizes(tiled, n):
    r = np.random.default_rng(100 + n)
    X = r.standard_normal((n, 2))
    N = r.standard_normal((n, 2))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    q = inti.Quadrature(X, N, r.uniform(0.5, 1.5, n), 0)
    x = density(n, False, 3)
    for K, okind in KERNELS.values():
        A = inti.GpuOperator(K(inti.Laplace(dim=2)), q, q, None, "fp64", tiled)
        assert A.tuning["symmetric"] and not A.tuning["single_launch"]
        got = A @ x
        if n == 1:
            assert np.all(got == 0)
        else:
            assert relerr(got, oracle_apply(O.LAPLACE, okind, 0.0, q, q, x)) < 1e-12


@pytest.mark.parametrize("n", [1, 7, 513, 1025])
def test_symmetric_fp32c_edge_sizes(ctx, n):
    """The paired-FP32 form (FP32C Laplace SL, DL and combined field) at node
    counts around its 256/512-node blocks: one pair of targets per thread
    straddling the end of the nodes, padded records, a single node."""
    r = np.random.default_rng(200 + n)
    X = r.standard_normal((n, 3))
    N = r.standard_normal((n, 3))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    q = inti.Quadrature(X, N, r.uniform(0.5, 1.5, n), 0)
    x = density(n, False, 4)
    op = inti.Laplace(dim=3)
    S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp32c", ctx)
    D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, None, "fp32c", ctx)
    CF = inti.CombinedFieldOperator(D, S, 0.5, 2.0)
    assert S.tuning["symmetric"] and D.tuning["symmetric"] and CF.tuning["symmetric"]
    rs = oracle_apply(O.LAPLACE, O.SL, 0.0, q, q, x)
    rd = oracle_apply(O.LAPLACE, O.DL, 0.0, q, q, x)
    for A, ref in ((S, rs), (D, rd), (CF, 0.5 * rd + 2.0 * rs)):
        got = A @ x
        if n == 1:
            assert np.all(got == 0)
        else:
            assert relerr(got, ref) < 5e-5


@pytest.mark.parametrize("n", [1, 7, 257, 513, 1025])
def test_symmetric_fp32c_helmholtz_edge_sizes(ctx, n):
    """The FP32C Helmholtz symmetric kernel (SL, DL and the combined field
    with complex coefficients) at node counts around its 256-source tiles
    and 256/512-node blocks: padded records, targets straddling the end of
    the nodes, a single node; against the oracle."""
    r = np.random.default_rng(300 + n)
    X = r.standard_normal((n, 3))
    N = r.standard_normal((n, 3))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    q = inti.Quadrature(X, N, r.uniform(0.5, 1.5, n), 0)
    x = density(n, True, 4)
    k = 4.0
    op = inti.Helmholtz(k=k, dim=3)
    S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp32c", ctx)
    D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, None, "fp32c", ctx)
    CF = inti.CombinedFieldOperator(D, S, 1.0, -1j * k)
    assert S.tuning["symmetric"] and D.tuning["symmetric"] and CF.tuning["symmetric"]
    rs = oracle_apply(O.HELMHOLTZ, O.SL, k, q, q, x)
    rd = oracle_apply(O.HELMHOLTZ, O.DL, k, q, q, x)
    for A, ref in ((S, rs), (D, rd), (CF, rd - 1j * k * rs)):
        got = A @ x
        if n == 1:
            assert np.all(got == 0)
        else:
            assert relerr(got, ref) < 5e-5
