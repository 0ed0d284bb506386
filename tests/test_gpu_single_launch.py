"""Single-launch form of small FP64 operators (at most 2^20 target-source
pairs): one kernel per product, which builds the source records itself and
splits the sources over the CTAs of a cluster.  Checked against the oracle
and against the tiled kernels (a context with the form off) for every
kernel family in 2D and 3D, square and rectangular operators, one to eight
source slices per cluster and several staged tiles per slice, with the DIM
correction and alpha/beta, at node counts from one node to the 1,000-node
kite (the C1 configuration)."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, relerr

pytestmark = pytest.mark.gpu

KERNELS = {"SL": (inti.SingleLayerKernel, O.SL), "DL": (inti.DoubleLayerKernel, O.DL),
           "ADL": (inti.AdjointDoubleLayerKernel, O.ADL), "HS": (inti.HyperSingularKernel, O.HS)}


@pytest.fixture(scope="module")
def tiled():
    c = inti.Context(0)
    c.set_single_launch(False)
    return c


def _points(n, dim, seed):
    r = np.random.default_rng(seed)
    X = r.standard_normal((n, dim))
    N = r.standard_normal((n, dim))
    N /= np.linalg.norm(N, axis=1, keepdims=True)
    return inti.Quadrature(X, N, r.uniform(0.5, 1.5, n), 0)


@pytest.mark.parametrize("case", ["laplace2d", "laplace3d", "helmholtz3d"])
@pytest.mark.parametrize("n", [1, 7, 33, 300, 1024])
def test_single_launch_matches_oracle_and_tiled(ctx, tiled, case, n):
    dim = 2 if case == "laplace2d" else 3
    q = _points(n, dim, 40 + n)
    op = inti.Helmholtz(k=3.0, dim=3) if case == "helmholtz3d" else inti.Laplace(dim=dim)
    pde, k = (O.HELMHOLTZ, 3.0) if case == "helmholtz3d" else (O.LAPLACE, 0.0)
    x = density(n, pde == O.HELMHOLTZ, 5)
    for kname, (K, okind) in KERNELS.items():
        A = inti.GpuOperator(K(op), q, q, None, "fp64", ctx)
        B = inti.GpuOperator(K(op), q, q, None, "fp64", tiled)
        assert A.tuning["single_launch"] and not B.tuning["single_launch"]
        ya, yb = A @ x, B @ x
        if n == 1:
            assert np.all(ya == 0)  # the self pair is excluded
            continue
        assert relerr(ya, oracle_apply(pde, okind, k, q, q, x)) < 1e-12, kname
        assert relerr(ya, yb) < 1e-13, kname
        assert np.array_equal(A @ x, ya)  # deterministic


@pytest.mark.parametrize("case", ["laplace2d", "helmholtz3d"])
@pytest.mark.parametrize("m,n", [(40, 20000), (5, 3001), (96, 700), (2000, 500)])
def test_single_launch_few_targets_many_sources(ctx, tiled, case, m, n):
    """Few row blocks and many sources (eight slices per cluster, each slice
    several staged tiles with a ragged last tile), and many row blocks (two
    slices)."""
    dim = 2 if case == "laplace2d" else 3
    src, tgt = _points(n, dim, 7 + m), _points(m, dim, 9 + n)
    op = inti.Helmholtz(k=3.0, dim=3) if case == "helmholtz3d" else inti.Laplace(dim=dim)
    pde, k = (O.HELMHOLTZ, 3.0) if case == "helmholtz3d" else (O.LAPLACE, 0.0)
    x = density(n, pde == O.HELMHOLTZ, 6)
    for kname, (K, okind) in KERNELS.items():
        A = inti.GpuOperator(K(op), tgt, src, None, "fp64", ctx)
        B = inti.GpuOperator(K(op), tgt, src, None, "fp64", tiled)
        assert A.tuning["single_launch"]
        ya = A @ x
        assert relerr(ya, oracle_apply(pde, okind, k, tgt, src, x)) < 1e-12, kname
        assert relerr(ya, B @ x) < 1e-13, kname


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
def test_single_launch_rectangular_corrected_alpha_beta(ctx, tiled, pde):
    """Off-surface targets with their DIM correction, alpha/beta, and the
    combined field (c1 DL + c2 SL in one pass)."""
    q = inti.ellipsoid_quadrature(3, 5)  # 486 nodes
    tgt = inti.points(0.9 * q.coords[::3])  # inside, near the surface
    op = inti.Laplace(dim=3) if pde == O.LAPLACE else inti.Helmholtz(k=2.0, dim=3)
    k = 0.0 if pde == O.LAPLACE else 2.0
    cplx = pde == O.HELMHOLTZ
    S, D = inti.single_double_layer(op=op, target=tgt, source=q, ctx=ctx,
                                    correction={"method": "dim", "target_location": "inside"})
    assert D.tuning["single_launch"]
    x, y0 = density(len(q), cplx, 7), density(len(tgt), cplx, 8)
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, 1.5)
    rp, col, val = D.correction.arrays()
    ref = alpha * (O.apply(pde, O.DL, k, tgt.coords, None, q.coords, q.normals, q.weights, x)
                   + O.csr_apply(rp, col, val, x)) + beta * y0
    assert relerr(D.mul(y0.copy(), x, alpha=alpha, beta=beta), ref) < 1e-12
    ct = inti.CorrectionMatrix.from_csr(rp, col, val, D.shape, ctx=tiled)
    Dt = inti.GpuOperator(inti.DoubleLayerKernel(op), tgt, q, ct, "fp64", tiled)
    assert not Dt.tuning["single_launch"]
    assert relerr(Dt.mul(y0.copy(), x, alpha=alpha, beta=beta), ref) < 1e-12
    # combined field on the surface, with both corrections merged
    S2, D2 = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    cS = -2.0j if cplx else 0.7
    CF = inti.CombinedFieldOperator(D2, S2, 1.0, cS)
    assert CF.tuning["single_launch"]
    want = (oracle_apply(pde, O.DL, k, q, q, x) + O.csr_apply(*D2.correction.arrays(), x)
            + cS * (oracle_apply(pde, O.SL, k, q, q, x) + O.csr_apply(*S2.correction.arrays(), x)))
    assert relerr(CF @ x, want) < 1e-12


def test_c1_kite_single_launch(ctx):
    """The C1 operator (kite, N = 1,000, Laplace DL with DIM): one pack and
    one fused launch per product, equal to the oracle with the same
    correction."""
    q = inti.kite_quadrature()
    S, D = inti.single_double_layer(op=inti.Laplace(dim=2), target=q, source=q, correction={"method": "dim"},
                                    ctx=ctx)
    assert D.tuning["single_launch"] and D.tuning["symmetric"]
    sigma = density(len(q), False, 1)
    before = ctx.launch_count
    y = D @ sigma
    assert ctx.launch_count - before == 1
    ref = oracle_apply(O.LAPLACE, O.DL, 0.0, q, q, sigma) + O.csr_apply(*D.correction.arrays(), sigma)
    assert relerr(y, ref) < 1e-12


def test_single_launch_eligibility(ctx):
    """FP64 only, at most 2^20 pairs and 65,536 sources."""
    lap = inti.Laplace(dim=3)
    small, many = _points(8, 3, 1), _points(70000, 3, 2)
    assert inti.GpuOperator(inti.SingleLayerKernel(lap), small, _points(1024, 3, 3), None, "fp64", ctx).tuning[
        "single_launch"]
    assert not inti.GpuOperator(inti.SingleLayerKernel(lap), small, many, None, "fp64", ctx).tuning["single_launch"]
    q = _points(1025, 3, 4)  # 1,050,625 pairs
    assert not inti.GpuOperator(inti.SingleLayerKernel(lap), q, q, None, "fp64", ctx).tuning["single_launch"]
    q = _points(300, 3, 5)
    assert not inti.GpuOperator(inti.SingleLayerKernel(lap), q, q, None, "fp32c", ctx).tuning["single_launch"]


@pytest.mark.parametrize("case", ["laplace2d", "laplace3d", "helmholtz3d"])
def test_single_launch_derivative_kernels_with_correction(ctx, tiled, case):
    """ADL and HS with their derivative DIM corrections, complex alpha/beta on
    the Helmholtz kernels: the single-launch form against the tiled kernels
    with the same correction arrays."""
    if case == "laplace2d":
        q, op, cplx = inti.kite_quadrature(120, 9), inti.Laplace(dim=2), False  # 600 nodes
    elif case == "laplace3d":
        q, op, cplx = inti.ellipsoid_quadrature(3, 5), inti.Laplace(dim=3), False  # 486 nodes
    else:
        q, op, cplx = inti.p2_sphere_quadrature(4), inti.Helmholtz(k=3.0, dim=3), True  # 768 nodes
    K, H = inti.adj_double_layer_hypersingular(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    x, y0 = density(len(q), cplx, 21), density(len(q), cplx, 22)
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, 1.5)
    for A, K_ in ((K, inti.AdjointDoubleLayerKernel), (H, inti.HyperSingularKernel)):
        assert A.tuning["single_launch"]
        rp, col, val = A.correction.arrays()
        ct = inti.CorrectionMatrix.from_csr(rp, col, val, A.shape, ctx=tiled)
        B = inti.GpuOperator(K_(op), q, q, ct, "fp64", tiled)
        got = A.mul(y0.copy(), x, alpha=alpha, beta=beta)
        assert relerr(got, B.mul(y0.copy(), x, alpha=alpha, beta=beta)) < 1e-12, K_
        assert np.array_equal(got, A.mul(y0.copy(), x, alpha=alpha, beta=beta))


@pytest.mark.parametrize("case", ["laplace2d", "laplace3d", "helmholtz3d"])
def test_single_launch_transpose(ctx, tiled, case):
    """Transposed products of small square operators (every kernel, with the
    DIM correction, complex alpha/beta) in the single-launch form: the
    transposed kernel with unit source weights and each row scaled by its
    weight, against the tiled kernels and the dense oracle transpose."""
    import scipy.sparse as sp

    if case == "laplace2d":
        q, op, cplx, pde, k = inti.kite_quadrature(120, 9), inti.Laplace(dim=2), False, O.LAPLACE, 0.0
    elif case == "laplace3d":
        q, op, cplx, pde, k = inti.ellipsoid_quadrature(3, 5), inti.Laplace(dim=3), False, O.LAPLACE, 0.0
    else:
        q, op, cplx, pde, k = inti.p2_sphere_quadrature(4), inti.Helmholtz(k=3.0, dim=3), True, O.HELMHOLTZ, 3.0
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    K, H = inti.adj_double_layer_hypersingular(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    g, y0 = density(len(q), cplx, 31), density(len(q), cplx, 32)
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, 1.5)
    for A, kind, K_ in ((S, O.SL, inti.SingleLayerKernel), (D, O.DL, inti.DoubleLayerKernel),
                        (K, O.ADL, inti.AdjointDoubleLayerKernel), (H, O.HS, inti.HyperSingularKernel)):
        assert A.tuning["single_launch"]
        rp, col, val = A.correction.arrays()
        dense = O.assemble(pde, kind, k, q.coords, q.normals, q.coords, q.normals, q.weights) + \
            sp.csr_matrix((val, col, rp), shape=A.shape).toarray()
        got = A._apply(g, y=y0.copy(), alpha=alpha, beta=beta, transpose=True)
        assert relerr(got, alpha * (dense.T @ g) + beta * y0) < 1e-12, kind
        B = inti.GpuOperator(K_(op), q, q, inti.CorrectionMatrix.from_csr(rp, col, val, A.shape, ctx=tiled),
                             "fp64", tiled)
        assert relerr(got, B._apply(g, y=y0.copy(), alpha=alpha, beta=beta, transpose=True)) < 1e-12, kind
        before = ctx.launch_count
        A.rmatvec(g)
        assert ctx.launch_count - before == 1
