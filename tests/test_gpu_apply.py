"""GPU pair product versus the oracle, through the C ABI (ctypes).

FP64: relative 2-norm error <= 1e-12 (the reference's matrix-free vs
entry-wise test allows 1e-7, test/fmm3d_test.jl:42).  FP32C: <= 2e-5 for
Laplace, <= 5e-5 for Helmholtz (FP32 kernel evaluation with compensated sums).
"""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, relerr, small_surfaces

pytestmark = pytest.mark.gpu

SURF = small_surfaces()
KINDS = [("SL", inti.SingleLayerKernel, O.SL), ("DL", inti.DoubleLayerKernel, O.DL),
         ("ADL", inti.AdjointDoubleLayerKernel, O.ADL), ("HS", inti.HyperSingularKernel, O.HS)]


def ops_for(q):
    if q.dim == 2:
        return [(inti.Laplace(dim=2), O.LAPLACE, 0.0)]
    return [(inti.Laplace(dim=3), O.LAPLACE, 0.0), (inti.Helmholtz(k=4.0, dim=3), O.HELMHOLTZ, 4.0)]


CASES = [(s, ki) for s in SURF for ki in range(4)]


@pytest.mark.parametrize("surf,ki", CASES)
def test_fp64_matches_oracle(ctx, surf, ki):
    q = SURF[surf]
    name, Kc, kind = KINDS[ki]
    for op, pde, k in ops_for(q):
        A = inti.IntegralOperator(Kc(op), q, q, ctx=ctx)
        x = density(len(q), pde == O.HELMHOLTZ, seed=ki + 3)
        y = A @ x
        ref = oracle_apply(pde, kind, k, q, q, x)
        assert relerr(y, ref) < 1e-12, (surf, name, op)


@pytest.mark.parametrize("surf,ki", CASES)
def test_fp32c_matches_oracle(ctx, surf, ki):
    q = SURF[surf]
    name, Kc, kind = KINDS[ki]
    for op, pde, k in ops_for(q):
        A = inti.IntegralOperator(Kc(op), q, q, precision="fp32c", ctx=ctx)
        x = density(len(q), pde == O.HELMHOLTZ, seed=ki + 7)
        ref = oracle_apply(pde, kind, k, q, q, x)
        tol = 5e-5 if pde == O.HELMHOLTZ else 2e-5
        assert relerr(A @ x, ref) < tol, (surf, name, op)


def test_off_surface_targets_and_potential(ctx):
    q = SURF["ellipsoid"]
    tgt = inti.points(3.0 * SURF["ellipsoid"].coords[::5])
    sigma = density(len(q), False, 11)
    Spot, Dpot = inti.single_double_layer_potential(op=inti.Laplace(dim=3), source=q, ctx=ctx)
    u = Dpot[sigma](tgt.coords)
    ref = O.apply(O.LAPLACE, O.DL, 0.0, tgt.coords, None, q.coords, q.normals, q.weights, sigma)
    assert relerr(u, ref) < 1e-12
    # exterior points: the double layer of a constant vanishes (Gauss's law),
    # up to the quadrature error of the coarse mesh
    assert np.max(np.abs(Dpot[np.ones(len(q))](tgt.coords))) < 1e-3


def test_alpha_beta_and_multi_rhs(ctx):
    q = SURF["p2sphere"]
    op = inti.Helmholtz(k=3.0, dim=3)
    A = inti.IntegralOperator(inti.DoubleLayerKernel(op), q, ctx=ctx)
    X = np.stack([density(len(q), True, s) for s in range(3)], 1)
    Y0 = np.stack([density(len(q), True, 10 + s) for s in range(3)], 1)
    alpha, beta = 0.3 - 1.1j, -0.7 + 0.2j
    Y = Y0.copy()
    A.mul(Y, X, alpha, beta)
    for c in range(3):
        ref = alpha * oracle_apply(O.HELMHOLTZ, O.DL, 3.0, q, q, X[:, c]) + beta * Y0[:, c]
        assert relerr(Y[:, c], ref) < 1e-12
    # beta = 0 must not read y (NaN in y is ignored, BLAS semantics)
    Yn = np.full_like(Y0, np.nan)
    A.mul(Yn, X, 1.0, 0.0)
    assert np.isfinite(Yn).all()


def test_dense_assembly_matches_oracle(ctx):
    q = SURF["kite"]
    for Kc, kind in ((inti.SingleLayerKernel, O.SL), (inti.HyperSingularKernel, O.HS)):
        A = inti.assemble_matrix(inti.IntegralOperator(Kc(inti.Laplace(dim=2)), q, ctx=ctx))
        ref = O.assemble(O.LAPLACE, kind, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights)
        assert relerr(A, ref) < 1e-13


def test_transpose_apply(ctx):
    q = SURF["ellipsoid"]
    for op, pde, k in ops_for(q):
        A = inti.IntegralOperator(inti.DoubleLayerKernel(op), q, ctx=ctx)
        dense = O.assemble(pde, O.DL, k, q.coords, q.normals, q.coords, q.normals, q.weights)
        g = density(len(q), pde == O.HELMHOLTZ, 21)
        assert relerr(A.rmatvec(g), dense.T @ g) < 1e-12


@pytest.mark.parametrize("surf,ki", CASES)
def test_transpose_apply_every_kernel(ctx, surf, ki):
    """A^T runs the forward pair kernel with targets and sources swapped
    (DL <-> ADL, SL and HS unchanged) and the weights applied per row; checked
    against the transpose of the oracle's dense matrix, in FP64 and FP32C."""
    q = SURF[surf]
    name, Kc, kind = KINDS[ki]
    for op, pde, k in ops_for(q):
        dense = O.assemble(pde, kind, k, q.coords, q.normals, q.coords, q.normals, q.weights)
        g = density(len(q), pde == O.HELMHOLTZ, 31 + ki)
        for prec, tol in (("fp64", 1e-12), ("fp32c", 5e-5)):
            A = inti.GpuOperator(Kc(op), q, q, None, prec, ctx)
            assert relerr(A.rmatvec(g), dense.T @ g) < tol, (surf, name, op, prec)


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
def test_transpose_apply_off_surface_and_corrected(ctx, pde):
    """Rectangular A (targets off the surface) and A + δ with the DIM
    correction, with alpha/beta, through the transposed apply."""
    q = SURF["ellipsoid"]
    op = inti.Laplace(dim=3) if pde == O.LAPLACE else inti.Helmholtz(k=4.0, dim=3)
    k = 0.0 if pde == O.LAPLACE else 4.0
    cplx = pde == O.HELMHOLTZ
    r = np.random.default_rng(5)
    T = 1.8 * r.standard_normal((150, 3))
    D = inti.GpuOperator(inti.DoubleLayerKernel(op), inti.points(T), q, None, "fp64", ctx)
    dense = O.assemble(pde, O.DL, k, T, None, q.coords, q.normals, q.weights)
    g = density(len(T), cplx, 7)
    assert relerr(D.rmatvec(g), dense.T @ g) < 1e-12
    S, _ = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    import scipy.sparse as sp

    rp, col, val = S.correction.arrays()
    full = O.assemble(pde, O.SL, k, q.coords, q.normals, q.coords, q.normals, q.weights) + \
        sp.csr_matrix((val, col, rp), shape=S.shape).toarray()
    g = density(len(q), cplx, 8)
    y0 = density(len(q), cplx, 9)
    alpha, beta = (0.5 - 1.0j, 2.0 + 0.5j) if cplx else (0.5, 2.0)
    got = S._apply(g, y=y0.copy(), alpha=alpha, beta=beta, transpose=True)
    assert relerr(got, alpha * (full.T @ g) + beta * y0) < 1e-12


@pytest.mark.parametrize("pde", [O.LAPLACE, O.HELMHOLTZ])
def test_transpose_of_rectangular_correction(ctx, pde):
    """Off-surface targets with their DIM correction (a rectangular CSR, built
    and transposed on the device) through the transposed apply."""
    import scipy.sparse as sp

    q = SURF["ellipsoid"]
    tgt = inti.points(0.9 * q.coords[::3])
    op = inti.Laplace(dim=3) if pde == O.LAPLACE else inti.Helmholtz(k=4.0, dim=3)
    k = 0.0 if pde == O.LAPLACE else 4.0
    cplx = pde == O.HELMHOLTZ
    S, D = inti.single_double_layer(op=op, target=tgt, source=q, ctx=ctx,
                                    correction={"method": "dim", "target_location": "inside"})
    for A, kind, tn in ((D, O.DL, None), (S, O.SL, None)):
        rp, col, val = A.correction.arrays()
        full = O.assemble(pde, kind, k, tgt.coords, tn, q.coords, q.normals, q.weights) + \
            sp.csr_matrix((val, col, rp), shape=A.shape).toarray()
        g = density(len(tgt), cplx, 3)
        assert relerr(A.rmatvec(g), full.T @ g) < 1e-12
        assert np.array_equal(A.rmatvec(g), A.rmatvec(g))  # deterministic


def test_launch_counter_advances(ctx):
    q = SURF["kite"]
    A = inti.IntegralOperator(inti.DoubleLayerKernel(inti.Laplace(dim=2)), q, ctx=ctx)
    assert A.tuning["single_launch"]
    before = ctx.launch_count
    A @ np.ones(len(q))
    assert ctx.launch_count - before == 1  # one kernel: records, pair sums, epilogue
    tiled = inti.Context(0)
    tiled.set_single_launch(False)
    B = inti.IntegralOperator(inti.DoubleLayerKernel(inti.Laplace(dim=2)), q, ctx=tiled)
    before = tiled.launch_count
    B @ np.ones(len(q))
    assert tiled.launch_count - before == 3  # pack, pair, epilogue


def test_fast_special_functions_accuracy(ctx):
    """The pair loops' rsqrt, x^{-3/2}, reciprocal and e^{iθ} against extended precision."""
    r = ctx.selftest_math()
    assert r["rsqrt_f64_maxrel"] < 4e-16, r
    assert r["rsqrt_cube_f64_maxrel"] < 8e-16, r
    assert r["rcp_f64_maxrel"] < 3e-16, r
    assert r["expi_f64_maxabs_25"] < 8e-16, r
    assert r["expi_f64_maxabs_1000"] < 2e-13, r
    assert r["expi_f32_maxabs_25"] < 4e-6, r


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32c", 5e-5)])
def test_combined_field_operator(ctx, prec, tol):
    """c_D·(D + δD) + c_S·(S + δS) in one pass equals the two products."""
    q = SURF["ellipsoid"]
    for op, pde, k, cD, cS in ((inti.Laplace(dim=3), O.LAPLACE, 0.0, 1.0, 0.7),
                              (inti.Helmholtz(k=3.0, dim=3), O.HELMHOLTZ, 3.0, 1.0, -3.0j)):
        S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
        C = inti.CombinedFieldOperator(D, S, cD, cS, precision=prec)
        x = density(len(q), pde == O.HELMHOLTZ, 31)
        dS, dD = S.correction.arrays(), D.correction.arrays()
        ref = cD * (oracle_apply(pde, O.DL, k, q, q, x) + O.csr_apply(*dD, x)) + \
            cS * (oracle_apply(pde, O.SL, k, q, q, x) + O.csr_apply(*dS, x))
        assert relerr(C @ x, ref) < tol, (op, prec)


def test_released_device_blocks_are_reused(ctx):
    """Operators created and destroyed again and again reuse the device
    memory released by the previous round (the memory pool for small blocks,
    cudaMalloc/cudaFree for large ones): device memory in use stays flat
    after the first round."""
    import gc

    import torch

    q = inti.ellipsoid_quadrature(12, 5)  # 7,776 nodes
    op = inti.Helmholtz(k=3.0, dim=3)
    x = density(len(q), True, 3)
    used = []
    for _ in range(4):
        S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
        CF = inti.CombinedFieldOperator(D, S, 1.0, -3.0j)
        y = CF @ x
        del S, D, CF
        gc.collect()
        ctx.synchronize()
        free, total = torch.cuda.mem_get_info()
        used.append(total - free)
    assert max(used[1:]) - min(used[1:]) < (64 << 20), used
    assert np.all(np.isfinite(y))


def test_bounded_wait_timeout_is_reported_and_context_survives(ctx):
    """A device-side bounded wait that runs out (an mbarrier nothing arrives
    at) ends its kernel with INTI_E_TIMEOUT in the context's flag; the call
    reports it, and the context keeps working with the flag cleared."""
    import time

    from inti_b200 import _lib as L

    t0 = time.perf_counter()
    status = ctx.lib.inti_selftest_wait_timeout(ctx.handle)
    elapsed = time.perf_counter() - t0
    assert status == L.E_TIMEOUT
    assert b"bounded wait" in ctx.lib.inti_last_error(ctx.handle)
    assert elapsed < 30.0, elapsed
    print(f"bounded wait ran out after {elapsed:.3f} s")
    q = SURF["ellipsoid"]
    A = inti.GpuOperator(inti.SingleLayerKernel(inti.Laplace(dim=3)), q, q, None, "fp64", ctx)
    x = density(len(q), False, 4)
    assert relerr(A @ x, oracle_apply(O.LAPLACE, O.SL, 0.0, q, q, x)) < 1e-12
    ctx.synchronize()  # no stale timeout


@pytest.mark.parametrize("case", ["kite", "ellipsoid", "helmholtz"])
def test_pinned_host_vectors_match_pageable(ctx, case):
    """Host-pointer applies of small vectors in page-locked memory (read by a
    copy kernel, y written in place in host memory) give the same bits as
    pageable buffers (copied by the copy engines): products and transposes,
    beta = 0 and beta != 0."""
    import torch

    if case == "kite":
        q, op, cplx = inti.kite_quadrature(200, 9), inti.Laplace(dim=2), False  # single-launch form
    elif case == "ellipsoid":
        q, op, cplx = inti.ellipsoid_quadrature(8, 5), inti.Laplace(dim=3), False  # 3,456 nodes, tiled
    else:
        q, op, cplx = inti.p2_sphere_quadrature(8), inti.Helmholtz(k=3.0, dim=3), True  # 3,072 nodes
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    dt = torch.complex128 if cplx else torch.float64
    x = density(len(q), cplx, 41)
    y0 = density(len(q), cplx, 42)
    alpha, beta = (0.5 - 0.25j, 1.5 + 0.5j) if cplx else (0.5, 1.5)
    for A in (S, D):
        px = torch.from_numpy(x.copy()).pin_memory().numpy()
        for transpose in (False, True):
            for b in (0.0, beta):
                py = torch.from_numpy(y0.copy()).to(dt).pin_memory().numpy()
                got = A._apply(px, y=py, alpha=alpha, beta=b, transpose=transpose)
                want = A._apply(x.copy(), y=y0.copy(), alpha=alpha, beta=b, transpose=transpose)
                assert np.array_equal(got, want), (case, transpose, b)
