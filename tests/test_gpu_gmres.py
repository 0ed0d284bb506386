"""GPU GMRES (FP64 and FP32-inner / FP64-outer refinement) against the
oracle's FP64 GMRES and dense solves; the residual is always measured in
FP64 (docs/src/examples/poisson.jl:166-168 solves -I/2 + D this way)."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, relerr

pytestmark = pytest.mark.gpu


def laplace_problem(ctx, n=4):
    q = inti.ellipsoid_quadrature(n, 5)
    op = inti.Laplace(dim=3)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    return q, S, D


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_gmres_laplace_matches_oracle(ctx, mode):
    """Interior Dirichlet problem (-I/2 + D) σ = b, docs/src/examples/poisson.jl:160-168."""
    q, S, D = laplace_problem(ctx)
    L = D - 0.5 * inti.I
    b = density(len(q), False, 3)
    x, st = inti.gmres(L, b, rtol=1e-10, restart=50, maxiter=300, mode=mode, history=True)
    assert st["converged"] == 1 and st["relres"] <= 1e-10, st
    dD = D.correction.arrays()  # same operator data on both sides
    xo, sto = O.gmres(O.LAPLACE, 0.0, q.coords, q.normals, q.weights, -0.5, [(O.DL, 1.0, dD)], b,
                      rtol=1e-13, restart=50, maxiter=300)
    # the FP64 residual of the GPU solution, recomputed by the oracle
    r = b - (-0.5 * x + oracle_apply(O.LAPLACE, O.DL, 0.0, q, q, x) + O.csr_apply(*dD, x))
    assert np.linalg.norm(r) / np.linalg.norm(b) < 2e-10
    assert relerr(x, xo) < 1e-9
    if mode == "mixed":
        assert st["fp32_applies"] > 0 and st["fp64_applies"] >= 2


def test_gmres_helmholtz_cfie(ctx):
    """I/2 + D - i k S (docs/src/examples/helmholtz_scattering.jl:485-495)."""
    q = inti.p2_sphere_quadrature(3)
    k = 2.0
    op = inti.Helmholtz(k=k, dim=3)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    L = 0.5 * inti.I + D - 1j * k * S
    b = density(len(q), True, 4)
    for mode in ("fp64", "mixed"):
        x, st = inti.gmres(L, b, rtol=1e-10, restart=60, maxiter=400, mode=mode)
        assert st["converged"] == 1, st
        dS, dD = S.correction.arrays(), D.correction.arrays()
        Lx = 0.5 * x + (oracle_apply(O.HELMHOLTZ, O.DL, k, q, q, x) + O.csr_apply(*dD, x)) \
            - 1j * k * (oracle_apply(O.HELMHOLTZ, O.SL, k, q, q, x) + O.csr_apply(*dS, x))
        assert np.linalg.norm(b - Lx) / np.linalg.norm(b) < 2e-10


def test_gmres_zero_rhs_and_restart_cycles(ctx):
    q, S, D = laplace_problem(ctx, 3)
    L = D - 0.5 * inti.I
    x, st = inti.gmres(L, np.zeros(len(q)))
    assert np.all(x == 0) and st["relres"] == 0
    b = density(len(q), False, 8)
    x, st = inti.gmres(L, b, rtol=1e-10, restart=3, maxiter=400)
    assert st["converged"] == 1


def test_gmres_reports_nonconvergence(ctx):
    q, S, D = laplace_problem(ctx, 3)
    L = D - 0.5 * inti.I
    b = density(len(q), False, 9)
    x, st = inti.gmres(L, b, rtol=1e-14, restart=5, maxiter=4)
    assert st["converged"] == 0 and st["iterations"] == 4


def test_gmres_repeated_solves_reuse_derived_operators(ctx):
    """The fused combined-field operator and the FP32C twins are kept on the
    operators: a second solve repeats the first bit for bit, and a solve with
    another single layer or other coefficients rebuilds the fused operator."""
    q = inti.p2_sphere_quadrature(3)
    k = 2.0
    op = inti.Helmholtz(k=k, dim=3)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    b = density(len(q), True, 5)
    for mode in ("fp64", "mixed"):
        x1, st1 = inti.gmres(0.5 * inti.I + D - 1j * k * S, b, rtol=1e-10, restart=60, maxiter=400, mode=mode)
        x2, st2 = inti.gmres(0.5 * inti.I + D - 1j * k * S, b, rtol=1e-10, restart=60, maxiter=400, mode=mode)
        assert st1["converged"] == 1 and np.array_equal(x1, x2), mode
        assert st1["iterations"] == st2["iterations"]
    # other coefficients on the same pair of operators
    x3, st3 = inti.gmres(0.5 * inti.I + D - 2j * k * S, b, rtol=1e-10, restart=60, maxiter=400, mode="mixed")
    Lx = 0.5 * x3 + D @ x3 - 2j * k * (S @ x3)
    assert st3["converged"] == 1 and np.linalg.norm(b - Lx) / np.linalg.norm(b) < 2e-10
    # another single layer (no correction) with the same double layer
    S2 = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", ctx)
    x4, st4 = inti.gmres(0.5 * inti.I + D - 1j * k * S2, b, rtol=1e-10, restart=60, maxiter=400, mode="mixed")
    Lx = 0.5 * x4 + D @ x4 - 1j * k * (S2 @ x4)
    assert st4["converged"] == 1 and np.linalg.norm(b - Lx) / np.linalg.norm(b) < 2e-10
    assert not np.allclose(x3, x4)


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_gmres_small_form_matches_multi_kernel_form(ctx, mode):
    """The single-CTA Arnoldi step (systems of at most 8192 unknowns) and the
    multi-CTA kernels with a host Givens update give the same iterates up to
    rounding, real and complex, across restarts."""
    q, S, D = laplace_problem(ctx)
    qh = inti.p2_sphere_quadrature(3)
    Sh, Dh = inti.single_double_layer(op=inti.Helmholtz(k=2.0, dim=3), target=qh, source=qh,
                                      correction={"method": "dim"}, ctx=ctx)
    cases = [(D - 0.5 * inti.I, density(len(q), False, 13)), (0.5 * inti.I + Dh - 2j * Sh, density(len(qh), True, 14))]
    for L, b in cases:
        for restart in (4, 50):
            out = []
            for small in (8192, 0):
                ctx.set_gmres_small(small)
                try:
                    out.append(inti.gmres(L, b, rtol=1e-10, restart=restart, maxiter=400, mode=mode, history=True))
                finally:
                    ctx.set_gmres_small(8192)
            (x1, st1), (x0, st0) = out
            assert st1["converged"] == 1 and st0["converged"] == 1
            assert abs(st1["iterations"] - st0["iterations"]) <= 1, (st1, st0)
            assert relerr(x1, x0) < 1e-8
            assert st1["relres"] <= 1e-10


@pytest.mark.parametrize("small", [8192, 0])
def test_gmres_iteration_cap_across_batches_and_restarts(ctx, small):
    """maxiter reached inside a batch of small-system steps and across a
    restart: exactly maxiter iterations, reported as not converged, in both
    forms."""
    q, S, D = laplace_problem(ctx, 3)
    L = D - 0.5 * inti.I
    b = density(len(q), False, 17)
    ctx.set_gmres_small(small)
    try:
        for restart, maxiter in ((5, 6), (3, 7), (4, 4)):
            x, st = inti.gmres(L, b, rtol=1e-15, restart=restart, maxiter=maxiter, history=True)
            assert st["converged"] == 0 and st["iterations"] == maxiter, (restart, maxiter, st)
            assert np.all(np.isfinite(x))
            h = st["history"]
            assert len(h) >= maxiter + 1 and np.all(np.isfinite(h[: maxiter + 1]))
    finally:
        ctx.set_gmres_small(8192)


@pytest.mark.parametrize("small", [8192, 0])
def test_gmres_lucky_breakdown(ctx, small):
    """L = I + 0·S: the first Krylov step breaks down (the new vector is
    zero), which ends the cycle with the exact solution in both forms."""
    q, S, D = laplace_problem(ctx, 3)
    b = density(len(q), False, 19)
    ctx.set_gmres_small(small)
    try:
        x, st = inti.gmres(1.0 * inti.I + 0.0 * S, b, rtol=1e-12, restart=10, maxiter=50)
    finally:
        ctx.set_gmres_small(8192)
    assert st["converged"] == 1 and st["iterations"] == 1, st
    assert relerr(x, b) < 1e-14
