"""GPU BDIM correction versus the oracle.

* Pattern and indexing: bit-exact.
* Values: each weight solves a small least-squares problem with matrix
  M_e^T (src/bdim.jl:160-170), whose condition number reaches 1e11-1e15 on
  fine meshes; no two implementations (LAPACK included) agree beyond
  cond(M_e)·eps (times a modest factor: least-squares problems with a
  nonzero residual are more sensitive still).  The check is per element:
  max|Δδ| <= 1024·eps·cond(M_e)·max|δ|.
* The quantity the correction exists for — the Green-identity combination
  S[γ₁u] − D[γ₀u] on traces of a harmonic u — must agree with the oracle's
  to 1e-9 relative.
"""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import (block_rows_apply, density, dim_values_close, harmonic_traces, oracle_apply, oracle_dim_csr,
                     relerr, small_surfaces, smooth_density)

pytestmark = pytest.mark.gpu

SURF = small_surfaces()


def _identity_combo(pde, k, q, dS, dD, derivative, xs):
    g0, g1 = harmonic_traces(pde, k, q, xs)
    kS, kD = (O.ADL, O.HS) if derivative else (O.SL, O.DL)
    a = oracle_apply(pde, kS, k, q, q, g1) + O.csr_apply(*dS, g1)
    b = oracle_apply(pde, kD, k, q, q, g0) + O.csr_apply(*dD, g0)
    return a - b, (g1 if derivative else g0)


@pytest.mark.parametrize("surf", list(SURF))
@pytest.mark.parametrize("derivative", [False, True])
def test_dim_matches_oracle(ctx, surf, derivative):
    q = SURF[surf]
    ops = [(inti.Laplace(dim=q.dim), O.LAPLACE, 0.0)]
    if q.dim == 3:
        ops.append((inti.Helmholtz(k=2.5, dim=3), O.HELMHOLTZ, 2.5))
    xs = np.full(q.dim, 3.0)
    for op, pde, k in ops:
        gS, gD = inti.bdim_correction(op, q, q, derivative=derivative, ctx=ctx)
        oS, oD = oracle_dim_csr(pde, k, q, derivative=derivative)
        gs, gd = gS.arrays(), gD.arrays()
        for g, o in ((gs, oS), (gd, oD)):
            assert np.array_equal(g[0], o[0]) and np.array_equal(g[1], o[1])
            assert dim_values_close(pde, k, q, g, o) <= 1.0
        cg, ref = _identity_combo(pde, k, q, gs, gd, derivative, xs)
        co, _ = _identity_combo(pde, k, q, oS, oD, derivative, xs)
        assert np.max(np.abs(cg - co)) <= 1e-9 * np.max(np.abs(ref)), (surf, op)


def test_dim_kite_workload(ctx):
    """2D Laplace double layer on the kite, 200 GL-5 panels (N = 1000): the
    fused GPU product equals the oracle's product with the same correction
    data to 1e-12; the corrections agree through Green's identity."""
    q = inti.kite_quadrature()
    op = inti.Laplace(dim=2)
    S, D = inti.single_double_layer(op=op, target=q, source=q, compression={"method": "none"},
                                    correction={"method": "dim"}, ctx=ctx)
    sigma = density(len(q), False, 1)
    gD = D.correction.arrays()
    ref = oracle_apply(O.LAPLACE, O.DL, 0.0, q, q, sigma) + O.csr_apply(*gD, sigma)
    assert relerr(D @ sigma, ref) < 1e-12
    oS, oD = oracle_dim_csr(O.LAPLACE, 0.0, q)
    assert np.array_equal(gD[0], oD[0]) and np.array_equal(gD[1], oD[1])
    assert D.correction.nnz == 5000
    xs = np.array([3.0, -5.2])
    g0, g1 = harmonic_traces(O.LAPLACE, 0.0, q, xs, 1.3)
    e_gpu = np.max(np.abs(S @ g1 - D @ g0 - 0.5 * g0)) / np.max(np.abs(g0))
    cg, _ = _identity_combo(O.LAPLACE, 0.0, q, S.correction.arrays(), gD, False, xs)
    co, _ = _identity_combo(O.LAPLACE, 0.0, q, oS, oD, False, xs)
    assert e_gpu < 1e-6  # test/normal_orientation_test.jl:112
    assert np.max(np.abs(cg - co)) <= 1e-9 * np.max(np.abs(g0))


def test_green_multiplier_vector(ctx):
    q = SURF["ellipsoid"]
    gm = np.linspace(-1.0, 0.0, len(q))
    pair = inti.bdim_correction(inti.Laplace(dim=3), q, q, green_multiplier=gm, ctx=ctx)
    ref = oracle_dim_csr(O.LAPLACE, 0.0, q, green_multiplier=gm)
    for g, r in zip(pair, ref):
        assert dim_values_close(O.LAPLACE, 0.0, q, g.arrays(), r) <= 1.0


def test_gauss_law_and_green_identity_on_gpu(ctx):
    """D[1] = -1/2 and Green's identity < 1e-2 (test/green_identities_test.jl)."""
    q = inti.ellipsoid_quadrature(3, 5, (1.0, 1.0, 1.0))
    op = inti.Laplace(dim=3)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    assert np.max(np.abs(D @ np.ones(len(q)) + 0.5)) < 1e-2
    g0, g1 = harmonic_traces(O.LAPLACE, 0.0, q, np.array([3.0, 3.0, 3.0]))
    e1 = np.max(np.abs(S @ g1 - D @ g0 - 0.5 * g0)) / np.max(np.abs(g0))
    assert e1 < 1e-2


# Product-level bounds of the corrected C1 operators, (A + δ_gpu)σ against
# (A + δ_oracle)σ with δ_oracle from the oracle's own BDIM.  On the kite the
# element matrices reach cond(M_e) ≈ 8e14, so the weights are fixed only up
# to the near-null directions of M_e: rounding-level differences in the
# traces and in Θ move them there.  An N(0,1) density picks those up; a
# smooth density (what the correction is built to integrate) does not.
# Measured on the host with the oracle's own problems: a second QR solver
# changes the random-density product by 6.8e-3, relative perturbations of
# the traces of 1e-15 / 1e-14 by 3.1e-2 / 7.8e-2.  The GPU traces (their own
# log and reciprocal square root) and Θ (FP64 MMA, another summation order)
# differ at that level.  Measured on the B200: DL 8.5e-2 (random) and
# 5.8e-10 (smooth), SL 1.2e-3 and 4.8e-9; the bounds below.
C1_BOUNDS = {"DL": (0.2, 5e-9), "SL": (1e-2, 2e-8)}  # (random N(0,1), smooth)


def test_c1_corrected_product_against_oracle_correction(ctx):
    q = inti.kite_quadrature()
    assert len(q) == 1000
    op = inti.Laplace(dim=2)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    oS, oD = O.bdim(O.LAPLACE, 0.0, q.coords, q.normals, q.weights, q.nq)
    els = np.arange(q.nel)
    dens = {"random": density(len(q), False, 1), "smooth": smooth_density(O.LAPLACE, 0.0, q, np.array([3.0, -5.2]))}
    for name, A, kind, ov in (("DL", D, O.DL, oD), ("SL", S, O.SL, oS)):
        for which, sigma in dens.items():
            ref = oracle_apply(O.LAPLACE, kind, 0.0, q, q, sigma) + block_rows_apply(ov, q.nq, els, sigma)
            err = relerr(A @ sigma, ref)
            print(f"C1 {name} {which}: (A+dgpu)s vs (A+dora)s rel err {err:.3e}")
            assert err < C1_BOUNDS[name][0 if which == "random" else 1], (name, which, err)
