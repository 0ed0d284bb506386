"""Pins of the CPU oracle against the reference's own known-answer tests.

Inti.jl has no golden vectors; its tests check identities.  The same
identities, with the reference's tolerances, are re-run here on the oracle:

* Green's identity ``S[γ₁u] − D[γ₀u] − σγ₀u ≈ 0`` with the DIM correction,
  circle (2D) and ellipsoid (3D), meshsize 0.5, qorder 5, Laplace and
  Helmholtz(k=1.2), interior/exterior, rtol 1e-2 (SL/DL) and 5e-2 (ADL/HS),
  and the corrected error below the uncorrected one
  (test/green_identities_test.jl:28-133);
* the tight form of it on a smooth closed curve, error < 1e-6
  (test/normal_orientation_test.jl:94-113; the annulus there is a gmsh
  mesh, the kite of the 2D workload stands in for it);
* normal-derivative consistency of the kernels by finite differences
  (pattern of test/kernels_test.jl:41-67);
* quadrature identities (src/reference_integration.jl doctest,
  test/quadrature_test.jl:156-161, test/meshgen_test.jl:16-26);
* matrix-free versus entry-wise rows, rtol 1e-7 (test/fmm3d_test.jl:19-46);
* closed forms on the unit sphere (S[1] = 1 for Laplace,
  S[1] = e^{ik} sin(k)/k for Helmholtz, D[1] = −1/2).
"""
import math

import numpy as np
import pytest

import oracle as O
from helpers import density, harmonic_traces, oracle_dim_csr, relerr
from inti_b200 import geometry as G


def circle_q():
    # meshsize 0.5 on the unit circle: ceil(2π/0.5) = 13 elements, qorder 5
    return G.circle_quadrature(13, 5)


def ellipsoid_q():
    # meshsize 0.5 on the unit ellipsoid: patch edges of length acos(1/3) -> 3 cells
    return G.ellipsoid_quadrature(3, 5, (1.0, 1.0, 1.0))


def _green_errors(pde, k, q, xs, sigma_jump, derivative):
    """(e0, e1): uncorrected and DIM-corrected Green-identity errors."""
    c = 0.7 - 0.3j if pde == O.HELMHOLTZ else 0.7
    dt = np.complex128 if pde == O.HELMHOLTZ else np.float64
    g0 = np.array([O.kernel(pde, O.SL, k, x, n, xs, None) for x, n in zip(q.coords, q.normals)]) * c
    g1 = np.array([O.kernel(pde, O.ADL, k, x, n, xs, None) for x, n in zip(q.coords, q.normals)]) * c
    g0, g1 = (g0, g1) if dt is np.complex128 else (g0.real.copy(), g1.real.copy())
    if derivative:
        kS, kD, ref = O.ADL, O.HS, g1
    else:
        kS, kD, ref = O.SL, O.DL, g0
    args = (q.coords, q.normals, q.coords, q.normals, q.weights)
    Sg1 = O.apply(pde, kS, k, *args, g1)
    Dg0 = O.apply(pde, kD, k, *args, g0)
    e0 = np.max(np.abs(Sg1 - Dg0 - sigma_jump * ref)) / np.max(np.abs(ref))
    dS, dD = oracle_dim_csr(pde, k, q, derivative=derivative)
    Sg1c = Sg1 + O.csr_apply(*dS, g1)
    Dg0c = Dg0 + O.csr_apply(*dD, g0)
    e1 = np.max(np.abs(Sg1c - Dg0c - sigma_jump * ref)) / np.max(np.abs(ref))
    return e0, e1


CASES = [
    ("laplace2d", O.LAPLACE, 0.0, 2),
    ("laplace3d", O.LAPLACE, 0.0, 3),
    ("helmholtz3d", O.HELMHOLTZ, 1.2, 3),
]


@pytest.mark.parametrize("name,pde,k,dim", CASES)
@pytest.mark.parametrize("side", ["interior", "exterior"])
@pytest.mark.parametrize("derivative", [False, True])
def test_green_identity_dim(name, pde, k, dim, side, derivative):
    q = circle_q() if dim == 2 else ellipsoid_q()
    xs = np.full(dim, 3.0) if side == "interior" else np.full(dim, 0.1)
    sigma = 0.5 if side == "interior" else -0.5
    e0, e1 = _green_errors(pde, k, q, xs, sigma, derivative)
    rtol = 5e-2 if derivative else 1e-2
    assert e1 < rtol, (e0, e1)
    assert e0 > e1, (e0, e1)


def test_green_identity_tight_kite():
    """A smooth curve with qorder 9 (GL5) and 200 panels: error < 1e-6."""
    q = G.kite_quadrature(200, 9)
    e0, e1 = _green_errors(O.LAPLACE, 0.0, q, np.array([3.0, -5.2]), 0.5, False)
    assert e1 < 1e-6, e1
    assert e0 > e1


def test_gauss_law_kite():
    """D[1] = -1/2 on the curve (the :on green multiplier, src/nystrom.jl:196-207)."""
    q = G.kite_quadrature(200, 9)
    one = np.ones(len(q))
    D1 = O.apply(O.LAPLACE, O.DL, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights, one)
    _, dD = oracle_dim_csr(O.LAPLACE, 0.0, q)
    assert np.max(np.abs(D1 + O.csr_apply(*dD, one) + 0.5)) < 1e-6


def test_sphere_closed_forms():
    """Unit sphere (P2 triangles, VR-6): S[1] = 1, D[1] = -1/2 (Laplace) and
    S[1] = e^{ik} sin(k)/k (Helmholtz), with DIM corrections."""
    q = G.p2_sphere_quadrature(4)
    n = len(q)
    one = np.ones(n)
    dS, dD = oracle_dim_csr(O.LAPLACE, 0.0, q)
    args = (q.coords, q.normals, q.coords, q.normals, q.weights)
    S1 = O.apply(O.LAPLACE, O.SL, 0.0, *args, one) + O.csr_apply(*dS, one)
    D1 = O.apply(O.LAPLACE, O.DL, 0.0, *args, one) + O.csr_apply(*dD, one)
    assert np.max(np.abs(S1 - 1.0)) < 2e-3
    assert np.max(np.abs(D1 + 0.5)) < 2e-3
    k = 2.0
    hS, _ = oracle_dim_csr(O.HELMHOLTZ, k, q)
    onec = one.astype(np.complex128)
    HS1 = O.apply(O.HELMHOLTZ, O.SL, k, *args, onec) + O.csr_apply(*hS, onec)
    ref = np.exp(1j * k) * np.sin(k) / k
    assert np.max(np.abs(HS1 - ref)) < 5e-3 * abs(ref) + 2e-3


@pytest.mark.parametrize("pde,k,dim", [(O.LAPLACE, 0.0, 2), (O.LAPLACE, 0.0, 3), (O.HELMHOLTZ, 1.7, 3)])
def test_kernel_normal_derivatives(pde, k, dim):
    """DL = ∂SL/∂n_y, ADL = ∂SL/∂n_x, HS = ∂DL/∂n_x (central differences)."""
    r = np.random.default_rng(0)
    x = r.standard_normal(dim)
    y = r.standard_normal(dim)
    nx = r.standard_normal(dim)
    nx /= np.linalg.norm(nx)
    ny = r.standard_normal(dim)
    ny /= np.linalg.norm(ny)
    h = 1e-6
    sl = lambda a, b: O.kernel(pde, O.SL, k, a, None, b, None)
    dl = lambda a, b: O.kernel(pde, O.DL, k, a, None, b, ny)
    d_dny = (sl(x, y + h * ny) - sl(x, y - h * ny)) / (2 * h)
    assert abs(O.kernel(pde, O.DL, k, x, None, y, ny) - d_dny) < 1e-7 * max(1, abs(d_dny))
    d_dnx = (sl(x + h * nx, y) - sl(x - h * nx, y)) / (2 * h)
    assert abs(O.kernel(pde, O.ADL, k, x, nx, y, None) - d_dnx) < 1e-7 * max(1, abs(d_dnx))
    dd = (dl(x + h * nx, y) - dl(x - h * nx, y)) / (2 * h)
    assert abs(O.kernel(pde, O.HS, k, x, nx, y, ny) - dd) < 1e-6 * max(1, abs(dd))


def test_self_pair_is_zero():
    """K(x, x) = 0 for every kernel (src/utils.jl:235)."""
    x = np.array([0.3, -0.2, 0.5])
    n = np.array([0.0, 0.0, 1.0])
    for pde, k in ((O.LAPLACE, 0.0), (O.HELMHOLTZ, 3.0)):
        for kind in (O.SL, O.DL, O.ADL, O.HS):
            assert O.kernel(pde, kind, k, x, n, x, n) == 0
            # within the tolerance: still excluded
            assert O.kernel(pde, kind, k, x, n, x + 5e-15, n) == 0


def test_quadrature_identities():
    x, w = G.gauss_legendre_for_order(10)
    assert abs(np.sum(w * np.cos(x)) - math.sin(1.0)) < 1e-15
    # parametric circle, ∫1 = 2π (test/quadrature_test.jl:156-161)
    q = G.circle_quadrature(63, 2)
    assert abs(q.integrate(lambda x: 1.0) - 2 * np.pi) < 1e-12
    # meshgen'd circle of radius 0.5 split in two arcs, 100 elements each
    # (test/meshgen_test.jl:16-26): perimeter 2π r
    q = G.circle_quadrature(200, 2, r=0.5)
    assert abs(q.integrate(lambda x: 1.0) - np.pi) < 1e-12
    # unit sphere area through the cube-sphere patches
    s = G.ellipsoid_quadrature(8, 5, (1, 1, 1))
    assert abs(s.integrate(lambda x: 1.0) - 4 * np.pi) < 1e-6
    # divergence theorem on the (1, 0.7, 0.5) ellipsoid: ∫ x·n = 3 vol
    e = G.ellipsoid_quadrature(12, 5)
    vol = np.sum(np.sum(e.coords * e.normals, 1) * e.weights) / 3
    assert abs(vol - 4 / 3 * np.pi * 0.35) < 1e-9


def test_matrix_free_vs_entrywise():
    """On-the-fly rows equal rows of the assembled matrix times x, rtol 1e-7
    (test/fmm3d_test.jl:40-42); here the agreement is to rounding."""
    q = G.ellipsoid_quadrature(3, 5)
    for pde, k in ((O.LAPLACE, 0.0), (O.HELMHOLTZ, 1.2)):
        for kind in (O.SL, O.DL, O.ADL, O.HS):
            x = density(len(q), pde == O.HELMHOLTZ)
            args = (q.coords, q.normals, q.coords, q.normals, q.weights)
            A = O.assemble(pde, kind, k, *args)
            idx = np.random.default_rng(2).integers(0, len(q), 10)
            y = O.apply(pde, kind, k, *args, x, rows=idx)
            assert relerr(y, A[idx, :] @ x) < 1e-12


def test_coo_to_csr_sums_duplicates():
    I = np.array([2, 0, 2, 1, 0])
    J = np.array([1, 3, 1, 0, 0])
    V = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    rp, col, val = O.coo_to_csr(3, I, J, V)
    assert rp.tolist() == [0, 2, 3, 4]
    assert col.tolist() == [0, 3, 0, 1]
    assert val.tolist() == [5.0, 2.0, 4.0, 4.0]


def test_dim_sources():
    xs = O.dim_sources(3, 27, 2.0, np.array([0.1, 0.2, 0.3]))
    assert np.allclose(np.linalg.norm(xs - [0.1, 0.2, 0.3], axis=1), 2.0)
    xs2 = O.dim_sources(2, 15, 1.5, np.zeros(2))
    assert np.allclose(xs2[0], [1.5, 0.0])


def test_gmres_oracle_against_dense_solve():
    q = G.kite_quadrature(30, 9)
    n = len(q)
    _, dD = oracle_dim_csr(O.LAPLACE, 0.0, q)
    A = O.assemble(O.LAPLACE, O.DL, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights)
    import scipy.sparse as sp

    Dfull = A + sp.csr_matrix((dD[2], dD[1], dD[0]), shape=(n, n)).toarray()
    L = -0.5 * np.eye(n) + Dfull
    b = density(n, False, 5)
    x, st = O.gmres(O.LAPLACE, 0.0, q.coords, q.normals, q.weights, -0.5, [(O.DL, 1.0, dD)], b, rtol=1e-12)
    assert st["relres"] < 1e-12
    assert relerr(x, np.linalg.solve(L, b)) < 1e-9


def test_dual_number_jvp_matches_finite_differences():
    q = G.ellipsoid_quadrature(2, 5)
    r = np.random.default_rng(4)
    tgt = 1.5 * G.ellipsoid_quadrature(1, 3).coords
    sigma = r.standard_normal(len(q))
    dsx = r.standard_normal(q.coords.shape)
    u, du = O.dl_potential_jvp(tgt, q.coords, q.normals, q.weights, sigma, dsx=dsx)
    h = 1e-6
    up = O.apply(O.LAPLACE, O.DL, 0.0, tgt, None, q.coords + h * dsx, q.normals, q.weights, sigma)
    um = O.apply(O.LAPLACE, O.DL, 0.0, tgt, None, q.coords - h * dsx, q.normals, q.weights, sigma)
    assert relerr(du, (up - um) / (2 * h)) < 1e-7
    assert relerr(u, O.apply(O.LAPLACE, O.DL, 0.0, tgt, None, q.coords, q.normals, q.weights, sigma)) < 1e-14


# ----------------------------------------------------------------------------
# Off-surface DIM (target !== source), the reference's "Issue 136 - mixed
# targets" test (test/dim_test.jl:42-91): unit circle, meshsize 0.2 (32 panels),
# qorder 3; targets on the 31 x 31 grid of [-1.5, 1.5]^2.
# ----------------------------------------------------------------------------
def _targets_apply(pde, kind, k, T, q, corr, x):
    near, vals = corr
    ip, ix, dv = O.targets_csr(near, vals, q.nq, len(q))
    import scipy.sparse as sp

    return O.apply(pde, kind, k, T, None, q.coords, q.normals, q.weights, x) + \
        sp.csr_matrix((dv, ix, ip), shape=(len(T), len(q))) @ x


def test_dim_mixed_targets_known_answers():
    q = G.circle_quadrature(32, 3)
    g = np.arange(-1.5, 1.5 + 1e-9, 0.1)
    T = np.array([(a, b) for a in g for b in g])
    inn = np.linalg.norm(T, axis=1) < 1.0
    u = np.ones(len(q))
    # mixed green multipliers, maxdist = Inf
    near, dS, dD = O.bdim_targets(O.LAPLACE, 0.0, T, q.coords, q.normals, q.weights, q.nq, np.where(inn, -1.0, 0.0))
    # separately for the outside (0) and inside (-1) targets
    To, Ti = T[~inn], T[inn]
    no, dSo, dDo = O.bdim_targets(O.LAPLACE, 0.0, To, q.coords, q.normals, q.weights, q.nq, 0.0)
    ni, dSi, dDi = O.bdim_targets(O.LAPLACE, 0.0, Ti, q.coords, q.normals, q.weights, q.nq, -1.0)
    Dout = _targets_apply(O.LAPLACE, O.DL, 0.0, To, q, (no, dDo), u)
    Din = _targets_apply(O.LAPLACE, O.DL, 0.0, Ti, q, (ni, dDi), u)
    assert np.max(np.abs(Dout)) < 1e-3          # test/dim_test.jl:79
    assert np.max(np.abs(Din + 1)) < 1e-3       # test/dim_test.jl:80
    S = _targets_apply(O.LAPLACE, O.SL, 0.0, T, q, (near, dS), u)
    So = _targets_apply(O.LAPLACE, O.SL, 0.0, To, q, (no, dSo), u)
    Si = _targets_apply(O.LAPLACE, O.SL, 0.0, Ti, q, (ni, dSi), u)
    assert np.max(np.abs(S[inn] - Si)) < 1e-3   # test/dim_test.jl:89
    assert np.max(np.abs(S[~inn] - So)) < 1e-3  # test/dim_test.jl:90
    # every target is near something when maxdist = Inf
    assert np.all(near >= 0)


def _sphere_targets(m=200, seed=0):
    r = np.random.default_rng(seed)
    d = r.standard_normal((m, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rad = np.where(np.arange(m) % 2 == 0, 0.9, 1.1)
    return d * rad[:, None], rad < 1


@pytest.mark.parametrize("pde,k", [(O.LAPLACE, 0.0), (O.HELMHOLTZ, 3.0)])
def test_dim_off_surface_green_identity_3d(pde, k):
    """Green's representation S[γ₁u] − D[γ₀u] = u inside, 0 outside for u
    radiating from x0 outside, at targets 0.1 off the unit sphere, where the
    plain quadrature is off by ~2.5e-3."""
    q = G.ellipsoid_quadrature(6, 5, scaling=(1.0, 1.0, 1.0))
    T, inn = _sphere_targets()
    x0 = np.array([1.8, 0.3, -0.2])
    g0, g1 = harmonic_traces(pde, k, q, x0, c=1.0)
    uT = np.array([O.kernel(pde, O.SL, k, t, None, x0, None) for t in T])
    uT = uT.real if pde == O.LAPLACE else uT
    near, dS, dD = O.bdim_targets(pde, k, T, q.coords, q.normals, q.weights, q.nq, np.where(inn, -1.0, 0.0))
    lhs0 = O.apply(pde, O.SL, k, T, None, q.coords, q.normals, q.weights, g1) - \
        O.apply(pde, O.DL, k, T, None, q.coords, q.normals, q.weights, g0)
    lhs = _targets_apply(pde, O.SL, k, T, q, (near, dS), g1) - _targets_apply(pde, O.DL, k, T, q, (near, dD), g0)
    ref = np.where(inn, uT, 0)
    err0, err = np.max(np.abs(lhs0 - ref)), np.max(np.abs(lhs - ref))
    assert err < 1e-4 and err < err0 / 50, (err, err0)


# ----------------------------------------------------------------------------
# VDIM on the unit disk (src/vdim.jl:30-130): the volume potential of radial
# densities is known in closed form, V[1] = (1 - r^2)/4, V[r^2] = (1 - r^4)/16
# (−ΔV = f inside, V = 0 on the unit circle for radial f).
# ----------------------------------------------------------------------------
@pytest.mark.parametrize("order", [2, 4])
def test_vdim_disk_known_answers(order):
    Y = G.disk_triangle_quadrature(4)
    B = G.circle_quadrature(64, 8)
    near, vals = O.vdim(Y.coords, Y.coords, Y.weights, Y.nq, B.coords, B.normals, B.weights, B.nq, -1.0, order,
                        same=True)
    ip, ix, dv = O.targets_csr(near, vals, Y.nq, len(Y))
    r2 = (Y.coords ** 2).sum(1)
    for f, exact in ((np.ones(len(Y)), (1 - r2) / 4), (r2, (1 - r2 ** 2) / 16)):
        V0 = O.apply(O.LAPLACE, O.SL, 0.0, Y.coords, None, Y.coords, None, Y.weights, f)
        Vc = V0 + O.csr_apply(ip, ix, dv, f)
        err0, err = np.max(np.abs(V0 - exact)), np.max(np.abs(Vc - exact))
        assert err < 1e-6 and err < err0 / 1e3, (err, err0)


# VDIM in the unit ball (3D Laplace): V[1] = (3 - r^2)/6 and
# V[r^2] = 1/4 - r^4/20 inside (the Newton potential of radial densities).
def test_vdim_ball_known_answers():
    Y = G.ball_hex_quadrature(2)
    B = G.ellipsoid_quadrature(16, 5, scaling=(1.0, 1.0, 1.0))
    near, vals = O.vdim(Y.coords, Y.coords, Y.weights, Y.nq, B.coords, B.normals, B.weights, B.nq, -1.0, 2,
                        same=True)
    ip, ix, dv = O.targets_csr(near, vals, Y.nq, len(Y))
    r2 = (Y.coords ** 2).sum(1)
    for f, exact in ((np.ones(len(Y)), (3 - r2) / 6), (r2, 0.25 - r2 ** 2 / 20)):
        V0 = O.apply(O.LAPLACE, O.SL, 0.0, Y.coords, None, Y.coords, None, Y.weights, f)
        Vc = V0 + O.csr_apply(ip, ix, dv, f)
        err0, err = np.max(np.abs(V0 - exact)), np.max(np.abs(Vc - exact))
        assert err < 1e-6 and err < err0 / 1e3, (err, err0)


# VDIM in the unit ball, 3D Helmholtz (src/vdim.jl:369-373: the polynomial
# solutions of ΔP + k²P = p, unique): V[1] = -1/k² + (1 - ik) e^{ik}
# sin(kr) / (k³ r) inside, the outgoing volume potential of the indicator
# (radial, regular at 0, matched to e^{ikr}/r at r = 1; k -> 0 gives the
# Laplace (3 - r²)/6).
@pytest.mark.parametrize("k", [2.0, 4.0])
def test_vdim_ball_helmholtz_known_answer(k):
    Y = G.ball_hex_quadrature(2)
    B = G.ellipsoid_quadrature(16, 5, scaling=(1.0, 1.0, 1.0))
    near, vals = O.vdim(Y.coords, Y.coords, Y.weights, Y.nq, B.coords, B.normals, B.weights, B.nq, -1.0, 2,
                        same=True, pde=O.HELMHOLTZ, k=k)
    ip, ix, dv = O.targets_csr(near, vals, Y.nq, len(Y))
    r = np.sqrt((Y.coords ** 2).sum(1))
    exact = -1 / k ** 2 + (1 - 1j * k) * np.exp(1j * k) * np.sin(k * r) / (k ** 3 * r)
    f = np.ones(len(Y))
    V0 = O.apply(O.HELMHOLTZ, O.SL, k, Y.coords, None, Y.coords, None, Y.weights, f)
    Vc = V0 + O.csr_apply(ip, ix, dv, f)
    err0, err = np.max(np.abs(V0 - exact)), np.max(np.abs(Vc - exact))
    assert err < 1e-6 and err < err0 / 1e3, (err, err0)


def test_ball_quadrature_moments():
    """Volume and second moment of the curved-hexahedron ball converge."""
    errs = []
    for m in (2, 3):
        Y = G.ball_hex_quadrature(m)
        r2 = (Y.coords ** 2).sum(1)
        errs.append(max(abs(Y.weights.sum() - 4 * np.pi / 3), abs((Y.weights * r2).sum() - 4 * np.pi / 5)))
        assert np.all(np.sqrt(r2) < 1.0) and Y.nq == 27 and len(Y) == 7 * m ** 3 * 27
    assert errs[1] < 1e-4 and errs[1] < errs[0] / 10, errs
