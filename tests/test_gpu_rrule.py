"""The reverse rule of u = A σ (the Python counterpart of the Julia
binding's ChainRules rrule): pullbacks against central finite differences
(h = 1e-6, FP64), the oracle's dual-number directional derivatives (the
method of ForwardDiff, the reference's only differentiation route:
src/reference_interpolation.jl:36-39, test/kernels_test.jl:41-67), and the
dense oracle transpose for corrected and complex operators; the torch
autograd wrapper against the same rule."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, relerr

pytestmark = pytest.mark.gpu


def _potential_setup(ctx, kind):
    q = inti.ellipsoid_quadrature(3, 5)
    tgt = inti.points(1.5 * inti.ellipsoid_quadrature(2, 3).coords)
    A = inti.GpuOperator(kind(inti.Laplace(dim=3)), tgt, q, ctx=ctx)
    return q, tgt, A, density(len(q), False, 2), 0.01 * density(len(tgt), False, 3)


def _J(tgt, x, n, w, s, ustar, okind):
    u = O.apply(O.LAPLACE, okind, 0.0, tgt.coords, None, x, n, w, s)
    return 0.5 * np.sum((u - ustar) ** 2)


@pytest.mark.parametrize("kind,okind", [(inti.DoubleLayerKernel, O.DL), (inti.SingleLayerKernel, O.SL)])
def test_pullback_matches_finite_differences(ctx, kind, okind):
    q, tgt, A, sigma, ustar = _potential_setup(ctx, kind)
    u, pb = inti.rrule(A, sigma)
    g = pb(u - ustar)
    assert g["geometry"] == "exact"
    r = np.random.default_rng(5)
    h = 1e-6
    base = {"coords": q.coords, "normals": q.normals, "weights": q.weights, "sigma": sigma}
    for name in base:
        v = r.standard_normal(base[name].shape)
        p, m = dict(base), dict(base)
        p[name], m[name] = base[name] + h * v, base[name] - h * v
        fd = (_J(tgt, p["coords"], p["normals"], p["weights"], p["sigma"], ustar, okind)
              - _J(tgt, m["coords"], m["normals"], m["weights"], m["sigma"], ustar, okind)) / (2 * h)
        ad = float(np.sum(g[name] * v))
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-8), (name, ad, fd)


def test_pullback_matches_dual_numbers(ctx):
    q, tgt, A, sigma, ustar = _potential_setup(ctx, inti.DoubleLayerKernel)
    u, pb = inti.rrule(A, sigma)
    ubar = u - ustar
    g = pb(ubar)
    r = np.random.default_rng(6)
    dsx, dsn, dsw, dsg = (r.standard_normal(q.coords.shape), r.standard_normal(q.normals.shape),
                          r.standard_normal(len(q)), r.standard_normal(len(q)))
    _, du = O.dl_potential_jvp(tgt.coords, q.coords, q.normals, q.weights, sigma, dsx, dsn, dsw, dsg)
    jvp = float(np.dot(ubar, du))
    ad = float(np.sum(g["coords"] * dsx) + np.sum(g["normals"] * dsn) + np.sum(g["weights"] * dsw)
               + np.sum(g["sigma"] * dsg))
    assert abs(ad - jvp) <= 1e-10 * max(abs(jvp), 1.0)


@pytest.mark.parametrize("pde", ["laplace", "helmholtz"])
def test_corrected_operator_density_cotangent_is_adjoint(ctx, pde):
    """On-surface operators with their DIM correction: ∂J/∂σ = (A + C)ᴴ ū
    against the dense oracle matrix plus the oracle-built correction."""
    q = inti.p2_sphere_quadrature(3) if pde == "helmholtz" else inti.ellipsoid_quadrature(3, 5)
    op = inti.Helmholtz(k=4.0, dim=3) if pde == "helmholtz" else inti.Laplace(dim=3)
    opde, k = (O.HELMHOLTZ, 4.0) if pde == "helmholtz" else (O.LAPLACE, 0.0)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    cplx = pde == "helmholtz"
    sigma, ubar = density(len(q), cplx, 7), density(len(q), cplx, 8)
    u, pb = inti.rrule(D, sigma)
    g = pb(ubar)
    Ad = O.assemble(opde, O.DL, k, q.coords, q.normals, q.coords, q.normals, q.weights)
    rp, col, val = D.correction.arrays()
    Cd = np.zeros_like(Ad)
    for i in range(len(q)):
        Cd[i, col[rp[i]:rp[i + 1]]] += val[rp[i]:rp[i + 1]]
    assert relerr(u, (Ad + Cd) @ sigma) < 1e-12
    assert relerr(g["sigma"], (Ad + Cd).conj().T @ ubar) < 1e-12
    if cplx:
        assert g["coords"] is None
    else:
        assert g["geometry"].startswith("pair terms only")
        # the geometry cotangents of the pair part equal the uncorrected operator's
        A0 = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, None, "fp64", ctx)
        g0 = inti.rrule(A0, sigma)[1](ubar)
        for name in ("coords", "normals", "weights"):
            assert relerr(g[name], g0[name]) < 1e-14


def test_torch_autograd_wrapper(ctx):
    """J = ½‖u − u*‖² through TorchPotential: torch's backward equals the
    rule's pullback and central differences of the oracle."""
    import torch

    q, tgt, A, sigma, ustar = _potential_setup(ctx, inti.DoubleLayerKernel)
    dev = torch.device("cuda:0")
    ts = torch.tensor(sigma, device=dev, requires_grad=True)
    tx = torch.tensor(q.coords, device=dev, requires_grad=True)
    tn = torch.tensor(q.normals, device=dev, requires_grad=True)
    tw = torch.tensor(q.weights, device=dev, requires_grad=True)
    tt = torch.tensor(tgt.coords, device=dev)
    u = inti.TorchPotential(ts, tx, tn, tw, tt, "DL", ctx)
    J = 0.5 * torch.sum((u - torch.tensor(ustar, device=dev)) ** 2)
    J.backward()
    ref_u, pb = inti.rrule(A, sigma)
    g = pb(ref_u - ustar)
    assert relerr(u.detach().cpu().numpy(), ref_u) < 1e-14
    for t, name in ((ts, "sigma"), (tx, "coords"), (tn, "normals"), (tw, "weights")):
        assert relerr(t.grad.cpu().numpy(), g[name]) < 1e-14, name
    h, v = 1e-6, np.random.default_rng(9).standard_normal(q.coords.shape)
    fd = (_J(tgt, q.coords + h * v, q.normals, q.weights, sigma, ustar, O.DL)
          - _J(tgt, q.coords - h * v, q.normals, q.weights, sigma, ustar, O.DL)) / (2 * h)
    assert abs(float(np.sum(tx.grad.cpu().numpy() * v)) - fd) <= 1e-6 * abs(fd)
