"""Hand-written adjoint: gradients of J = ½‖u − u*‖², u = D[σ] at exterior
targets, with respect to σ and every node's coordinates, normal and weight,
checked against central finite differences (h = 1e-6, FP64) and against a
forward-mode (dual number) restatement of the CPU matvec; single and double
layer, 3D and 2D, one and many thread blocks of sources."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, relerr

pytestmark = pytest.mark.gpu


def setup(ctx, kind=inti.DoubleLayerKernel):
    q = inti.ellipsoid_quadrature(3, 5)
    tgt = inti.points(1.5 * inti.ellipsoid_quadrature(2, 3).coords)
    op = inti.GpuOperator(kind(inti.Laplace(dim=3)), tgt, q, ctx=ctx)
    sigma = density(len(q), False, 2)
    ustar = density(len(tgt), False, 3) * 0.01
    return q, tgt, op, sigma, ustar


def J(tgt, coords, normals, weights, sigma, ustar, kind=O.DL):
    u = O.apply(O.LAPLACE, kind, 0.0, tgt.coords, None, coords, normals, weights, sigma)
    return 0.5 * np.sum((u - ustar) ** 2)


@pytest.mark.parametrize("kind,okind", [(inti.DoubleLayerKernel, O.DL), (inti.SingleLayerKernel, O.SL)])
def test_gradients_match_finite_differences(ctx, kind, okind):
    q, tgt, op, sigma, ustar = setup(ctx, kind)
    u = op @ sigma
    grad = op.grad_sources(u - ustar, sigma)
    r = np.random.default_rng(5)
    h = 1e-6
    for name in ("sigma", "coords", "normals", "weights"):
        if okind == O.SL and name == "normals":
            assert np.all(grad[name] == 0)
            continue
        base = {"coords": q.coords, "normals": q.normals, "weights": q.weights, "sigma": sigma}
        v = r.standard_normal(base[name].shape)
        plus = dict(base)
        minus = dict(base)
        plus[name] = base[name] + h * v
        minus[name] = base[name] - h * v
        fd = (J(tgt, plus["coords"], plus["normals"], plus["weights"], plus["sigma"], ustar, okind)
              - J(tgt, minus["coords"], minus["normals"], minus["weights"], minus["sigma"], ustar, okind)) / (2 * h)
        ad = float(np.sum(grad[name] * v))
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-8), (name, ad, fd)


def test_gradient_matches_dual_numbers(ctx):
    q, tgt, op, sigma, ustar = setup(ctx)
    u = op @ sigma
    g = u - ustar
    grad = op.grad_sources(g, sigma)
    r = np.random.default_rng(6)
    dsx, dsn, dsw, dsg = (r.standard_normal(q.coords.shape), r.standard_normal(q.normals.shape),
                          r.standard_normal(len(q)), r.standard_normal(len(q)))
    _, du = O.dl_potential_jvp(tgt.coords, q.coords, q.normals, q.weights, sigma, dsx, dsn, dsw, dsg)
    jvp = float(np.dot(g, du))
    ad = float(np.sum(grad["coords"] * dsx) + np.sum(grad["normals"] * dsn) + np.sum(grad["weights"] * dsw)
               + np.sum(grad["sigma"] * dsg))
    assert abs(ad - jvp) <= 1e-10 * max(abs(jvp), 1.0)


def test_density_gradient_is_transpose_apply(ctx):
    q, tgt, op, sigma, ustar = setup(ctx)
    g = density(len(tgt), False, 9)
    assert relerr(op.grad_sources(g, sigma)["sigma"], op.rmatvec(g)) < 1e-13


def test_device_gradients_match_host(ctx):
    import torch

    q, tgt, op, sigma, ustar = setup(ctx)
    g = density(len(tgt), False, 9)
    ref = op.grad_sources(g, sigma)
    dev = torch.device("cuda:0")
    n = len(q)
    gd, sd = torch.from_numpy(g).to(dev), torch.from_numpy(sigma).to(dev)
    outs = {k: torch.full((s,), np.nan, dtype=torch.float64, device=dev)
            for k, s in (("sigma", n), ("coords", 3 * n), ("normals", 3 * n), ("weights", n))}
    torch.cuda.synchronize()
    op.grad_sources_device(gd.data_ptr(), sd.data_ptr(), outs["sigma"].data_ptr(), outs["coords"].data_ptr(),
                           outs["normals"].data_ptr(), outs["weights"].data_ptr())
    ctx.synchronize()
    for k, v in outs.items():
        assert np.array_equal(v.cpu().numpy().reshape(ref[k].shape), ref[k]), k
    # a zero output pointer skips that gradient
    outs["weights"].fill_(np.nan)
    torch.cuda.synchronize()
    op.grad_sources_device(gd.data_ptr(), sd.data_ptr(), outs["sigma"].data_ptr(), 0, 0, 0)
    ctx.synchronize()
    assert torch.isnan(outs["weights"]).all()


@pytest.mark.parametrize("dim", [3, 2])
@pytest.mark.parametrize("kind,okind", [(inti.DoubleLayerKernel, O.DL), (inti.SingleLayerKernel, O.SL)])
def test_gradients_many_source_blocks(ctx, dim, kind, okind):
    """Sources over many thread blocks (two sources per thread, the last
    block ragged) and targets over several chunks, in 3D and 2D: dJ/dsigma
    against the transpose apply, the geometry gradients against central
    differences."""
    if dim == 3:
        q = inti.ellipsoid_quadrature(8, 5)  # 3,456 sources
        d = np.random.default_rng(7).standard_normal((300, 3))
        tgt = inti.points(1.6 * d / np.linalg.norm(d, axis=1, keepdims=True))
    else:
        q = inti.kite_quadrature(200, 9)  # 1,000 sources
        t = np.linspace(0, 2 * np.pi, 300, endpoint=False)
        tgt = inti.points(np.stack([3.0 * np.cos(t), 3.0 * np.sin(t)], axis=1))
    op = inti.GpuOperator(kind(inti.Laplace(dim=dim)), tgt, q, ctx=ctx)
    sigma = density(len(q), False, 12)
    ustar = density(len(tgt), False, 13) * 0.01
    g = op @ sigma - ustar
    grad = op.grad_sources(g, sigma)
    assert relerr(grad["sigma"], op.rmatvec(g)) < 1e-13
    r = np.random.default_rng(14)
    h = 1e-6
    base = {"coords": q.coords, "normals": q.normals, "weights": q.weights, "sigma": sigma}

    def Jd(p):
        u = O.apply(O.LAPLACE, okind, 0.0, tgt.coords, None, p["coords"], p["normals"], p["weights"], p["sigma"])
        return 0.5 * np.sum((u - ustar) ** 2)

    for name in ("coords", "normals", "weights"):
        if okind == O.SL and name == "normals":
            assert np.all(grad[name] == 0)
            continue
        v = r.standard_normal(base[name].shape)
        fd = (Jd(dict(base, **{name: base[name] + h * v})) - Jd(dict(base, **{name: base[name] - h * v}))) / (2 * h)
        ad = float(np.sum(grad[name] * v))
        assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-8), (name, ad, fd)
