"""Volume potential with the VDIM correction (src/api.jl:282-378,
src/vdim.jl:30-130), Laplace on the unit disk (2D) and the unit ball (3D),
Helmholtz in the unit ball,
through the public API: the GPU path (boundary layer operators with their
off-surface DIM, plain volume potential, fused δV) against the closed forms
V[1] = (1 - r^2)/4, V[r^2] = (1 - r^4)/16 (disk), V[1] = (3 - r^2)/6,
V[r^2] = 1/4 - r^4/20 (ball) and against the oracle's restatement."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from inti_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _case():
    return G.disk_triangle_quadrature(4), G.circle_quadrature(64, 8)


@pytest.mark.parametrize("order", [2, 4])
def test_vdim_known_answers_and_oracle(ctx, order):
    Y, B = _case()
    op = inti.Laplace(dim=2)
    V = inti.volume_potential(op=op, target=Y, source=Y, ctx=ctx,
                              correction={"method": "dim", "boundary": B, "interpolation_order": order})
    V0 = inti.volume_potential(op=op, target=Y, source=Y, correction={"method": "none"}, ctx=ctx)
    near, vals = O.vdim(Y.coords, Y.coords, Y.weights, Y.nq, B.coords, B.normals, B.weights, B.nq, -1.0, order,
                        same=True)
    ip, ix, dv = O.targets_csr(near, vals, Y.nq, len(Y))
    rp, col, val = V.correction.arrays()
    assert np.array_equal(rp, ip) and np.array_equal(col, ix)  # pattern: each element's own nodes
    r2 = (Y.coords ** 2).sum(1)
    for f, exact in ((np.ones(len(Y)), (1 - r2) / 4), (r2, (1 - r2 ** 2) / 16)):
        got, naive = V @ f, V0 @ f
        assert np.max(np.abs(got - exact)) < 1e-6 < np.max(np.abs(naive - exact))
        ref = O.apply(O.LAPLACE, O.SL, 0.0, Y.coords, None, Y.coords, None, Y.weights, f) + O.csr_apply(ip, ix, dv, f)
        assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref))


def test_vdim_ball_known_answers_and_oracle(ctx):
    Y = G.ball_hex_quadrature(2)
    B = G.ellipsoid_quadrature(16, 5, scaling=(1.0, 1.0, 1.0))
    op = inti.Laplace(dim=3)
    V = inti.volume_potential(op=op, target=Y, source=Y, ctx=ctx,
                              correction={"method": "dim", "boundary": B, "interpolation_order": 2})
    V0 = inti.volume_potential(op=op, target=Y, source=Y, correction={"method": "none"}, ctx=ctx)
    near, vals = O.vdim(Y.coords, Y.coords, Y.weights, Y.nq, B.coords, B.normals, B.weights, B.nq, -1.0, 2,
                        same=True)
    ip, ix, dv = O.targets_csr(near, vals, Y.nq, len(Y))
    rp, col, val = V.correction.arrays()
    assert np.array_equal(rp, ip) and np.array_equal(col, ix)
    r2 = (Y.coords ** 2).sum(1)
    for f, exact in ((np.ones(len(Y)), (3 - r2) / 6), (r2, 0.25 - r2 ** 2 / 20)):
        got, naive = V @ f, V0 @ f
        assert np.max(np.abs(got - exact)) < 1e-6 < np.max(np.abs(naive - exact))
        ref = O.apply(O.LAPLACE, O.SL, 0.0, Y.coords, None, Y.coords, None, Y.weights, f) + O.csr_apply(ip, ix, dv, f)
        assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref))


@pytest.mark.parametrize("k", [2.0, 4.0])
def test_vdim_ball_helmholtz_known_answer_and_oracle(ctx, k):
    """3D Helmholtz: the polynomial solutions of ΔP + k²P = p are unique, so
    they are the reference's (src/vdim.jl:369-373); V[1] = -1/k² + (1 - ik)
    e^{ik} sin(kr)/(k³ r) in the unit ball."""
    Y = G.ball_hex_quadrature(2)
    B = G.ellipsoid_quadrature(16, 5, scaling=(1.0, 1.0, 1.0))
    op = inti.Helmholtz(k=k, dim=3)
    V = inti.volume_potential(op=op, target=Y, source=Y, ctx=ctx,
                              correction={"method": "dim", "boundary": B, "interpolation_order": 2})
    V0 = inti.volume_potential(op=op, target=Y, source=Y, correction={"method": "none"}, ctx=ctx)
    near, vals = O.vdim(Y.coords, Y.coords, Y.weights, Y.nq, B.coords, B.normals, B.weights, B.nq, -1.0, 2,
                        same=True, pde=O.HELMHOLTZ, k=k)
    ip, ix, dv = O.targets_csr(near, vals, Y.nq, len(Y))
    rp, col, val = V.correction.arrays()
    assert np.array_equal(rp, ip) and np.array_equal(col, ix)
    r = np.sqrt((Y.coords ** 2).sum(1))
    exact = -1 / k ** 2 + (1 - 1j * k) * np.exp(1j * k) * np.sin(k * r) / (k ** 3 * r)
    f = np.ones(len(Y))
    got, naive = V @ f, V0 @ f
    assert np.max(np.abs(got - exact)) < 1e-6 < np.max(np.abs(naive - exact))
    ref = O.apply(O.HELMHOLTZ, O.SL, k, Y.coords, None, Y.coords, None, Y.weights, f) + O.csr_apply(ip, ix, dv, f)
    assert np.max(np.abs(got - ref)) <= 1e-9 * np.max(np.abs(ref))


def test_volume_potential_argument_errors(ctx):
    Y, B = _case()
    op = inti.Laplace(dim=2)
    with pytest.raises(inti.ArgumentError):  # the boundary is required for the DIM correction
        inti.volume_potential(op=op, target=Y, source=Y, correction={"method": "dim"}, ctx=ctx)
    with pytest.raises(inti.UnsupportedError):  # 2D Helmholtz (Hankel kernels) is not built
        inti.polynomial_solutions_vdim(inti.Helmholtz(k=1.0, dim=2), 2)
