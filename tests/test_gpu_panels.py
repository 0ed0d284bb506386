"""Symmetric operators whose partial sums exceed the partial budget run their
work items in panels of source blocks (one launch per panel, the partials
of one panel at a time folded into running sums), so memory stays O(N) plus
the budget.  A small budget forces panels on small problems: the paneled
product equals the one-launch product to rounding (only the order of the
partial sums differs) and the oracle's sampled rows; transposes, the fused
correction with alpha/beta, item shards and the paired-FP32 kernel too."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import KIND, PDE, density, oracle_apply, relerr

pytestmark = pytest.mark.gpu

KERNELS = {"SL": inti.SingleLayerKernel, "DL": inti.DoubleLayerKernel, "ADL": inti.AdjointDoubleLayerKernel,
           "HS": inti.HyperSingularKernel}
CASES = [
    ("helmholtz", "SL", "fp64"), ("helmholtz", "DL", "fp64"), ("helmholtz", "HS", "fp64"),
    ("helmholtz", "SL", "fp32c"), ("laplace", "DL", "fp64"), ("laplace", "ADL", "fp64"),
    ("laplace", "DL", "fp32c"), ("laplace", "SL", "fp32c"), ("laplace2d", "DL", "fp64"),
]


def _surface(pde):
    if pde == "laplace2d":
        return inti.kite_quadrature(800, 9), inti.Laplace(dim=2), 0.0  # 4,000 nodes
    if pde == "helmholtz":
        return inti.p2_sphere_quadrature(12), inti.Helmholtz(k=8.0, dim=3), 8.0  # 6,912 nodes
    return inti.ellipsoid_quadrature(10, 5), inti.Laplace(dim=3), 0.0  # 5,400 nodes


def _paneled(ctx, make):
    """The operator built by make() with the default budget and with a budget
    small enough for several panels."""
    one = make()
    ctx.set_partial_budget(2.5e5)
    try:
        pan = make()
    finally:
        ctx.set_partial_budget(0)
    assert one.tuning["symmetric"] and one.tuning["panels"] == 1
    assert pan.tuning["symmetric"] and pan.tuning["panels"] > 2, pan.tuning
    return one, pan


@pytest.mark.parametrize("pde,kname,prec", CASES)
def test_panels_match_one_launch_and_oracle(ctx, pde, kname, prec):
    q, op, k = _surface(pde)
    K = KERNELS[kname](op)
    one, pan = _paneled(ctx, lambda: inti.GpuOperator(K, q, q, None, prec, ctx))
    sigma = density(len(q), one.is_complex, 3)
    y1, yp = one @ sigma, pan @ sigma
    fp64 = prec == "fp64"
    assert relerr(yp, y1) < (1e-13 if fp64 else 1e-6)
    rows = np.random.default_rng(4).choice(len(q), 24, replace=False)
    ref = oracle_apply(PDE["laplace" if pde == "laplace2d" else pde], KIND[kname], k, q, q, sigma, rows=rows)
    assert relerr(yp[rows], ref) < (1e-12 if fp64 else 5e-5)
    # the transpose runs on the same panels
    g = density(len(q), one.is_complex, 5)
    assert relerr(pan.rmatvec(g), one.rmatvec(g)) < (1e-13 if fp64 else 1e-6)


@pytest.mark.parametrize("pde", ["helmholtz", "laplace"])
def test_panels_with_correction_alpha_beta_and_shards(ctx, pde):
    q, op, k = _surface(pde)
    dS, dD = inti.bdim_correction(op, q, q, ctx=ctx)
    one, pan = _paneled(ctx, lambda: inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, dD, "fp64", ctx))
    cplx = one.is_complex
    x, y0 = density(len(q), cplx, 11), density(len(q), cplx, 12)
    alpha, beta = (0.5 - 0.25j, 2.0 + 1.0j) if cplx else (0.5, 2.0)
    full = one.mul(y0.copy(), x, alpha=alpha, beta=beta)
    assert relerr(pan.mul(y0.copy(), x, alpha=alpha, beta=beta), full) < 1e-13
    # item shards of the paneled operator, summed (the all-reduce of one process per GPU)
    total = np.zeros_like(full)
    for r in range(3):
        pan.set_shard(r, 3)
        total += pan.mul(y0.copy(), x, alpha=alpha, beta=beta)
    pan.set_shard(0, 1)
    assert relerr(total, full) < 1e-13
    assert relerr(pan.mul(y0.copy(), x, alpha=alpha, beta=beta), full) < 1e-13


def test_partial_budget_rejects_negative(ctx):
    with pytest.raises(inti.ArgumentError):
        ctx.set_partial_budget(-1.0)


def test_symmetric_operators_share_the_context_scratch(ctx):
    """The symmetric form's partials belong to the context and are shared by
    its operators: applies of different operators enqueued back to back on
    the context's stream (no synchronisation in between), one of them in
    panels, give the products each operator gives alone."""
    import torch

    q, op, k = _surface("helmholtz")
    A = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", ctx)
    ctx.set_partial_budget(2.5e5)
    try:
        B = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, None, "fp64", ctx)
    finally:
        ctx.set_partial_budget(0)
    assert A.tuning["panels"] == 1 and B.tuning["panels"] > 2
    sigma = density(len(q), True, 21)
    ya, yb = A @ sigma, B @ sigma
    dev = torch.device("cuda:0")
    xs = torch.from_numpy(np.ascontiguousarray(sigma).view(np.float64).copy()).to(dev)
    outs = [torch.zeros_like(xs) for _ in range(4)]
    torch.cuda.synchronize()
    for i, M in enumerate((A, B, A, B)):
        M.apply_device(xs.data_ptr(), outs[i].data_ptr())
    ctx.synchronize()
    got = [o.cpu().numpy().view(np.complex128) for o in outs]
    assert np.array_equal(got[0], ya) and np.array_equal(got[2], ya)
    assert np.array_equal(got[1], yb) and np.array_equal(got[3], yb)
