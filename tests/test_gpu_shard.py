"""Row-sharded operators (the multi-GPU split of one product) on one GPU:
the row blocks of (A + δ)σ built with inti_b200.shard, applied one after
another, reproduce the full product (only the partial-sum grouping differs)."""
import numpy as np
import pytest

import inti_b200 as inti
from helpers import density, relerr
from inti_b200 import geometry as G
from inti_b200 import shard as SH

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["kite_laplace_dl", "sphere_helmholtz_sl"])
@pytest.mark.parametrize("world", [2, 3, 8])
def test_row_blocks_reproduce_full_product(ctx, case, world):
    if case == "kite_laplace_dl":
        q, op, kern = G.kite_quadrature(60, 9), inti.Laplace(dim=2), inti.DoubleLayerKernel
    else:
        q, op, kern = G.p2_sphere_quadrature(4), inti.Helmholtz(k=10.0, dim=3), inti.SingleLayerKernel
    dS, dD = inti.bdim_correction(op, q, q, ctx=ctx)
    corr = dD if kern is inti.DoubleLayerKernel else dS
    A = inti.GpuOperator(kern(op), q, q, corr, "fp64", ctx)
    sigma = density(len(q), A.is_complex, 4)
    full = A @ sigma
    ip, ix, dv = corr.arrays()
    parts = []
    for r0, r1 in SH.row_blocks(len(q), world):
        c = inti.CorrectionMatrix.from_csr(*SH.slice_csr_rows(ip, ix, dv, r0, r1), (r1 - r0, len(q)), ctx=ctx)
        Ab = inti.GpuOperator(kern(op), SH.target_block(q, r0, r1), q, c, "fp64", ctx)
        parts.append(Ab @ sigma)
    assert relerr(np.concatenate(parts), full) < 1e-13


@pytest.mark.parametrize("pde", ["helmholtz", "laplace", "laplace2d"])
@pytest.mark.parametrize("kname", ["DL", "HS"])
@pytest.mark.parametrize("world", [2, 3])
def test_item_shards_sum_to_the_full_product(ctx, pde, kname, world):
    """Item shards of a symmetric operator (inti_op_set_shard): the ranks'
    partial products over all rows, summed (the all-reduce of one process
    per GPU), give alpha*(A + C)x + beta*y; rank 0 carries C and beta*y.
    Double layer and hypersingular kernel, 3D and 2D."""
    if pde == "laplace2d":
        q, op = G.kite_quadrature(700, 9), inti.Laplace(dim=2)  # 3,500 nodes
    else:
        q = G.ellipsoid_quadrature(8, 5)  # 3,456 nodes: several node blocks
        op = inti.Helmholtz(k=6.0, dim=3) if pde == "helmholtz" else inti.Laplace(dim=3)
    hs = kname == "HS"
    dS, dD = inti.bdim_correction(op, q, q, derivative=hs, ctx=ctx)
    K = inti.HyperSingularKernel if hs else inti.DoubleLayerKernel
    A = inti.GpuOperator(K(op), q, q, dD, "fp64", ctx)
    assert A.tuning["symmetric"]
    cplx = A.is_complex
    x, y0 = density(len(q), cplx, 11), density(len(q), cplx, 12)
    alpha, beta = (0.5 - 0.25j, 2.0 + 1.0j) if cplx else (0.5, 2.0)
    full = A.mul(y0.copy(), x, alpha=alpha, beta=beta)
    total = np.zeros_like(full)
    for r in range(world):
        A.set_shard(r, world)
        total += A.mul(y0.copy(), x, alpha=alpha, beta=beta)
    A.set_shard(0, 1)
    assert relerr(total, full) < 1e-13
    assert relerr(A.mul(y0.copy(), x, alpha=alpha, beta=beta), full) < 1e-15  # whole again


def test_item_shards_are_refused_where_they_do_not_apply(ctx):
    q = G.ellipsoid_quadrature(4, 5)
    op = inti.Laplace(dim=3)
    T = inti.points(1.5 * q.coords[::3])
    B = inti.GpuOperator(inti.SingleLayerKernel(op), T, q, None, "fp64", ctx)  # not square: no symmetric form
    with pytest.raises(inti.UnsupportedError):
        B.set_shard(0, 2)
    A = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", ctx)
    with pytest.raises(inti.ArgumentError):
        A.set_shard(2, 2)
    A.set_shard(1, 2)
    with pytest.raises(inti.UnsupportedError):
        A.rmatvec(np.ones(len(q)))
    with pytest.raises(inti.ArgumentError):  # INTI_E_STATE: GMRES takes whole operators
        inti.gmres(0.5 * inti.I + A, np.ones(len(q)), rtol=1e-8)
