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
