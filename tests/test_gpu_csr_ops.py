"""Device set-up of sparse corrections: the union merge of two corrections
with different patterns (the fused combined-field operator's c1·δD + c2·δS)
and the transpose used by transposed applies, checked through the operators
against scipy's sums and transposes of the same arrays."""
import numpy as np
import pytest
import scipy.sparse as sp

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, relerr

pytestmark = pytest.mark.gpu


def _random_csr(m, n, per_row, cplx, seed):
    r = np.random.default_rng(seed)
    rows = []
    for i in range(m):
        k = r.integers(0, per_row + 1)  # some rows empty
        rows.append(np.sort(r.choice(n, size=k, replace=False)))
    indptr = np.zeros(m + 1, np.int64)
    indptr[1:] = np.cumsum([len(c) for c in rows])
    indices = np.concatenate(rows).astype(np.int32) if indptr[-1] else np.zeros(0, np.int32)
    data = r.standard_normal(len(indices))
    if cplx:
        data = data + 1j * r.standard_normal(len(indices))
    return indptr, indices, data


@pytest.mark.parametrize("pde", ["laplace", "helmholtz"])
def test_merge_of_different_patterns(ctx, pde):
    q = inti.ellipsoid_quadrature(4, 5)  # 864 nodes
    n = len(q)
    cplx = pde == "helmholtz"
    op = inti.Helmholtz(k=3.0, dim=3) if cplx else inti.Laplace(dim=3)
    k = 3.0 if cplx else 0.0
    P = O.HELMHOLTZ if cplx else O.LAPLACE
    a = _random_csr(n, n, 7, cplx, 1)
    b = _random_csr(n, n, 5, cplx, 2)
    CA = inti.CorrectionMatrix.from_csr(*a, (n, n), ctx=ctx)
    CB = inti.CorrectionMatrix.from_csr(*b, (n, n), ctx=ctx)
    D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, CA, "fp64", ctx)
    S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, CB, "fp64", ctx)
    c1, c2 = (1.0, -2.5j) if cplx else (0.75, 1.5)
    CF = inti.CombinedFieldOperator(D, S, c1, c2)
    x = density(n, cplx, 3)
    sA = sp.csr_matrix((a[2], a[1], a[0]), shape=(n, n))
    sB = sp.csr_matrix((b[2], b[1], b[0]), shape=(n, n))
    want = c1 * (oracle_apply(P, O.DL, k, q, q, x) + sA @ x) + c2 * (oracle_apply(P, O.SL, k, q, q, x) + sB @ x)
    assert relerr(CF @ x, want) < 1e-12
    # one side without a correction
    D0 = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, None, "fp64", ctx)
    CF0 = inti.CombinedFieldOperator(D0, S, c1, c2)
    want0 = c1 * oracle_apply(P, O.DL, k, q, q, x) + c2 * (oracle_apply(P, O.SL, k, q, q, x) + sB @ x)
    assert relerr(CF0 @ x, want0) < 1e-12


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("square", [True, False])
def test_transpose_of_random_correction(ctx, cplx, square):
    q = inti.ellipsoid_quadrature(4, 5)
    n = len(q)
    tgt = q if square else inti.points(1.5 * q.coords[::2])
    m = len(tgt)
    op = inti.Helmholtz(k=2.0, dim=3) if cplx else inti.Laplace(dim=3)
    k = 2.0 if cplx else 0.0
    P = O.HELMHOLTZ if cplx else O.LAPLACE
    c = _random_csr(m, n, 9, cplx, 7)
    C = inti.CorrectionMatrix.from_csr(*c, (m, n), ctx=ctx)
    A = inti.GpuOperator(inti.SingleLayerKernel(op), tgt, q, C, "fp64", ctx)
    dense = O.assemble(P, O.SL, k, tgt.coords, None, q.coords, q.normals, q.weights) + \
        sp.csr_matrix((c[2], c[1], c[0]), shape=(m, n)).toarray()
    g = density(m, cplx, 8)
    got = A.rmatvec(g)
    assert relerr(got, dense.T @ g) < 1e-12
    assert np.array_equal(got, A.rmatvec(g))
