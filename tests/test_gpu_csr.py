"""Standalone correction SpMV y = alpha*C*x + beta*y (inti_csr_apply), the
replacement of SparseMatrixCSC * Vector in LinearMap(S) + LinearMap(δS)
(src/api.jl:179-184), against scipy's product of the same arrays, over the
row-length regimes the kernel distinguishes: DIM element blocks, ragged rows
with empty ones, a row block that overflows the shared-memory buffer, and
long rows."""
import numpy as np
import pytest
import scipy.sparse as sp

import inti_b200 as inti

pytestmark = pytest.mark.gpu


def pattern(kind, r):
    if kind == "dim9":  # element blocks of 9 (C3's DIM pattern)
        m = 9 * 2000
        rp = np.arange(0, 9 * m + 1, 9)
        col = ((np.arange(m) // 9 * 9)[:, None] + np.arange(9)).ravel()
        return m, m, rp, col
    if kind == "ragged":  # 0..20 per row, with empty rows
        m, n = 7001, 5000
        lens = r.integers(0, 21, m)
        lens[r.integers(0, m, 300)] = 0
    elif kind == "overflow":  # mean 6, a few rows of several thousand
        m, n = 4000, 9000
        lens = r.integers(0, 13, m)
        lens[[5, 1234, 3999]] = [5000, 8000, 2500]
    else:  # "long": mean 100
        m, n = 1500, 4000
        lens = r.integers(50, 151, m)
    rp = np.concatenate([[0], np.cumsum(lens)])
    col = np.concatenate([np.sort(r.choice(n, int(k), replace=False)) for k in lens]) if rp[-1] else np.zeros(0, int)
    return m, n, rp, col


@pytest.mark.parametrize("kind", ["dim9", "ragged", "overflow", "long"])
@pytest.mark.parametrize("cplx", [False, True])
def test_csr_apply_matches_scipy(ctx, kind, cplx):
    import torch

    r = np.random.default_rng(["dim9", "ragged", "overflow", "long"].index(kind) * 2 + int(cplx))
    m, n, rp, col = pattern(kind, r)
    nnz = int(rp[-1])
    val = r.standard_normal(nnz) + (1j * r.standard_normal(nnz) if cplx else 0)
    x = r.standard_normal(n) + (1j * r.standard_normal(n) if cplx else 0)
    y0 = r.standard_normal(m) + (1j * r.standard_normal(m) if cplx else 0)
    Cm = inti.CorrectionMatrix.from_csr(rp, col, val, (m, n), ctx)
    ref_mat = sp.csr_matrix((val, col, rp), shape=(m, n))
    # host entry point, alpha = 1, beta = 0
    y = Cm @ x
    ref = ref_mat @ x
    scale = np.abs(ref_mat) @ np.abs(x) + 1e-300
    assert np.max(np.abs(y - ref) / scale) < 1e-14
    # device entry point with alpha, beta
    alpha, beta = (0.75 - 0.5j, 1.5 + 0.25j) if cplx else (0.75, -1.5)
    dev = torch.device("cuda:0")
    xd = torch.from_numpy(np.ascontiguousarray(x).view(np.float64).copy()).to(dev)
    yd = torch.from_numpy(np.ascontiguousarray(y0).view(np.float64).copy()).to(dev)
    torch.cuda.synchronize()
    Cm.apply_device(xd.data_ptr(), yd.data_ptr(), alpha, beta)
    ctx.synchronize()
    got = yd.cpu().numpy()
    got = got.view(np.complex128) if cplx else got
    want = alpha * ref + beta * y0
    assert np.max(np.abs(got - want) / (abs(alpha) * scale + abs(beta) * np.abs(y0) + 1e-300)) < 1e-14
    # deterministic: the same call twice gives the same bits
    yd2 = torch.from_numpy(np.ascontiguousarray(y0).view(np.float64).copy()).to(dev)
    torch.cuda.synchronize()
    Cm.apply_device(xd.data_ptr(), yd2.data_ptr(), alpha, beta)
    ctx.synchronize()
    assert torch.equal(yd, yd2)
