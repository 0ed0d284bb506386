"""GPU BDIM correction versus the oracle: the sparsity pattern and indexing
bit-exact, values within a stated relative tolerance (the least-squares
problems are solved by the same Householder algorithm in both, so the values
agree to a small multiple of cond(M)·eps)."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, oracle_dim_csr, relerr, small_surfaces

pytestmark = pytest.mark.gpu

SURF = small_surfaces()
VAL_TOL = 1e-8


def _compare(pde, k, q, gpu_pair, derivative=False, elements=None):
    ref = oracle_dim_csr(pde, k, q, derivative=derivative, elements=elements)
    for g, r in zip(gpu_pair, ref):
        rp, col, val = g.arrays()
        if elements is None:
            assert np.array_equal(rp, r[0]) and np.array_equal(col, r[1])
            assert relerr(val, r[2]) < VAL_TOL
        else:
            nq = q.nq
            rows = (np.asarray(elements)[:, None] * nq + np.arange(nq)).reshape(-1)
            sel = np.concatenate([np.arange(rp[i], rp[i + 1]) for i in rows])
            gv = val[sel]
            rv = np.concatenate([r[2][r[0][i]:r[0][i + 1]] for i in rows])
            assert np.array_equal(col[sel], np.concatenate([r[1][r[0][i]:r[0][i + 1]] for i in rows]))
            assert relerr(gv, rv) < VAL_TOL


@pytest.mark.parametrize("surf", list(SURF))
@pytest.mark.parametrize("derivative", [False, True])
def test_dim_matches_oracle(ctx, surf, derivative):
    q = SURF[surf]
    ops = [(inti.Laplace(dim=q.dim), O.LAPLACE, 0.0)]
    if q.dim == 3:
        ops.append((inti.Helmholtz(k=2.5, dim=3), O.HELMHOLTZ, 2.5))
    for op, pde, k in ops:
        pair = inti.bdim_correction(op, q, q, derivative=derivative, ctx=ctx)
        _compare(pde, k, q, pair, derivative)


def test_dim_kite_workload(ctx):
    """2D Laplace double layer on the kite, 200 GL-5 panels (N = 1000):
    dense product + correction SpMV against the oracle's."""
    q = inti.kite_quadrature()
    op = inti.Laplace(dim=2)
    S, D = inti.single_double_layer(op=op, target=q, source=q, compression={"method": "none"},
                                    correction={"method": "dim"}, ctx=ctx)
    sigma = density(len(q), False, 1)
    dS, dD = oracle_dim_csr(O.LAPLACE, 0.0, q)
    ref = oracle_apply(O.LAPLACE, O.DL, 0.0, q, q, sigma) + O.csr_apply(*dD, sigma)
    assert relerr(D @ sigma, ref) < 1e-11
    rp, col, _ = D.correction.arrays()
    assert np.array_equal(rp, dD[0]) and np.array_equal(col, dD[1])
    assert D.correction.nnz == 5000


def test_green_multiplier_vector(ctx):
    q = SURF["ellipsoid"]
    gm = np.linspace(-1.0, 0.0, len(q))
    pair = inti.bdim_correction(inti.Laplace(dim=3), q, q, green_multiplier=gm, ctx=ctx)
    ref = oracle_dim_csr(O.LAPLACE, 0.0, q, green_multiplier=gm)
    for g, r in zip(pair, ref):
        assert relerr(g.arrays()[2], r[2]) < VAL_TOL


def test_gauss_law_and_green_identity_on_gpu(ctx):
    """D[1] = -1/2 and Green's identity < 1e-2 (test/green_identities_test.jl)."""
    q = inti.ellipsoid_quadrature(3, 5, (1.0, 1.0, 1.0))
    op = inti.Laplace(dim=3)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    assert np.max(np.abs(D @ np.ones(len(q)) + 0.5)) < 1e-2
    xs = np.array([3.0, 3.0, 3.0])
    r = q.coords - xs
    d = np.linalg.norm(r, axis=1)
    g0 = 1 / (4 * np.pi * d)
    g1 = -np.sum(r * q.normals, 1) / (4 * np.pi * d**3)
    e1 = np.max(np.abs(S @ g1 - D @ g0 - 0.5 * g0)) / np.max(np.abs(g0))
    assert e1 < 1e-2
