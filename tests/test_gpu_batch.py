"""Batched multi-surface, multi-RHS operators (one launch over uneven star
surfaces).  FP64 batch against the single-surface operators (themselves
checked against the oracle); the TF32 tensor-core batch (tcgen05) against the
FP64 batch at TF32 accuracy."""
import numpy as np
import pytest

import inti_b200 as inti
from helpers import relerr

pytestmark = pytest.mark.gpu


def stars(ns=(3, 2, 4), seed=0):
    r = np.random.default_rng(seed)
    return [inti.star_quadrature(inti.star_coefficients(r), n) for n in ns]


def rhs(n, nrhs, cplx, seed=1):
    r = np.random.default_rng(seed)
    X = r.standard_normal((n, nrhs))
    if cplx:
        X = X + 1j * r.standard_normal((n, nrhs))
    return X


def per_surface(op, quads, kind, corrs, X, cD=1.0, cS=1.0, ctx=None):
    out = []
    off = 0
    for q, (dS, dD) in zip(quads, corrs):
        n = len(q)
        Xs = X[off:off + n]
        if kind == "SL":
            A = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, dS, ctx=ctx)
        elif kind == "DL":
            A = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, dD, ctx=ctx)
        else:
            D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, dD, ctx=ctx)
            S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, dS, ctx=ctx)
            A = inti.CombinedFieldOperator(D, S, cD, cS)
        out.append(A @ Xs)
        off += n
    return np.concatenate(out, axis=0)


@pytest.mark.parametrize("kind", ["SL", "DL", "CF"])
@pytest.mark.parametrize("pde", ["helmholtz", "laplace"])
@pytest.mark.parametrize("nrhs", [5, 70])
def test_batch_fp64_matches_single_surface_operators(ctx, kind, pde, nrhs):
    """70 columns: two 64-column groups, the second ragged."""
    quads = stars()
    op = inti.Helmholtz(k=5.0, dim=3) if pde == "helmholtz" else inti.Laplace(dim=3)
    corrs = [inti.bdim_correction(op, q, q, ctx=ctx) for q in quads]
    cD, cS = (1.0, -5.0j) if pde == "helmholtz" else (1.0, 0.5)
    B = inti.BatchOperator(op, quads, kind, corrs, cD, cS, ctx=ctx)
    X = rhs(B.n, nrhs, pde == "helmholtz")
    ref = per_surface(op, quads, kind, corrs, X, cD, cS, ctx)
    assert relerr(B.apply(X), ref) < 1e-12
    # alpha / beta
    Y0 = rhs(B.n, nrhs, pde == "helmholtz", 9)
    got = B.apply(X, Y=Y0, alpha=0.5, beta=2.0)
    assert relerr(got, 0.5 * ref + 2.0 * Y0) < 1e-12


@pytest.mark.parametrize("kind", ["SL", "DL", "CF", "CF_general"])
@pytest.mark.parametrize("nrhs", [5, 64, 70])
def test_batch_tf32_tensor_cores_match_fp64(ctx, kind, nrhs):
    quads = stars((4, 3, 6, 2), seed=3)
    op = inti.Helmholtz(k=5.0, dim=3)
    corrs = [inti.bdim_correction(op, q, q, ctx=ctx) for q in quads]
    # D - 5i S takes the Brakhage-Werner kernel variant; other couplings the general one
    cD, cS = (0.7 + 0.2j, 0.3 - 2.0j) if kind == "CF_general" else (1.0, -5.0j)
    B = inti.BatchOperator(op, quads, kind[:2], corrs, cD, cS, ctx=ctx)
    X = rhs(B.n, nrhs, True, 4)
    y64 = B.apply(X, "fp64")
    y32 = B.apply(X, "tf32")
    # TF32 inputs (11-bit significands), FP32 accumulation
    for c in range(nrhs):
        assert relerr(y32[:, c], y64[:, c]) < 5e-3, c


def test_batch_tf32_second_call_and_beta(ctx):
    quads = stars((3, 5), seed=5)
    op = inti.Helmholtz(k=5.0, dim=3)
    B = inti.BatchOperator(op, quads, "SL", None, ctx=ctx)
    X1, X2 = rhs(B.n, 8, True, 1), rhs(B.n, 8, True, 2)
    Y0 = rhs(B.n, 8, True, 3)
    a = B.apply(X1, "tf32")
    b = B.apply(X2, "tf32", Y=Y0, alpha=1.5, beta=-1.0)
    assert relerr(a, B.apply(X1)) < 5e-3
    assert relerr(b, 1.5 * B.apply(X2) - Y0) < 5e-3


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_gmres_cfie(ctx, mode):
    """I/2 + D - i k S on each surface, every column, one lockstep solve;
    each system's FP64 residual <= 1e-10, and the solutions agree with
    one-surface solves."""
    quads = stars((3, 2, 4), seed=7)
    k = 3.0
    op = inti.Helmholtz(k=k, dim=3)
    corrs = [inti.bdim_correction(op, q, q, ctx=ctx) for q in quads]
    B = inti.BatchOperator(op, quads, "CF", corrs, 1.0, -1j * k, ctx=ctx)
    R = 4
    rhs_ = rhs(B.n, R, True, 11)
    X, st = B.gmres(rhs_, shift=0.5, rtol=1e-10, restart=30, maxiter=300, mode=mode)
    assert st["converged"] == 1, st
    assert np.max(st["relres_all"]) <= 1e-10
    # independent FP64 check of the residual with the FP64 batch operator
    res = rhs_ - (0.5 * X + B.apply(X, "fp64"))
    off = B.offsets
    for s in range(len(quads)):
        for c in range(R):
            seg = slice(off[s], off[s + 1])
            assert np.linalg.norm(res[seg, c]) <= 2e-10 * np.linalg.norm(rhs_[seg, c])
    # against the single-surface solver
    q = quads[1]
    dS, dD = corrs[1]
    S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, dS, ctx=ctx)
    D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, dD, ctx=ctx)
    x1, _ = inti.gmres(0.5 * inti.I + D - 1j * k * S, rhs_[off[1]:off[2], 2], rtol=1e-12)
    assert relerr(X[off[1]:off[2], 2], x1) < 1e-8


def test_batch_tf32_apply_replays_in_cuda_graph():
    """The batched tensor-core apply (pack + persistent kernel + correction)
    captured into a CUDA graph after one warm-up call, then replayed on new
    densities written into the same buffers: bit-identical to direct calls
    (the kernel's per-item sums have a fixed order)."""
    import torch

    s = torch.cuda.Stream()
    c = inti.Context(0, stream=s.cuda_stream)
    quads = stars((4, 3, 6, 2), seed=3)
    op = inti.Helmholtz(k=5.0, dim=3)
    corrs = [inti.bdim_correction(op, q, q, ctx=c) for q in quads]
    B = inti.BatchOperator(op, quads, "CF", corrs, 1.0, -5.0j, ctx=c)
    nrhs = 64
    dev = torch.device("cuda:0")

    def dev_cols(X):  # column-major complex -> flat float64 device buffer
        return torch.from_numpy(np.asfortranarray(X).T.copy().view(np.float64)).to(dev)

    xs = dev_cols(rhs(B.n, nrhs, True, 7))
    ys = torch.zeros_like(xs)
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        B.apply_device(xs.data_ptr(), ys.data_ptr(), nrhs, "tf32")  # warm-up: builds the tiles, sets attributes
    s.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        B.apply_device(xs.data_ptr(), ys.data_ptr(), nrhs, "tf32")
    for seed in (8, 9):
        xs.copy_(dev_cols(rhs(B.n, nrhs, True, seed)))
        ys.zero_()
        torch.cuda.synchronize()
        g.replay()
        torch.cuda.synchronize()
        got = ys.clone()
        ys.zero_()
        torch.cuda.synchronize()
        with torch.cuda.stream(s):
            B.apply_device(xs.data_ptr(), ys.data_ptr(), nrhs, "tf32")
        s.synchronize()
        assert torch.equal(got, ys)
        assert torch.count_nonzero(got) > 0
    del g


def _c4_build(ctx):
    """The batched workload: 32 seeded star surfaces (n in [6, 27] cells per
    patch edge, 1,944 .. 39,366 nodes), k = 5, D - i k S with per-surface DIM
    corrections, 64 plane waves e^{i k d.x}."""
    r = np.random.default_rng(4)
    ns = r.integers(6, 28, 32)
    quads = [inti.star_quadrature(inti.star_coefficients(r), int(n)) for n in ns]
    k = 5.0
    op = inti.Helmholtz(k=k, dim=3)
    corrs = [inti.bdim_correction(op, q, q, ctx=ctx) for q in quads]
    B = inti.BatchOperator(op, quads, "CF", corrs, 1.0, -1j * k, ctx=ctx)
    d = r.standard_normal((64, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    X = np.concatenate([np.exp(1j * k * (q.coords @ d.T)) for q in quads], axis=0)
    return quads, corrs, B, X, k


def test_c4_batch_sampled_rows_against_oracle(ctx):
    """The full C4 batch (687,852 nodes, 64 right-hand sides) against the
    oracle on 64 sampled rows (2 per surface) x 3 columns, in the pattern of
    test/fmm3d_test.jl:40-42: FP64 batch <= 1e-12 and TF32 batch <= 5e-3
    against the oracle's D - i k S row sums plus the same correction rows;
    and the FP64 batch against the oracle's own DIM corrections of the
    sampled elements (product-level bound)."""
    import oracle as O
    from helpers import block_rows_apply

    quads, corrs, B, X, k = _c4_build(ctx)
    assert B.n == 687_852
    Y64 = B.apply(X, "fp64")
    Y32 = B.apply(X, "tf32")
    r = np.random.default_rng(21)
    cols = [0, 31, 63]
    got64, got32, ref_g, ref_o = ([[] for _ in cols] for _ in range(4))
    for s, q in enumerate(quads):
        off = B.offsets[s]
        els = np.sort(r.choice(q.nel, 2, replace=False))
        rows = els * q.nq + r.integers(0, q.nq, 2)
        gS, gD = (c.arrays() for c in corrs[s])
        oS, oD = O.bdim(O.HELMHOLTZ, k, q.coords, q.normals, q.weights, q.nq, elements=els)
        sel = np.searchsorted(els, rows // q.nq) * q.nq + rows % q.nq
        for ci, c in enumerate(cols):
            x = X[off:off + len(q), c]
            pair = O.apply(O.HELMHOLTZ, O.DL, k, q.coords, q.normals, q.coords, q.normals, q.weights, x, rows=rows) \
                - 1j * k * O.apply(O.HELMHOLTZ, O.SL, k, q.coords, q.normals, q.coords, q.normals, q.weights, x,
                                   rows=rows)
            corr = O.csr_apply(*gD, x)[rows] - 1j * k * O.csr_apply(*gS, x)[rows]
            # product level: the oracle's own corrections of the sampled elements
            odd = block_rows_apply(oD, q.nq, els, x) - 1j * k * block_rows_apply(oS, q.nq, els, x)
            got64[ci].append(Y64[off + rows, c])
            got32[ci].append(Y32[off + rows, c])
            ref_g[ci].append(pair + corr)
            ref_o[ci].append(pair + odd[sel])
    cat = np.concatenate
    worst64 = max(relerr(cat(g), cat(f)) for g, f in zip(got64, ref_g))
    worst32 = max(relerr(cat(g), cat(f)) for g, f in zip(got32, ref_g))
    worst_dim = max(relerr(cat(g), cat(f)) for g, f in zip(got64, ref_o))
    print(f"C4 64 sampled rows x {len(cols)} columns vs oracle: fp64 {worst64:.3e}, tf32 {worst32:.3e}, "
          f"fp64 vs oracle DIM {worst_dim:.3e}")
    # measured on the B200: 1.0e-14, 1.6e-4, 1.4e-14
    assert worst64 < 1e-12
    assert worst32 < 2e-3
    assert worst_dim < 1e-12
