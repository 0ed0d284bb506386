"""The allocation-free entry point, inti_apply_noalloc.

It exists for callers that cannot allocate device memory at the point where
they apply the operator — for instance when a framework's caching allocator
already holds the GPU's memory, or inside a solver loop that must not pay for
an allocation.  Its scratch is a fixed static device array, so these tests
check that it reproduces the allocating entry point (inti_op_apply, via
GpuOperator) on two calls in a row with different densities: a second call
must not see the first call's leftovers.  The products are also checked
against the oracle (pair sums plus the same correction rows).  The tests run
on their own and after the rest of the suite (pytest collects this file
last).
"""
import ctypes as C

import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from inti_b200 import _lib as L
from helpers import density, oracle_apply, relerr

pytestmark = pytest.mark.gpu


def _to_device(ctx, a):
    a = np.ascontiguousarray(a)
    p = C.c_void_p()
    ctx.check(ctx.lib.inti_dev_alloc(ctx.handle, a.nbytes, C.byref(p)))
    ctx.check(ctx.lib.inti_memcpy(ctx.handle, p, a.ctypes.data, a.nbytes, L.H2D))
    return p


def _free(ctx, *ptrs):
    for p in ptrs:
        ctx.check(ctx.lib.inti_dev_free(ctx.handle, p))


def _noalloc(ctx, pde, kind, k, prec, q, corr, sigma, alpha=1.0, beta=0.0, y0=None):
    """Apply through inti_apply_noalloc with caller-owned device buffers."""
    lib = ctx.lib
    cplx = pde == L.HELMHOLTZ
    n = len(q)
    bufs = [_to_device(ctx, q.coords), _to_device(ctx, q.normals), _to_device(ctx, q.weights)]
    if corr is not None:
        rp, col, val = corr
        bufs += [_to_device(ctx, rp), _to_device(ctx, col), _to_device(ctx, val)]
    else:
        bufs += [None, None, None]
    x = _to_device(ctx, sigma)
    yh = np.zeros(n, np.complex128 if cplx else np.float64) if y0 is None else y0.copy()
    y = _to_device(ctx, yh)
    st = lib.inti_apply_noalloc(pde, kind, q.dim, k, prec, n, bufs[0], bufs[1], n, bufs[0], bufs[1], bufs[2],
                                bufs[3], bufs[4], bufs[5], x, y, L.cpair(alpha), L.cpair(beta),
                                C.c_void_p(ctx.stream), 1)
    L.check(st, None)
    ctx.check(lib.inti_memcpy(ctx.handle, yh.ctypes.data, y, yh.nbytes, L.D2H))
    _free(ctx, *[b for b in bufs if b is not None], x, y)
    return yh


SL_, DL_, ADL_, HS_ = inti.SingleLayerKernel, inti.DoubleLayerKernel, inti.AdjointDoubleLayerKernel, \
    inti.HyperSingularKernel
# (name, operator, kernel class, ABI kernel, precision, tolerance, correction, surface)
CASES = [
    ("helmholtz_sl_fp64", lambda: inti.Helmholtz(k=6.0, dim=3), SL_, L.SL, "fp64", 1e-12, True, "p2"),
    ("laplace_dl_fp64", lambda: inti.Laplace(dim=3), DL_, L.DL, "fp64", 1e-12, True, "ell"),
    ("laplace_dl_fp32c", lambda: inti.Laplace(dim=3), DL_, L.DL, "fp32c", 2e-5, True, "ell"),
    ("helmholtz_hs_fp64", lambda: inti.Helmholtz(k=6.0, dim=3), HS_, L.HS, "fp64", 1e-12, True, "p2"),
    ("laplace_adl_fp64_nocorr", lambda: inti.Laplace(dim=3), ADL_, L.ADL, "fp64", 1e-12, False, "ell"),
    ("laplace2d_dl_fp64", lambda: inti.Laplace(dim=2), DL_, L.DL, "fp64", 1e-12, True, "kite"),
]
ORACLE_KIND = {L.SL: O.SL, L.DL: O.DL, L.ADL: O.ADL, L.HS: O.HS}


def _surface(name):
    return {"p2": lambda: inti.p2_sphere_quadrature(6), "ell": lambda: inti.ellipsoid_quadrature(5, 5),
            "kite": lambda: inti.kite_quadrature(60, 9)}[name]()


@pytest.mark.parametrize("name,mkop,Kc,kind,prec,tol,with_corr,surf", CASES)
def test_noalloc_matches_allocating_apply_twice(ctx, name, mkop, Kc, kind, prec, tol, with_corr, surf):
    q = _surface(surf)
    op = mkop()
    corr = None
    if with_corr:
        derivative = Kc in (ADL_, HS_)
        if derivative:
            pair = inti.adj_double_layer_hypersingular(op=op, target=q, source=q, correction={"method": "dim"},
                                                       ctx=ctx)
        else:
            pair = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
        corr = pair[0 if Kc in (SL_, ADL_) else 1].correction
    A = inti.GpuOperator(Kc(op), q, q, corr, prec, ctx)
    pde = op.pde
    k = float(getattr(op, "k", 0.0))
    P = {"fp64": L.FP64, "fp32c": L.FP32C}[prec]
    cplx = pde == L.HELMHOLTZ
    carr = corr.arrays() if corr is not None else None
    for call, seed in enumerate((3, 4)):  # two calls in a row, different densities
        sigma = density(len(q), cplx, seed)
        ref = A @ sigma
        got = _noalloc(ctx, pde, kind, k, P, q, carr, sigma)
        assert relerr(got, ref) < tol, (name, call)
        # and against the oracle: pair sums plus the same correction rows
        ora = oracle_apply(pde, ORACLE_KIND[kind], k, q, q, sigma)
        if carr is not None:
            ora = ora + O.csr_apply(*carr, sigma)
        assert relerr(got, ora) < tol, (name, call, "oracle")
    # alpha/beta as inti_op_apply; complex coefficients for the complex operators
    alpha, beta = (0.5 + 0.3j, -2.0 + 1.0j) if cplx else (0.5, -2.0)
    sigma = density(len(q), cplx, 5)
    y0 = density(len(q), cplx, 6)
    ref = y0.copy()
    A.mul(ref, sigma, alpha, beta)
    got = _noalloc(ctx, pde, kind, k, P, q, carr, sigma, alpha, beta, y0)
    assert relerr(got, ref) < tol


def test_noalloc_rejects_problems_beyond_its_scratch(ctx):
    q = inti.ellipsoid_quadrature(2, 5)
    bufs = [_to_device(ctx, a) for a in (q.coords, q.normals, q.weights, np.zeros(len(q)), np.zeros(len(q)))]
    big = 50_000_000  # sizes are checked before any device access
    st = ctx.lib.inti_apply_noalloc(L.LAPLACE, L.DL, 3, 0.0, L.FP64, big, bufs[0], bufs[1], big, bufs[0],
                                    bufs[1], bufs[2], None, None, None, bufs[3], bufs[4], None, None, None, 1)
    assert st == L.E_ARG
    assert b"MiB scratch" in ctx.lib.inti_last_error(None)
    _free(ctx, *bufs)
