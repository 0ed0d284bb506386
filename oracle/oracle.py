"""TEST INFRASTRUCTURE — ctypes binding of the CPU oracle (inti_oracle.cpp).

Imported only by tests/, __graft_entry__.smoke() (as the checker) and the
cpu_baseline / reference legs of bench.py.  The oracle is the FP64 CPU
restatement of Inti.jl's operator path; see the header of inti_oracle.cpp
for what pins it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import itertools
import math

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"

LAPLACE, HELMHOLTZ = 0, 1
SL, DL, ADL, HS = 0, 1, 2, 3

_lib = None


def build() -> Path:
    """Compile the oracle with the system g++ (no OpenMP dependency)."""
    env = dict(os.environ)
    # the image's default CXX wrapper may lack pieces of the toolchain
    if Path("/usr/bin/g++").exists():
        env["CXX"] = "/usr/bin/g++"
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True, env=env)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists() or LIB.stat().st_mtime < (HERE / "inti_oracle.cpp").stat().st_mtime:
            build()
        _lib = C.CDLL(str(LIB))
        P, D, I64 = C.c_void_p, C.c_double, C.c_int64
        _lib.or_kernel.argtypes = [C.c_int, C.c_int, C.c_int, D, P, P, P, P, P]
        _lib.or_apply.argtypes = [C.c_int, C.c_int, C.c_int, D, I64, I64, P, P, I64, P, P, P, P, P, C.c_int]
        _lib.or_assemble.argtypes = [C.c_int, C.c_int, C.c_int, D, I64, P, P, I64, P, P, P, P, C.c_int]
        _lib.or_csr_apply.argtypes = [I64, P, P, P, C.c_int, P, P]
        _lib.or_coo_to_csr.argtypes = [I64, I64, P, P, P, C.c_int, P, P, P]
        _lib.or_coo_to_csr.restype = I64
        _lib.or_dim_sources.argtypes = [C.c_int, C.c_int, D, P, P]
        _lib.or_bdim.argtypes = [C.c_int, C.c_int, D, I64, P, P, P, C.c_int, C.c_int, P, I64, P, P, P, P,
                                 C.c_int]
        _lib.or_gmres.argtypes = [C.c_int, C.c_int, D, I64, P, P, P, D, D, C.c_int, P, P, P, P, P, P, P, D,
                                  C.c_int, C.c_int, C.c_int, P, P, C.c_int]
        _lib.or_dim_traces.argtypes = [C.c_int, C.c_int, D, I64, P, P, C.c_int, P, P]
        _lib.or_bdim_targets.argtypes = [C.c_int, C.c_int, D, I64, P, P, I64, P, P, P, C.c_int, C.c_int, P, D,
                                         P, P, P, P, C.c_int]
        _lib.or_dl_potential_jvp.argtypes = [I64, P, I64, P, P, P, P, P, P, P, P, P, P, C.c_int]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _c(a, dt=np.float64):
    return None if a is None else np.ascontiguousarray(a, dtype=dt)


def kernel(pde, kind, k, x, nx, y, ny) -> complex:
    x, y = _c(x), _c(y)
    nx = _c(nx if nx is not None else np.zeros_like(x))
    ny = _c(ny if ny is not None else np.zeros_like(y))
    out = np.zeros(2)
    st = lib().or_kernel(pde, kind, len(x), k, _p(x), _p(nx), _p(y), _p(ny), _p(out))
    if st:
        raise ValueError("unsupported kernel")
    return complex(out[0], out[1])


def apply(pde, kind, k, tcoords, tnormals, scoords, snormals, sweights, sigma, rows=None,
          nthreads=0) -> np.ndarray:
    """Rows of y = A sigma, A_ij = K(x_i, y_j) w_j (on the fly)."""
    tc, sc = _c(tcoords), _c(scoords)
    dim = tc.shape[1]
    m, n = tc.shape[0], sc.shape[0]
    tn, sn, sw = _c(tnormals), _c(snormals), _c(sweights)
    cplx = pde == HELMHOLTZ
    sig = _c(sigma, np.complex128 if cplx else np.float64)
    if rows is None:
        out = np.zeros(m, sig.dtype)
        lib().or_apply(pde, kind, dim, k, 0, m, _p(tc), _p(tn), n, _p(sc), _p(sn), _p(sw), _p(sig), _p(out),
                       nthreads)
        return out
    rows = np.asarray(rows, np.int64)
    out = np.zeros(len(rows), sig.dtype)
    tmp = np.zeros(1, sig.dtype)
    for q, r in enumerate(rows):
        lib().or_apply(pde, kind, dim, k, int(r), 1, _p(tc), _p(tn), n, _p(sc), _p(sn), _p(sw), _p(sig),
                       _p(tmp), nthreads)
        out[q] = tmp[0]
    return out


def apply_rows_block(pde, kind, k, tcoords, tnormals, scoords, snormals, sweights, sigma, row0, nrows,
                     nthreads=0):
    tc, sc = _c(tcoords), _c(scoords)
    dim = tc.shape[1]
    n = sc.shape[0]
    cplx = pde == HELMHOLTZ
    sig = _c(sigma, np.complex128 if cplx else np.float64)
    out = np.zeros(nrows, sig.dtype)
    lib().or_apply(pde, kind, dim, k, int(row0), int(nrows), _p(tc), _p(_c(tnormals)), n, _p(sc),
                   _p(_c(snormals)), _p(_c(sweights)), _p(sig), _p(out), nthreads)
    return out


def assemble(pde, kind, k, tcoords, tnormals, scoords, snormals, sweights, nthreads=0) -> np.ndarray:
    tc, sc = _c(tcoords), _c(scoords)
    m, n, dim = tc.shape[0], sc.shape[0], tc.shape[1]
    cplx = pde == HELMHOLTZ
    out = np.zeros((m, n), np.complex128 if cplx else np.float64, order="F")
    lib().or_assemble(pde, kind, dim, k, m, _p(tc), _p(_c(tnormals)), n, _p(sc), _p(_c(snormals)),
                      _p(_c(sweights)), _p(out), nthreads)
    return out


def csr_apply(indptr, indices, data, x) -> np.ndarray:
    indptr = _c(indptr, np.int64)
    indices = _c(indices, np.int32)
    cplx = np.iscomplexobj(data) or np.iscomplexobj(x)
    data = _c(data, np.complex128 if cplx else np.float64)
    x = _c(x, data.dtype)
    y = np.zeros(len(indptr) - 1, data.dtype)
    lib().or_csr_apply(len(indptr) - 1, _p(indptr), _p(indices), _p(data), int(cplx), _p(x), _p(y))
    return y


def coo_to_csr(m, I, J, V):
    """The CSR of ``sparse(I, J, V, m, n)``: duplicates summed, rows sorted."""
    I, J = _c(I, np.int64), _c(J, np.int64)
    cplx = np.iscomplexobj(V)
    V = _c(V, np.complex128 if cplx else np.float64)
    nnz = len(I)
    rp = np.zeros(m + 1, np.int64)
    col = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1), V.dtype)
    out = lib().or_coo_to_csr(m, nnz, _p(I), _p(J), _p(V), int(cplx), _p(rp), _p(col), _p(val))
    return rp, col[:out], val[:out]


def dim_sources(dim, ns, R, c):
    c = _c(c)
    xs = np.zeros((ns, dim))
    lib().or_dim_sources(dim, ns, R, _p(c), _p(xs))
    return xs


def bdim(pde, k, coords, normals, weights, nq, derivative=False, green_multiplier=None, elements=None,
         nthreads=0, return_theta=False):
    """Block values of (δS, δD) for the selected elements (all if None):
    arrays (nsel*nq, nq); row q*nq+t, column a <-> target e*nq+t, source
    e*nq+a."""
    x, nrm, w = _c(coords), _c(normals), _c(weights)
    n, dim = x.shape
    cplx = pde == HELMHOLTZ
    sel = None if elements is None else _c(elements, np.int64)
    nsel = n // nq if sel is None else len(sel)
    dt = np.complex128 if cplx else np.float64
    dS = np.zeros((nsel * nq, nq), dt)
    dD = np.zeros((nsel * nq, nq), dt)
    ns = int(np.ceil(3 * nq))
    theta = np.zeros((nsel * nq, ns), np.complex128) if return_theta else None
    gm = None if green_multiplier is None else _c(np.broadcast_to(green_multiplier, (n,)))
    st = lib().or_bdim(pde, dim, k, n, _p(x), _p(nrm), _p(w), nq, int(derivative), _p(gm),
                       nsel if sel is not None else 0, _p(sel), _p(dS), _p(dD), _p(theta), nthreads)
    if st:
        raise ValueError(f"or_bdim failed ({st})")
    return (dS, dD, theta) if return_theta else (dS, dD)


def bdim_targets(pde, k, tcoords, scoords, snormals, sweights, nq, green_multiplier, maxdist=np.inf,
                 derivative=False, tnormals=None, nthreads=0, return_theta=False):
    """Off-surface DIM (target !== source): (near_elem, dS, dD[, theta]) with
    near_elem[i] the element of target i's nearest source node (-1 beyond
    maxdist) and rows (m, nq) of corrections to that element's nodes."""
    tx, x, nrm, w = _c(tcoords), _c(scoords), _c(snormals), _c(sweights)
    tn = _c(tnormals)
    m, dim = tx.shape
    n = x.shape[0]
    cplx = pde == HELMHOLTZ
    dt = np.complex128 if cplx else np.float64
    near = np.full(m, -1, np.int64)
    dS = np.zeros((m, nq), dt)
    dD = np.zeros((m, nq), dt)
    ns = int(np.ceil(3 * nq))
    theta = np.zeros((m, ns), np.complex128) if return_theta else None
    gm = _c(np.broadcast_to(np.asarray(green_multiplier, dtype=np.float64), (m,)))
    st = lib().or_bdim_targets(pde, dim, k, m, _p(tx), _p(tn), n, _p(x), _p(nrm), _p(w), nq, int(derivative),
                               _p(gm), float(maxdist), _p(near), _p(dS), _p(dD), _p(theta), nthreads)
    if st:
        raise ValueError(f"or_bdim_targets failed ({st})")
    return (near, dS, dD, theta) if return_theta else (near, dS, dD)


def targets_csr(near, values, nq, n):
    """CSR (indptr, indices, data) of off-surface DIM rows from bdim_targets."""
    m = len(near)
    counts = np.where(near >= 0, nq, 0)
    indptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    rows = np.nonzero(near >= 0)[0]
    indices = (near[rows][:, None] * nq + np.arange(nq)[None, :]).reshape(-1).astype(np.int32)
    data = values[rows].reshape(-1)
    return indptr, indices, data


def block_csr(values, nq, elements=None, n=None):
    """CSR arrays of the element-block pattern for block values from bdim()."""
    nsel = values.shape[0] // nq
    els = np.arange(nsel) if elements is None else np.asarray(elements)
    rows = (els[:, None] * nq + np.arange(nq)[None, :]).reshape(-1)
    I = np.repeat(rows, nq)
    J = np.repeat(els * nq, nq * nq) + np.tile(np.arange(nq), nsel * nq)
    m = n if n is not None else int(rows.max()) + 1
    return coo_to_csr(m, I, J, values.reshape(-1))


def gmres(pde, k, coords, normals, weights, shift, terms, b, rtol=1e-10, restart=100, maxiter=200,
          nthreads=0):
    """terms: list of (kind, coef, csr or None) with csr = (indptr, indices, data)."""
    x, nrm, w = _c(coords), _c(normals), _c(weights)
    n, dim = x.shape
    cplx = pde == HELMHOLTZ or np.iscomplexobj(b) or any(isinstance(c, complex) for _, c, _ in terms) or \
        isinstance(shift, complex)
    dt = np.complex128 if cplx else np.float64
    b = _c(b, dt)
    sol = np.zeros(n, dt)
    nt = len(terms)
    kinds = (C.c_int * nt)(*[t[0] for t in terms])
    coefs = (C.c_double * (2 * nt))()
    keep = []
    rps = (C.c_void_p * nt)()
    cols = (C.c_void_p * nt)()
    vals = (C.c_void_p * nt)()
    for i, (kind, c, csr) in enumerate(terms):
        c = complex(c)
        coefs[2 * i], coefs[2 * i + 1] = c.real, c.imag
        if csr is not None:
            rp, col, val = _c(csr[0], np.int64), _c(csr[1], np.int32), _c(csr[2], np.complex128 if cplx else np.float64)
            keep += [rp, col, val]
            rps[i], cols[i], vals[i] = rp.ctypes.data, col.ctypes.data, val.ctypes.data
    hist = np.zeros(maxiter + 1)
    fr = C.c_double()
    shift = complex(shift)
    if pde == HELMHOLTZ and not cplx:
        raise ValueError
    it = lib().or_gmres(pde, dim, k, n, _p(x), _p(nrm), _p(w), shift.real, shift.imag, nt, kinds, coefs,
                        C.cast(rps, C.c_void_p), C.cast(cols, C.c_void_p), C.cast(vals, C.c_void_p),
                        _p(b), _p(sol), rtol, restart, maxiter, int(cplx), _p(hist), C.byref(fr), nthreads)
    return sol, {"iterations": it, "relres": fr.value, "history": hist[: it + 1]}


def dl_potential_jvp(tcoords, scoords, snormals, sweights, sigma, dsx=None, dsn=None, dsw=None, dsigma=None,
                     nthreads=0):
    tc, sc, sn, sw, sg = map(_c, (tcoords, scoords, snormals, sweights, sigma))
    m, n = tc.shape[0], sc.shape[0]
    u, du = np.zeros(m), np.zeros(m)
    lib().or_dl_potential_jvp(m, _p(tc), n, _p(sc), _p(sn), _p(sw), _p(sg), _p(_c(dsx)), _p(_c(dsn)),
                              _p(_c(dsw)), _p(_c(dsigma)), _p(u), _p(du), nthreads)
    return u, du


def dim_element_conds(pde, k, coords, normals, nq, elements=None):
    """2-norm condition number of each element's least-squares matrix
    M^T = [g0[el,:]; g1[el,:]]^T (ns x 2nq), src/bdim.jl:160-163."""
    x, nrm = _c(coords), _c(normals)
    n, dim = x.shape
    ns = int(np.ceil(3 * nq))
    g0 = np.zeros((n, ns), np.complex128)
    g1 = np.zeros((n, ns), np.complex128)
    lib().or_dim_traces(pde, dim, k, n, _p(x), _p(nrm), nq, _p(g0), _p(g1))
    els = np.arange(n // nq) if elements is None else np.asarray(elements)
    M = np.concatenate([g0.reshape(-1, nq, ns)[els], g1.reshape(-1, nq, ns)[els]], axis=1)
    if pde == LAPLACE:
        M = M.real
    return np.linalg.cond(np.transpose(M, (0, 2, 1)))


# ----------------------------------------------------------------------------
# VDIM (src/vdim.jl:30-130, 261-285), Laplace in 2D and 3D, restated with
# dense coefficient arrays C[i, j(, k)] <-> x^i y^j (z^k); particular
# solutions of ΔP = p by the Almansi expansion P = Σ_j a_j r^(2j+2) Δ^j p.
# ----------------------------------------------------------------------------
def _ax(d, sl, nd):
    """Index selecting `sl` along axis d of an nd-array."""
    return tuple(sl if a == d else slice(None) for a in range(nd))


def _along(v, d, nd):
    """1-D array v shaped to broadcast along axis d."""
    return v.reshape(tuple(-1 if a == d else 1 for a in range(nd)))


def _pl_lap(C):
    out = np.zeros_like(C)
    nd, n = C.ndim, C.shape[0]
    for d in range(nd):
        k = np.arange(2, n)
        out[_ax(d, slice(None, -2), nd)] += C[_ax(d, slice(2, None), nd)] * _along(k * (k - 1), d, nd)
    return out


def _pl_r2(C):
    out = np.zeros_like(C)
    for d in range(C.ndim):
        out[_ax(d, slice(2, None), C.ndim)] += C[_ax(d, slice(None, -2), C.ndim)]
    return out


def _pl_eval(C, X):
    idx = np.nonzero(C)
    terms = C[idx][None, :]
    for d, e in enumerate(idx):
        terms = terms * X[:, d:d + 1] ** e[None, :]
    return terms.sum(axis=1)


def _pl_dx(C, d):
    out = np.zeros_like(C)
    nd, n = C.ndim, C.shape[0]
    out[_ax(d, slice(None, -1), nd)] = C[_ax(d, slice(1, None), nd)] * _along(np.arange(1, n), d, nd)
    return out


def vdim_basis(order, size=None, dim=2, k=None):
    """[(p, P)] for x^α/α!, |α| <= order, the first index fastest.  ΔP = p
    (Laplace, Almansi expansion) or, with a wavenumber k, ΔP + k²P = p
    (Helmholtz: P = Σ_j (−1)^j Δ^j p / k^(2j+2), the unique polynomial
    solution, src/vdim.jl:369-373)."""
    size = size or order + 2 * (order // 2 + 1) + 3
    out = []
    for rev in itertools.product(range(order + 1), repeat=dim):
        alpha = rev[::-1]
        if sum(alpha) > order:
            continue
        p = np.zeros((size,) * dim)
        p[alpha] = 1.0 / math.prod(math.factorial(a) for a in alpha)
        m, P, term, j, c = sum(alpha), np.zeros((size,) * dim), p.copy(), 0, 0.0
        if k is not None:
            c = 1.0 / (k * k)
            while np.any(term):
                P = P + c * term
                term = _pl_lap(term)
                c = -c / (k * k)
            out.append((p, P))
            continue
        while np.any(term):
            c = 1.0 / (2 * (2 * m + dim)) if j == 0 else -c / ((2 * j + 2) * (2 * m - 2 * j + dim))
            T = term
            for _ in range(j + 1):
                T = _pl_r2(T)
            P = P + c * T
            term = _pl_lap(term)
            j += 1
        out.append((p, P))
    return out


def vdim(tcoords, vcoords, vweights, nq, bcoords, bnormals, bweights, bnq, green_multiplier, order,
         maxdist=np.inf, same=False, pde=LAPLACE, k=0.0):
    """(near_elem, values (m, nq)) of δV (src/vdim.jl:30-130, 261-285);
    `same` when the targets are the volume nodes; Laplace (2D, 3D) or
    Helmholtz (3D, wavenumber k)."""
    from scipy.spatial import cKDTree

    T, Y = _c(tcoords), _c(vcoords)
    m = T.shape[0]
    mu = np.broadcast_to(np.asarray(green_multiplier, dtype=np.float64), (m,))
    dim = Y.shape[1]
    basis = vdim_basis(order, dim=dim, k=k if pde == HELMHOLTZ else None)
    b = np.stack([_pl_eval(p, Y) for p, _ in basis], axis=1)
    g0 = np.stack([_pl_eval(P, bcoords) for _, P in basis], axis=1)
    g1 = np.stack([sum(_pl_eval(_pl_dx(P, d), bcoords) * bnormals[:, d] for d in range(dim)) for _, P in basis], axis=1)
    near_b, bS, bD = bdim_targets(pde, k, T, bcoords, bnormals, bweights, bnq, mu, maxdist=maxdist)
    ipS, ixS, dvS = targets_csr(near_b, bS, bnq, len(bcoords))
    ipD, ixD, dvD = targets_csr(near_b, bD, bnq, len(bcoords))
    theta = np.zeros((m, len(basis)), np.complex128 if pde == HELMHOLTZ else np.float64)
    for n in range(len(basis)):
        sg = apply(pde, SL, k, T, None, bcoords, bnormals, bweights, g1[:, n]) + csr_apply(ipS, ixS, dvS, g1[:, n])
        dg = apply(pde, DL, k, T, None, bcoords, bnormals, bweights, g0[:, n]) + csr_apply(ipD, ixD, dvD, g0[:, n])
        vb = apply(pde, SL, k, T, None, Y, None, vweights, b[:, n])
        theta[:, n] = sg - dg - vb + mu * _pl_eval(basis[n][1], T)
    if same:
        near = np.arange(m) // nq
    else:
        d, j = cKDTree(Y).query(T)
        near = np.where(d <= maxdist, j // nq, -1)
    vals = np.zeros((m, nq), theta.dtype)
    for i in np.nonzero(near >= 0)[0]:
        e = near[i]
        Le = b[e * nq:(e + 1) * nq].T
        vals[i] = np.linalg.lstsq(Le, theta[i], rcond=None)[0]
    return near, vals
