"""Problem builders shared by the tests (seeded, small enough for the oracle)."""
import numpy as np

import oracle as O
from inti_b200 import geometry as G

PDE = {"laplace": O.LAPLACE, "helmholtz": O.HELMHOLTZ}
KIND = {"SL": O.SL, "DL": O.DL, "ADL": O.ADL, "HS": O.HS}


def density(n, cplx, seed=1):
    r = np.random.default_rng(seed)
    if cplx:
        return (r.standard_normal(n) + 1j * r.standard_normal(n)) / np.sqrt(2)
    return r.standard_normal(n)


def relerr(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_apply(pde, kind, k, tq, sq, sigma, rows=None):
    return O.apply(pde, kind, k, tq.coords, tq.normals, sq.coords, sq.normals, sq.weights, sigma, rows=rows)


def oracle_dim_csr(pde, k, q, derivative=False, green_multiplier=None, elements=None):
    """Oracle (δS, δD) as CSR triplets (element-block pattern)."""
    dS, dD = O.bdim(pde, k, q.coords, q.normals, q.weights, q.nq, derivative=derivative,
                    green_multiplier=green_multiplier, elements=elements)
    return (O.block_csr(dS, q.nq, elements, len(q)), O.block_csr(dD, q.nq, elements, len(q)))


def small_surfaces():
    """Small quadratures covering every geometry family of the workloads."""
    return {
        "kite": G.kite_quadrature(40, 9),
        "ellipsoid": G.ellipsoid_quadrature(3, 5),
        "p2sphere": G.p2_sphere_quadrature(3),
        "star": G.star_quadrature(G.star_coefficients(np.random.default_rng(3)), 3),
    }


EPS = np.finfo(float).eps


def dim_values_close(pde, k, q, gpu_csr, ora_csr, elements=None, factor=1024.0):
    """Condition-aware comparison of DIM weights: for each element block the
    max deviation must stay below factor*eps*cond(M_e)*max|δ| (each weight is
    the solution of a least-squares problem with matrix M_e^T, so no two
    implementations agree beyond that).  Returns the worst ratio
    deviation / allowance (<= 1 passes)."""
    nq = q.nq
    els = np.arange(q.nel) if elements is None else np.asarray(elements)
    conds = O.dim_element_conds(pde, k, q.coords, q.normals, nq, els)
    g_rp, g_col, g_val = gpu_csr
    o_rp, o_col, o_val = ora_csr
    worst = 0.0
    for e, c in zip(els, conds):
        rows = e * nq + np.arange(nq)
        gv = np.concatenate([g_val[g_rp[i]:g_rp[i + 1]] for i in rows])
        ov = np.concatenate([o_val[o_rp[i]:o_rp[i + 1]] for i in rows])
        allow = factor * EPS * c * max(np.max(np.abs(ov)), 1e-300) + 1e-300
        worst = max(worst, float(np.max(np.abs(gv - ov)) / allow))
    return worst


def harmonic_traces(pde, k, q, xs, c=0.7):
    """γ₀u, γ₁u of u = c*G(·, xs) on the nodes of q (smooth densities)."""
    g0 = np.array([O.kernel(pde, O.SL, k, x, n, xs, None) for x, n in zip(q.coords, q.normals)]) * c
    g1 = np.array([O.kernel(pde, O.ADL, k, x, n, xs, None) for x, n in zip(q.coords, q.normals)]) * c
    if pde == O.LAPLACE:
        return g0.real.copy(), g1.real.copy()
    return g0, g1


def block_rows_apply(values, nq, els, sigma):
    """Rows e*nq + t (e in els, t < nq, in that order) of the element-block
    correction applied to sigma; `values` are O.bdim block values for the
    same elements ((len(els)*nq, nq), column a <-> source node e*nq + a)."""
    els = np.asarray(els)
    v = np.asarray(values).reshape(len(els), nq, nq)
    s = np.asarray(sigma)[els[:, None] * nq + np.arange(nq)[None, :]]
    return np.einsum("eta,ea->et", v, s).reshape(-1)


def smooth_density(pde, k, q, xs):
    """A smooth density: the trace γ₀u of u = G(·, xs), xs off the surface."""
    return harmonic_traces(pde, k, q, xs, 1.0)[0]
