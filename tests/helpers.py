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
