"""GPU off-surface DIM (target !== source, src/api.jl:105-148 with
bdim.jl:50-196 and quadrature.jl:264-286) against the oracle.

* The near assignment (each target to the element of its nearest source node,
  filtered by maxdist) and so the CSR pattern: bit-exact.
* Values: per row, max|Δδ| <= 1024·eps·cond(M_e)·max|δ| with e the row's
  element (each row solves a least-squares problem with matrix M_e^T) and
  max|δ| over the whole matrix: rows far from the surface (or at a circle's
  centre) have corrections that are ~0 by cancellation, so their own scale
  says nothing about the rounding they carry.
* The corrected products (S + δS)·g, (D + δD)·g agree with the oracle's to
  1e-9 relative.
* Through the public API: Green's representation at targets 0.1 off the
  sphere, and the reference's mixed-target known answers on the circle
  (test/dim_test.jl:42-91).
"""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import EPS, harmonic_traces
from inti_b200 import geometry as G

pytestmark = pytest.mark.gpu


def circle_case():
    q = G.circle_quadrature(32, 3)
    g = np.arange(-1.5, 1.5 + 1e-9, 0.1)
    T = np.array([(a, b) for a in g for b in g])
    inn = np.linalg.norm(T, axis=1) < 1.0
    return q, T, inn


def sphere_case(m=200, seed=0):
    q = G.ellipsoid_quadrature(6, 5, scaling=(1.0, 1.0, 1.0))
    r = np.random.default_rng(seed)
    d = r.standard_normal((m, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rad = np.where(np.arange(m) % 2 == 0, 0.9, 1.1)
    return q, d * rad[:, None], rad < 1, d


CASES = [
    ("circle", O.LAPLACE, 0.0, np.inf, False),
    ("circle", O.LAPLACE, 0.0, 0.12, False),
    ("sphere", O.LAPLACE, 0.0, np.inf, False),
    ("sphere", O.LAPLACE, 0.0, 0.11, False),
    ("sphere", O.HELMHOLTZ, 3.0, np.inf, False),
    ("sphere", O.LAPLACE, 0.0, np.inf, True),
    ("sphere", O.HELMHOLTZ, 3.0, 0.11, True),
]


def _op(pde, k, dim):
    return inti.Laplace(dim=dim) if pde == O.LAPLACE else inti.Helmholtz(k=k, dim=dim)


@pytest.mark.parametrize("shape,pde,k,maxdist,derivative", CASES)
def test_off_surface_dim_matches_oracle(ctx, shape, pde, k, maxdist, derivative):
    if shape == "circle":
        q, T, inn = circle_case()
        tn = None
    else:
        q, T, inn, tn = sphere_case()
    mu = np.where(inn, -1.0, 0.0)
    tq = inti.Quadrature(T, tn if derivative else None, np.ones(len(T)), 0)
    dS, dD = inti.bdim_correction(_op(pde, k, q.dim), tq, q, green_multiplier=mu, maxdist=maxdist,
                                  derivative=derivative, ctx=ctx)
    near, oS, oD = O.bdim_targets(pde, k, T, q.coords, q.normals, q.weights, q.nq, mu, maxdist=maxdist,
                                  derivative=derivative, tnormals=tn if derivative else None)
    if maxdist == np.inf:
        assert np.all(near >= 0)
    else:
        assert 0 < np.count_nonzero(near >= 0) < len(T)  # the filter is exercised
    conds = O.dim_element_conds(pde, k, q.coords, q.normals, q.nq)
    import scipy.sparse as sp

    dens = np.cos(np.arange(len(q)) * 0.37) + (1j * np.sin(np.arange(len(q)) * 0.11) if pde == O.HELMHOLTZ else 0)
    kinds = (O.ADL, O.HS) if derivative else (O.SL, O.DL)
    for gpu, ora, kind in ((dS, oS, kinds[0]), (dD, oD, kinds[1])):
        rp, col, val = gpu.arrays()
        o_rp, o_col, o_val = O.targets_csr(near, ora, q.nq, len(q))
        assert gpu.shape == (len(T), len(q))
        assert np.array_equal(rp, o_rp) and np.array_equal(col, o_col)
        scale = max(np.max(np.abs(o_val)), 1e-300)
        worst = 0.0
        for i in np.nonzero(near >= 0)[0]:
            g = val[rp[i]:rp[i + 1]]
            o = o_val[o_rp[i]:o_rp[i + 1]]
            allow = 1024 * EPS * conds[near[i]] * scale
            worst = max(worst, float(np.max(np.abs(g - o)) / allow))
        assert worst <= 1.0, worst
        base = O.apply(pde, kind, k, T, tn if derivative else None, q.coords, q.normals, q.weights, dens)
        yg = base + sp.csr_matrix((val, col, rp), shape=gpu.shape) @ dens
        yo = base + sp.csr_matrix((o_val, o_col, o_rp), shape=gpu.shape) @ dens
        assert np.max(np.abs(yg - yo)) <= 1e-9 * np.max(np.abs(yo))


@pytest.mark.parametrize("pde,k", [(O.LAPLACE, 0.0), (O.HELMHOLTZ, 3.0)])
def test_off_surface_green_identity_through_api(ctx, pde, k):
    q, T, inn, _ = sphere_case()
    x0 = np.array([1.8, 0.3, -0.2])
    g0, g1 = harmonic_traces(pde, k, q, x0, c=1.0)
    uT = np.array([O.kernel(pde, O.SL, k, t, None, x0, None) for t in T])
    uT = uT.real if pde == O.LAPLACE else uT
    op = _op(pde, k, 3)
    S, D = inti.single_double_layer(op=op, target=inti.points(T), source=q,
                                    correction={"method": "dim", "green_multiplier": np.where(inn, -1.0, 0.0),
                                                "maxdist": np.inf}, ctx=ctx)
    lhs = S @ g1 - D @ g0
    err = np.max(np.abs(lhs - np.where(inn, uT, 0)))
    assert err < 1e-4, err


def test_mixed_targets_known_answers_through_api(ctx):
    """test/dim_test.jl:42-91 on the GPU."""
    q, T, inn = circle_case()
    op = inti.Laplace(dim=2)
    u = np.ones(len(q))
    S, D = inti.single_double_layer(op=op, target=inti.points(T), source=q,
                                    correction={"method": "dim", "green_multiplier": np.where(inn, -1.0, 0.0),
                                                "maxdist": np.inf}, ctx=ctx)
    So, Do = inti.single_double_layer(op=op, target=inti.points(T[~inn]), source=q,
                                      correction={"method": "dim", "target_location": "outside",
                                                  "maxdist": np.inf}, ctx=ctx)
    Si, Di = inti.single_double_layer(op=op, target=inti.points(T[inn]), source=q,
                                      correction={"method": "dim", "target_location": "inside",
                                                  "maxdist": np.inf}, ctx=ctx)
    assert np.max(np.abs(Do @ u)) < 1e-3
    assert np.max(np.abs(Di @ u + 1)) < 1e-3
    v = S @ u
    assert np.max(np.abs(v[inn] - Si @ u)) < 1e-3
    assert np.max(np.abs(v[~inn] - So @ u)) < 1e-3


def test_off_surface_argument_errors(ctx):
    q, T, inn = circle_case()
    op = inti.Laplace(dim=2)
    tq = inti.points(T)
    with pytest.raises(inti.ArgumentError):
        inti.bdim_correction(op, tq, q, ctx=ctx)  # green multiplier required
    with pytest.raises(inti.ArgumentError):
        inti.single_double_layer(op=op, target=tq, source=q, correction={"method": "dim"}, ctx=ctx)
    with pytest.raises(inti.ArgumentError):
        inti.single_double_layer(op=op, target=tq, source=q, ctx=ctx,
                                 correction={"method": "dim", "target_location": "inside",
                                             "green_multiplier": np.zeros(len(T))})
    with pytest.raises(inti.ArgumentError):  # ADL/HS corrections need target normals
        inti.bdim_correction(op, tq, q, green_multiplier=0.0, derivative=True, ctx=ctx)
    with pytest.raises(inti.ArgumentError):
        inti.bdim_correction(op, tq, q, green_multiplier=0.0, maxdist=-1.0, ctx=ctx)
