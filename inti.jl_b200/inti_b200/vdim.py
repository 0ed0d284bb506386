"""Volume density interpolation (VDIM) correction of the volume potential
(src/vdim.jl:30-130, 261-285; src/api.jl:282-378), Laplace in 2D and 3D and
Helmholtz in 3D.

    V + δV  with  δV_ij = w_j(i),  L_e w(i) = Θ[i, :]  (least squares),

where, for the monomials p_n(x) = x^α / α! (|α| <= order) and polynomials P_n
with ΔP_n = p_n (Laplace) or ΔP_n + k²P_n = p_n (Helmholtz),

    Θ = S·γ₁P − D·γ₀P − V·p + μ(x)·P(x)

(S, D: boundary layer operators from the boundary quadrature to the targets,
with their own near-field correction; V: the plain volume potential; μ the
Green multiplier).  For every element e with near targets, L_e[n, k] =
p_n(y_k) over the element's nodes, solved in the minimum-norm least-squares
sense (the SVD solve of src/vdim.jl:95-105).

The O(N^2 · nbasis) part, Θ, is computed with the GPU operators (the pair
kernel with the fused corrections); the polynomial algebra and the small
per-element solves run on the host.

Particular solutions.  The reference takes P_n from ElementaryPDESolutions
(`solve_laplace`, an absent third-party package).  Here P_n is the Almansi
expansion of the published method: for p homogeneous of degree m in N
dimensions,

    P = Σ_j a_j |x|^(2j+2) Δ^j p,  a_0 = 1/(2(2m+N)),
    a_j = −a_{j−1} / ((2j+2)(2m−2j+N)),

which satisfies ΔP = p exactly.  Any two particular solutions differ by a
harmonic polynomial H, whose contribution S·γ₁H − D·γ₀H + μH vanishes up to
the boundary quadrature's error, so the corrections agree with the
reference's to that accuracy, not to rounding.

For Helmholtz (`solve_helmholtz` in the reference) the polynomial solution
of ΔP + k²P = p is unique (a polynomial H with ΔH + k²H = 0 is zero: its
top-degree part would satisfy k²H = 0), so P is the reference's own:

    P = Σ_j (−1)^j Δ^j p / k^(2j+2)   (a finite sum: Δ lowers the degree),

since (Δ + k²)P telescopes to p.  Θ, the volume potential and the
corrections are then complex.
"""
from __future__ import annotations

import itertools
import math

import numpy as np

from . import _lib as L
from .geometry import Quadrature


# ----------------------------------------------------------------------------
# polynomials: dict {multi-index tuple: coefficient}
# ----------------------------------------------------------------------------
def _add(P, Q, c=1.0):
    out = dict(P)
    for k, v in Q.items():
        out[k] = out.get(k, 0.0) + c * v
    return {k: v for k, v in out.items() if v != 0.0}


def _mul_r2(P, N):
    """P · |x|^2."""
    out = {}
    for k, v in P.items():
        for d in range(N):
            kk = tuple(k[i] + (2 if i == d else 0) for i in range(N))
            out[kk] = out.get(kk, 0.0) + v
    return out


def _laplacian(P, N):
    out = {}
    for k, v in P.items():
        for d in range(N):
            if k[d] >= 2:
                kk = tuple(k[i] - (2 if i == d else 0) for i in range(N))
                out[kk] = out.get(kk, 0.0) + v * k[d] * (k[d] - 1)
    return {k: v for k, v in out.items() if v != 0.0}


def _derivative(P, d, N):
    out = {}
    for k, v in P.items():
        if k[d] >= 1:
            kk = tuple(k[i] - (1 if i == d else 0) for i in range(N))
            out[kk] = out.get(kk, 0.0) + v * k[d]
    return out


def _evaluate(P, X):
    X = np.asarray(X, dtype=np.float64)
    out = np.zeros(X.shape[0])
    for k, v in P.items():
        out += v * np.prod(X ** np.asarray(k)[None, :], axis=1)
    return out


def _laplace_particular(p, m, N):
    """Almansi expansion: ΔP = p for p homogeneous of degree m."""
    P, term, a, j = {}, dict(p), 0.0, 0
    while term:
        # a_j (Δ^j p has degree m - 2j >= 0 here, so the divisor is positive)
        a = 1.0 / (2 * (2 * m + N)) if j == 0 else -a / ((2 * j + 2) * (2 * m - 2 * j + N))
        T = term
        for _ in range(j + 1):
            T = _mul_r2(T, N)
        P = _add(P, T, a)
        term = _laplacian(term, N)
        j += 1
    return P


def _helmholtz_particular(p, k, N):
    """ΔP + k²P = p: P = Σ_j (−1)^j Δ^j p / k^(2j+2) (the unique polynomial
    solution)."""
    P, term, c = {}, dict(p), 1.0 / (k * k)
    while term:
        P = _add(P, term, c)
        term = _laplacian(term, N)
        c = -c / (k * k)
    return P


def polynomial_solutions_vdim(op, order: int):
    """(multiindices, p, P, ∇P) for every monomial p = x^α/α!, |α| <= order
    (src/vdim.jl:309-345); the multi-indices enumerate the first coordinate
    fastest (Iterators.product)."""
    N = op.dim
    if op.pde == L.HELMHOLTZ:
        if N != 3:
            raise L.UnsupportedError(L.E_UNSUPPORTED, "Helmholtz VDIM is implemented in 3D (the 2D Hankel "
                                                      "kernels are not)")
        k = float(op.k)
        if not k > 0:
            raise L.ArgumentError(L.E_ARG, "Helmholtz VDIM needs a positive wavenumber")
    elif op.pde != L.LAPLACE:
        raise L.UnsupportedError(L.E_UNSUPPORTED, "VDIM is implemented for the Laplace and Helmholtz operators")
    multi, ps, Ps, dPs = [], [], [], []
    for t in itertools.product(range(order + 1), repeat=N):
        alpha = t[::-1]
        if sum(alpha) > order:
            continue
        p = {tuple(alpha): 1.0 / math.prod(math.factorial(a) for a in alpha)}
        P = _helmholtz_particular(p, k, N) if op.pde == L.HELMHOLTZ else _laplace_particular(p, sum(alpha), N)
        multi.append(alpha)
        ps.append(p)
        Ps.append(P)
        dPs.append([_derivative(P, d, N) for d in range(N)])
    return multi, ps, Ps, dPs


# ----------------------------------------------------------------------------
# the correction
# ----------------------------------------------------------------------------
def _near_lists(target: Quadrature, source: Quadrature, maxdist: float):
    """etype_to_nearest_points (src/quadrature.jl:249-286): the element of
    each target (its own for target === source), -1 beyond maxdist."""
    nq = source.nq
    if target is source:
        return np.arange(len(source)) // nq
    from scipy.spatial import cKDTree

    d, j = cKDTree(source.coords).query(target.coords)
    return np.where(d <= maxdist, j // nq, -1)


def vdim_correction(op, target: Quadrature, source: Quadrature, boundary: Quadrature, S, D, V, *,
                    green_multiplier, interpolation_order: int | None = None, maxdist: float = np.inf,
                    center=None, ctx=None):
    """δV of src/vdim.jl:30-130 as a device CSR (a ``CorrectionMatrix``).
    S, D: boundary -> target layer operators (corrected); V: the plain volume
    potential source -> target."""
    from .core import CorrectionMatrix, default_context

    ctx = ctx or default_context()
    if source.nq <= 0:
        raise L.ArgumentError(L.E_ARG, "VDIM needs the element structure of the volume quadrature (nq > 0)")
    if boundary.normals is None:
        raise L.ArgumentError(L.E_ARG, "VDIM needs a boundary quadrature with normals")
    N = op.dim
    order = interpolation_order if interpolation_order is not None else int(source.meta.get("order", 2))
    multi, ps, Ps, dPs = polynomial_solutions_vdim(op, order)
    c = np.zeros(N) if center is None else np.asarray(center, dtype=np.float64)
    ys, yb, xt = source.coords - c, boundary.coords - c, target.coords - c
    b = np.stack([_evaluate(p, ys) for p in ps], axis=1)              # source nodes x basis
    g0 = np.stack([_evaluate(P, yb) for P in Ps], axis=1)             # boundary nodes x basis
    g1 = np.stack([sum(_evaluate(dP[d], yb) * boundary.normals[:, d] for d in range(N)) for dP in dPs], axis=1)
    mu = np.broadcast_to(np.asarray(green_multiplier, dtype=np.float64), (len(target),))
    # Θ <- S γ₁P − D γ₀P − V p + μ P(x)   (src/vdim.jl:268-283)
    theta = S @ g1 - D @ g0 - V @ b
    theta = theta + mu[:, None] * np.stack([_evaluate(P, xt) for P in Ps], axis=1)
    near = _near_lists(target, source, maxdist)
    nq = source.nq
    rows = np.nonzero(near >= 0)[0]
    indptr = np.zeros(len(target) + 1, np.int64)
    indptr[1:] = np.cumsum(np.where(near >= 0, nq, 0))
    indices = (near[rows][:, None] * nq + np.arange(nq)[None, :]).astype(np.int32)
    data = np.zeros((len(rows), nq), theta.dtype)
    for e in np.unique(near[rows]):
        sel = np.nonzero(near[rows] == e)[0]
        Le = b[e * nq:(e + 1) * nq].T                                   # basis x nq
        data[sel] = (np.linalg.pinv(Le) @ theta[rows[sel]].T).T          # min-norm least squares
    return CorrectionMatrix.from_csr(indptr, indices.reshape(-1), data.reshape(-1),
                                     (len(target), len(source)), ctx=ctx)
