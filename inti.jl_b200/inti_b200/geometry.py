"""Quadrature nodes for the surfaces and curves the operator runs on.

Host-side setup that mirrors how Inti.jl turns a parametrised geometry into
the flat node arrays its operators consume:

* ``meshgen(Γ, n)`` splits each parameter domain into equal cells and wraps
  each one in a parametric element (src/mesh.jl:379-387, ``_meshgen``; cells
  enumerated first-index-fastest, like ``CartesianIndices``);
* ``Quadrature(msh; qorder)`` pushes a reference rule through every element:
  node ``x = el(x̂)``, weight ``w = sqrt(det(JᵀJ))·ŵ`` and normal
  ``ν = s·normalize(t₂, −t₁)`` (curves) or ``normalize(t₁ × t₂)`` (surfaces)
  (src/quadrature.jl:133-162, src/utils.jl:90-135);
* rules: Gauss–Legendre on [0,1] with ``ceil((order+1)/2)`` points
  (src/reference_integration.jl:139-158), tensor products of it on squares
  (src/reference_integration.jl:241-260, src/quadrature.jl:212-215) and the
  tabulated 6-point Vioreanu–Rokhlin rule on triangles for order 4
  (src/quad_rules_tables_triangle.jl:262-269).

Jacobians are analytic here; Inti obtains the same matrices with ForwardDiff
(src/reference_interpolation.jl:36-39).  Nodes of one element are contiguous
(src/quadrature.jl:160), which is what the correction pattern relies on.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

__all__ = [
    "Quadrature",
    "gauss_legendre",
    "gauss_legendre_for_order",
    "VR4N6",
    "disk_triangle_quadrature",
    "curve_quadrature",
    "kite_quadrature",
    "circle_quadrature",
    "ellipsoid_quadrature",
    "star_quadrature",
    "p2_sphere_quadrature",
    "unit_sphere_patch",
]


@dataclass
class Quadrature:
    """Flat quadrature-node arrays of one closed curve or surface.

    ``coords`` is ``(n, dim)``, ``normals`` ``(n, dim)`` (or None for bare
    points), ``weights`` ``(n,)``.  Element ``e`` owns nodes
    ``e*nq .. e*nq+nq-1`` (Inti's ``etype2qtags``, src/quadrature.jl:160).
    """

    coords: np.ndarray
    normals: np.ndarray | None
    weights: np.ndarray
    nq: int = 0
    meta: dict = field(default_factory=dict)

    def __post_init__(self):
        self.coords = np.ascontiguousarray(self.coords, dtype=np.float64)
        if self.normals is not None:
            self.normals = np.ascontiguousarray(self.normals, dtype=np.float64)
        self.weights = np.ascontiguousarray(self.weights, dtype=np.float64)
        n, dim = self.coords.shape
        if dim not in (2, 3):
            raise ValueError(f"coords must be (n, 2) or (n, 3), got {self.coords.shape}")
        if self.weights.shape != (n,):
            raise ValueError("weights must have one entry per node")
        if self.normals is not None and self.normals.shape != (n, dim):
            raise ValueError("normals must match coords")
        if self.nq and n % self.nq:
            raise ValueError("node count is not a multiple of nodes per element")

    def __len__(self) -> int:
        return self.coords.shape[0]

    @property
    def dim(self) -> int:
        return self.coords.shape[1]

    @property
    def nel(self) -> int:
        return len(self) // self.nq if self.nq else 0

    def etype2qtags(self) -> np.ndarray:
        """``(nq, nel)`` 0-based node ids per element (column per element)."""
        return np.arange(len(self)).reshape(self.nel, self.nq).T

    def integrate(self, f) -> float:
        """``Σ f(x_i)·w_i`` (src/quadrature.jl:304-306)."""
        return float(np.sum(f(self.coords) * self.weights))


def points(coords) -> Quadrature:
    """Bare target points (no normals, unit weights): Inti accepts plain
    ``SVector`` targets in ``IntegralOperator`` (src/quadrature.jl:50)."""
    c = np.asarray(coords, dtype=np.float64)
    return Quadrature(c, None, np.ones(c.shape[0]), 0)


# ----------------------------------------------------------------------------
# reference rules
# ----------------------------------------------------------------------------
def gauss_legendre(n: int) -> tuple[np.ndarray, np.ndarray]:
    """n-point Gauss–Legendre nodes/weights on [0, 1], ascending.

    Newton iteration on the three-term recurrence of P_n (the published
    Golub–Welsch/Newton construction that QuadGK.gauss(T, n, 0, 1) also
    evaluates), then the affine map [-1,1] → [0,1].
    """
    if n < 1:
        raise ValueError("n must be >= 1")
    i = np.arange(1, n + 1)
    t = np.cos(np.pi * (i - 0.25) / (n + 0.5))
    for _ in range(100):
        p0 = np.ones_like(t)
        p1 = t.copy()
        for k in range(2, n + 1):
            p0, p1 = p1, ((2 * k - 1) * t * p1 - (k - 1) * p0) / k
        if n == 1:
            p0, p1 = np.ones_like(t), t.copy()
        dp = n * (t * p1 - p0) / (t * t - 1)
        dt = p1 / dp
        t = t - dt
        if np.max(np.abs(dt)) < 1e-16:
            break
    p0 = np.ones_like(t)
    p1 = t.copy()
    for k in range(2, n + 1):
        p0, p1 = p1, ((2 * k - 1) * t * p1 - (k - 1) * p0) / k
    if n == 1:
        p0, p1 = np.ones_like(t), t.copy()
    dp = n * (t * p1 - p0) / (t * t - 1)
    w = 2.0 / ((1 - t * t) * dp * dp)
    order = np.argsort(t)
    t, w = t[order], w[order]
    return (t + 1) / 2, w / 2


def gauss_legendre_for_order(order: int) -> tuple[np.ndarray, np.ndarray]:
    """``GaussLegendre(; order)`` = ceil((order+1)/2) points
    (src/reference_integration.jl:152)."""
    return gauss_legendre(int(math.ceil((order + 1) / 2)))


# 6-point Vioreanu–Rokhlin rule on the reference triangle (order 4): the
# tabulated values of src/quad_rules_tables_triangle.jl:262-269 (a data table
# that must be identical for the discretisation to be Inti's).
VR4N6 = (
    np.array(
        [
            [0.09157621350977069, 0.8168475729804586],
            [0.09157621350977072, 0.09157621350977081],
            [0.8168475729804584, 0.09157621350977081],
            [0.44594849091596483, 0.10810301816807029],
            [0.4459484909159649, 0.445948490915965],
            [0.10810301816807016, 0.445948490915965],
        ]
    ),
    np.array(
        [
            0.0549758718276609,
            0.0549758718276609,
            0.0549758718276609,
            0.1116907948390057,
            0.1116907948390057,
            0.1116907948390057,
        ]
    ),
)


def _square_rule(order: int):
    """TensorProductQuadrature(GL, GL) on [0,1]²; nodes enumerated with the
    first coordinate fastest (Iterators.product order,
    src/reference_integration.jl:254-259)."""
    x, w = gauss_legendre_for_order(order)
    X = np.array([[a, b] for b in x for a in x])
    W = np.array([wa * wb for wb in w for wa in w])
    return X, W


# ----------------------------------------------------------------------------
# curves (2D)
# ----------------------------------------------------------------------------
def curve_quadrature(f, df, a: float, b: float, nel: int, qorder: int) -> Quadrature:
    """Quadrature of ``meshgen(parametric_curve(f, a, b), nel)``.

    ``f(t) -> (len(t), 2)`` and ``df`` its derivative.  Element e maps
    x̂ ∈ [0,1] to t = a + (e + x̂)·Δ with Δ = (b − a)/nel.
    """
    xh, wh = gauss_legendre_for_order(qorder)
    nq = len(xh)
    delta = (b - a) / nel
    e = np.arange(nel)
    t = (a + (e[:, None] * delta)) + xh[None, :] * delta  # low + x̂·Δ
    t = t.reshape(-1)
    x = f(t)
    tang = df(t) * delta  # jacobian column
    mu = np.sqrt(tang[:, 0] ** 2 + tang[:, 1] ** 2)
    w = (mu.reshape(nel, nq) * wh[None, :]).reshape(-1)
    nrm = np.stack([tang[:, 1], -tang[:, 0]], axis=1) / mu[:, None]
    return Quadrature(x, nrm, w, nq, {"kind": "curve", "nel": nel, "qorder": qorder})


def kite_quadrature(nel: int = 200, qorder: int = 9) -> Quadrature:
    """Kite χ(t) = (cos t + 0.65 cos 2t − 0.65, 1.5 sin t), t ∈ [0, 2π)
    (docs/src/examples/pep.md:276-277).  Defaults give 200 GL-5 panels,
    N = 1000."""

    def f(t):
        return np.stack([np.cos(t) + 0.65 * np.cos(2 * t) - 0.65, 1.5 * np.sin(t)], axis=1)

    def df(t):
        return np.stack([-np.sin(t) - 1.3 * np.sin(2 * t), 1.5 * np.cos(t)], axis=1)

    q = curve_quadrature(f, df, 0.0, 2 * np.pi, nel, qorder)
    q.meta["shape"] = "kite"
    return q


def circle_quadrature(nel: int, qorder: int, r: float = 1.0) -> Quadrature:
    """Circle of radius r (test/green_identities_test.jl:43-47)."""

    def f(t):
        return r * np.stack([np.cos(t), np.sin(t)], axis=1)

    def df(t):
        return r * np.stack([-np.sin(t), np.cos(t)], axis=1)

    q = curve_quadrature(f, df, 0.0, 2 * np.pi, nel, qorder)
    q.meta["shape"] = "circle"
    return q


# ----------------------------------------------------------------------------
# surfaces (3D), cube-sphere parametrisation
# ----------------------------------------------------------------------------
def unit_sphere_patch(u, v, pid: int):
    """Point on the cube face ``pid`` (1..6) before projection, and its
    u/v derivatives (src/simpleshapes.jl:72-89)."""
    one = np.ones_like(u)
    zero = np.zeros_like(u)
    if pid == 1:
        p, pu, pv = (one, u, v), (zero, one, zero), (zero, zero, one)
    elif pid == 2:
        p, pu, pv = (-u, one, v), (-one, zero, zero), (zero, zero, one)
    elif pid == 3:
        p, pu, pv = (u, v, one), (one, zero, zero), (zero, one, zero)
    elif pid == 4:
        p, pu, pv = (-one, -u, v), (zero, -one, zero), (zero, zero, one)
    elif pid == 5:
        p, pu, pv = (u, -one, v), (one, zero, zero), (zero, zero, one)
    elif pid == 6:
        p, pu, pv = (-u, v, -one), (-one, zero, zero), (zero, one, zero)
    else:
        raise ValueError("patch id must be 1..6")
    return np.stack(p, -1), np.stack(pu, -1), np.stack(pv, -1)


def _sphere_map(u, v, pid):
    """x̂ = p/|p| on the unit sphere with its derivatives along u and v."""
    p, pu, pv = unit_sphere_patch(u, v, pid)
    s = np.sqrt(u * u + v * v + 1.0)[..., None]  # |p|
    xh = p / s
    xu = pu / s - p * (np.sum(p * pu, -1, keepdims=True) / s**3)
    xv = pv / s - p * (np.sum(p * pv, -1, keepdims=True) / s**3)
    return xh, xu, xv


def _surface_quadrature(radial, n: int, qorder: int, scaling=(1.0, 1.0, 1.0)) -> Quadrature:
    """6 patches × n×n cells × GL tensor rule.  ``radial(x̂) -> (r, ∇r)`` sets
    the surface x = scaling ⊙ (r(x̂)·x̂); r ≡ 1 gives the (scaled) sphere of
    src/simpleshapes.jl:43-70."""
    X, W = _square_rule(qorder)
    nq = len(W)
    h = 2.0 / n
    scal = np.asarray(scaling, dtype=np.float64)
    # cells first-index-fastest: cell (i1, i2) -> low = -1 + (i-1)h
    i1 = np.tile(np.arange(n), n)
    i2 = np.repeat(np.arange(n), n)
    lo1 = -1.0 + i1 * h
    lo2 = -1.0 + i2 * h
    u = lo1[:, None] + X[None, :, 0] * h
    v = lo2[:, None] + X[None, :, 1] * h
    xs, ns, ws = [], [], []
    for pid in range(1, 7):
        xh, xu, xv = _sphere_map(u, v, pid)
        r, gr = radial(xh)
        # x = r(x̂) x̂ ; dx = r dx̂ + x̂ (∇r·dx̂)
        tu = r[..., None] * xu + xh * np.sum(gr * xu, -1, keepdims=True)
        tv = r[..., None] * xv + xh * np.sum(gr * xv, -1, keepdims=True)
        x = scal * (r[..., None] * xh)
        tu = scal * tu * h  # chain rule of the element map (cell side h)
        tv = scal * tv * h
        cr = np.cross(tu, tv)
        mu = np.linalg.norm(cr, axis=-1)
        xs.append(x.reshape(-1, 3))
        ns.append((cr / mu[..., None]).reshape(-1, 3))
        ws.append((mu * W[None, :]).reshape(-1))
    return Quadrature(np.concatenate(xs), np.concatenate(ns), np.concatenate(ws), nq,
                      {"kind": "surface", "n": n, "qorder": qorder})


def ellipsoid_quadrature(n: int, qorder: int = 5, scaling=(1.0, 0.7, 0.5)) -> Quadrature:
    """``GeometricEntity("ellipsoid"; scaling)`` meshed with n×n cells per
    patch (src/simpleshapes.jl:43-70); qorder 5 → GL3×GL3, 9 nodes/element.
    n = 61 gives N = 200,934."""

    def radial(xh):
        return np.ones(xh.shape[:-1]), np.zeros_like(xh)

    q = _surface_quadrature(radial, n, qorder, scaling)
    q.meta.update(shape="ellipsoid", scaling=tuple(scaling))
    return q


# Real harmonic polynomials of degree 1..3 (unnormalised), as monomial lists
# (coefficient, (a, b, c)) meaning coef * x^a y^b z^c.
_HARMONICS = [
    [(1, (1, 0, 0))], [(1, (0, 1, 0))], [(1, (0, 0, 1))],
    [(1, (1, 1, 0))], [(1, (0, 1, 1))], [(1, (1, 0, 1))],
    [(1, (2, 0, 0)), (-1, (0, 2, 0))],
    [(2, (0, 0, 2)), (-1, (2, 0, 0)), (-1, (0, 2, 0))],
    [(1, (3, 0, 0)), (-3, (1, 2, 0))],
    [(3, (2, 1, 0)), (-1, (0, 3, 0))],
    [(1, (1, 1, 1))],
    [(1, (2, 0, 1)), (-1, (0, 2, 1))],
    [(4, (1, 0, 2)), (-1, (3, 0, 0)), (-1, (1, 2, 0))],
    [(4, (0, 1, 2)), (-1, (2, 1, 0)), (-1, (0, 3, 0))],
    [(2, (0, 0, 3)), (-3, (2, 0, 1)), (-3, (0, 2, 1))],
]


def _harmonic_eval(coefs, xh):
    val = np.zeros(xh.shape[:-1])
    grad = np.zeros_like(xh)
    x, y, z = xh[..., 0], xh[..., 1], xh[..., 2]

    def pw(t, e):
        return t**e if e > 0 else np.ones_like(t)

    for c, poly in zip(coefs, _HARMONICS):
        if c == 0:
            continue
        for m, (a, b, cc) in poly:
            val += c * m * pw(x, a) * pw(y, b) * pw(z, cc)
            if a:
                grad[..., 0] += c * m * a * pw(x, a - 1) * pw(y, b) * pw(z, cc)
            if b:
                grad[..., 1] += c * m * b * pw(x, a) * pw(y, b - 1) * pw(z, cc)
            if cc:
                grad[..., 2] += c * m * cc * pw(x, a) * pw(y, b) * pw(z, cc - 1)
    return val, grad


def star_coefficients(rng: np.random.Generator) -> np.ndarray:
    """Seeded low-degree (l ≤ 3) harmonic coefficients for a smooth star
    surface r = 1 + 0.2·Σ a·Y, scaled so that max |Σ a·Y| on S² is 1 (so
    r ∈ [0.8, 1.2])."""
    a = rng.standard_normal(len(_HARMONICS))
    # normalise on a dense sample of the sphere
    g = rng.standard_normal((20000, 3))
    g /= np.linalg.norm(g, axis=1, keepdims=True)
    v, _ = _harmonic_eval(a, g)
    return a / np.max(np.abs(v)) * 0.98


def star_quadrature(coefs, n: int, qorder: int = 5) -> Quadrature:
    """Star-shaped surface r(x̂) = 1 + 0.2·Σ a_lm Y_lm(x̂) on the cube-sphere
    parametrisation (the pattern of src/simpleshapes.jl:150-163)."""
    coefs = np.asarray(coefs, dtype=np.float64)

    def radial(xh):
        v, g = _harmonic_eval(coefs, xh)
        return 1.0 + 0.2 * v, 0.2 * g

    q = _surface_quadrature(radial, n, qorder)
    q.meta.update(shape="star")
    return q


# ----------------------------------------------------------------------------
# quadratic-triangle sphere (P2 Lagrange elements)
# ----------------------------------------------------------------------------
# P2 reference nodes (src/reference_interpolation.jl:499-509, product order
# with the first index fastest): (0,0),(½,0),(1,0),(0,½),(½,½),(0,1); as
# barycentric multi-indices (i, j, k - i - j) with k = 2.
_P2_IDX = [(0, 0, 2), (1, 0, 1), (2, 0, 0), (0, 1, 1), (1, 1, 0), (0, 2, 0)]


def _lag1d(m, t):
    """ℓ_m(t) = Π_{j=1..m} (t − (j−1))/j and its derivative."""
    if m == 0:
        return np.ones_like(t), np.zeros_like(t)
    if m == 1:
        return t, np.ones_like(t)
    return t * (t - 1) / 2, (2 * t - 1) / 2


def _p2_basis(u, v):
    """Values and (d/du, d/dv) of the six P2 Lagrange functions
    (src/reference_interpolation.jl:514-538: products of 1D Lagrange factors
    in the scaled barycentric coordinates)."""
    lam = (2 * u, 2 * v, 2 * (1 - u - v))
    dlam = ((2, 0), (0, 2), (-2, -2))
    vals, du, dv = [], [], []
    for idx in _P2_IDX:
        f = [_lag1d(idx[d], lam[d]) for d in range(3)]
        val = f[0][0] * f[1][0] * f[2][0]
        g = [f[d][1] * f[(d + 1) % 3][0] * f[(d + 2) % 3][0] for d in range(3)]
        vals.append(val)
        du.append(sum(g[d] * dlam[d][0] for d in range(3)))
        dv.append(sum(g[d] * dlam[d][1] for d in range(3)))
    return np.array(vals), np.array(du), np.array(dv)


def p2_sphere_quadrature(nsub: int = 36, radius: float = 1.0) -> Quadrature:
    """Unit sphere as 8·nsub² quadratic triangles with the VR-6 rule.

    Octahedron faces subdivided into nsub² flat triangles; the 6 P2 nodes of
    each (vertices and edge midpoints of the flat triangle) are projected
    radially onto the sphere, vertices ordered so that t₁ × t₂ points
    outward.  nsub = 36 gives 10,368 elements and N = 62,208.
    """
    X, W = VR4N6
    B, Bu, Bv = _p2_basis(X[:, 0], X[:, 1])  # (6 basis, 6 qpts)
    faces = []
    for sx in (1, -1):
        for sy in (1, -1):
            for sz in (1, -1):
                a = np.array([sx, 0, 0.0])
                b = np.array([0, sy, 0.0])
                c = np.array([0, 0, sz * 1.0])
                # orient so that (b - a) x (c - a) points away from origin
                if np.dot(np.cross(b - a, c - a), a + b + c) < 0:
                    b, c = c, b
                faces.append((a, b, c))
    tri = []
    for a, b, c in faces:
        e1 = (b - a) / nsub
        e2 = (c - a) / nsub
        for i in range(nsub):
            for j in range(nsub - i):
                p0 = a + i * e1 + j * e2
                tri.append((p0, p0 + e1, p0 + e2))  # upward
                if i + j < nsub - 1:
                    tri.append((p0 + e1, p0 + e1 + e2, p0 + e2))  # downward
    tri = np.array(tri)  # (nel, 3, 3): vertices v0 (ref (0,0)), v1 (1,0), v2 (0,1)
    v0, v1, v2 = tri[:, 0], tri[:, 1], tri[:, 2]
    # node positions at reference nodes (0,0),(½,0),(1,0),(0,½),(½,½),(0,1)
    ref = [(0, 0), (0.5, 0), (1, 0), (0, 0.5), (0.5, 0.5), (0, 1)]
    nodes = np.stack([v0 + s * (v1 - v0) + t * (v2 - v0) for s, t in ref], axis=1)
    nodes = radius * nodes / np.linalg.norm(nodes, axis=-1, keepdims=True)
    x = np.einsum("kq,ekd->eqd", B, nodes)
    tu = np.einsum("kq,ekd->eqd", Bu, nodes)
    tv = np.einsum("kq,ekd->eqd", Bv, nodes)
    cr = np.cross(tu, tv)
    mu = np.linalg.norm(cr, axis=-1)
    w = mu * W[None, :]
    nrm = cr / mu[..., None]
    q = Quadrature(x.reshape(-1, 3), nrm.reshape(-1, 3), w.reshape(-1), 6,
                   {"kind": "surface", "shape": "p2sphere", "nsub": nsub})
    return q


# ----------------------------------------------------------------------------
# volumes (2D): the unit disk in curved triangles
# ----------------------------------------------------------------------------
def _disk_patches(radius: float, a: float):
    """Five maps [0,1]^2 -> disk: the central square [-a, a]^2 and four
    transfinite patches blending a square edge into a quarter of the circle
    (P(s,t) = (1-t) L(s) + t C(s)).  Each returns (points, Jacobian det)."""

    def centre(s, t):
        x = np.stack([-a + 2 * a * s, -a + 2 * a * t], axis=-1)
        return x, np.full(s.shape, 4 * a * a)

    def outer(k):
        c, sn = np.cos(k * np.pi / 2), np.sin(k * np.pi / 2)
        rot = np.array([[c, -sn], [sn, c]])

        def f(s, t):
            L = np.stack([np.full(s.shape, a), -a + 2 * a * s], axis=-1)
            dL = np.stack([np.zeros(s.shape), np.full(s.shape, 2 * a)], axis=-1)
            phi = -np.pi / 4 + np.pi / 2 * s
            C = radius * np.stack([np.cos(phi), np.sin(phi)], axis=-1)
            dC = radius * np.pi / 2 * np.stack([-np.sin(phi), np.cos(phi)], axis=-1)
            x = (1 - t)[..., None] * L + t[..., None] * C
            xs = (1 - t)[..., None] * dL + t[..., None] * dC
            xt = C - L
            det = np.abs(xs[..., 0] * xt[..., 1] - xs[..., 1] * xt[..., 0])
            return x @ rot.T, det

        return f

    return [centre] + [outer(k) for k in range(4)]


def disk_triangle_quadrature(m: int, radius: float = 1.0, a: float | None = None) -> Quadrature:
    """The disk of the given radius as 5 patches x m x m cells x 2 curved
    triangles (10 m^2 elements), each with the 6-point Vioreanu-Rokhlin rule
    (nq = 6) mapped through its patch: x = P(A x^), w = w^ |det A| |det DP|.
    A volume quadrature for the volume potential (no normals)."""
    a = 0.5 * radius if a is None else a
    xh, wh = VR4N6
    h = 1.0 / m
    tri = []
    for i in range(m):
        for j in range(m):
            s0, s1, t0, t1 = i * h, (i + 1) * h, j * h, (j + 1) * h
            tri.append(((s0, t0), (s1, t0), (s0, t1)))
            tri.append(((s1, t1), (s0, t1), (s1, t0)))
    tri = np.array(tri)  # (2m^2, 3, 2) in patch coordinates
    V0, E1, E2 = tri[:, 0], tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0]
    detA = np.abs(E1[:, 0] * E2[:, 1] - E1[:, 1] * E2[:, 0])
    st = V0[:, None, :] + xh[None, :, 0:1] * E1[:, None, :] + xh[None, :, 1:2] * E2[:, None, :]
    coords, weights = [], []
    for patch in _disk_patches(radius, a):
        x, det = patch(st[..., 0], st[..., 1])
        coords.append(x.reshape(-1, 2))
        weights.append((wh[None, :] * detA[:, None] * det).reshape(-1))
    q = Quadrature(np.concatenate(coords), None, np.concatenate(weights), len(wh))
    q.meta.update(shape="disk", radius=radius, order=4)
    return q


# ----------------------------------------------------------------------------
# volumes (3D): the ball in curved hexahedra
# ----------------------------------------------------------------------------
def _cube_rule(order: int):
    """TensorProductQuadrature(GL, GL, GL) on [0,1]³, first coordinate fastest."""
    x, w = gauss_legendre_for_order(order)
    X = np.array([[a, b, c] for c in x for b in x for a in x])
    W = np.array([wa * wb * wc for wc in w for wb in w for wa in w])
    return X, W


def _ball_blocks(radius: float, a: float):
    """Seven maps [0,1]³ -> ball: the central cube [-a, a]³ and six blocks
    blending a face of that cube into the matching cube-sphere patch of the
    bounding sphere, P(s,t,ρ) = (1-ρ) L(s,t) + ρ C(s,t) with C = R p/|p| for
    p on the unit cube face (the patch map of `ellipsoid_quadrature`).  Each
    returns (points, |det DP|)."""

    def centre(s, t, r):
        x = np.stack([-a + 2 * a * s, -a + 2 * a * t, -a + 2 * a * r], axis=-1)
        return x, np.full(s.shape, 8 * a ** 3)

    def outer(pid):
        def f(s, t, r):
            u, v = -1 + 2 * s, -1 + 2 * t
            p, pu, pv = unit_sphere_patch(u, v, pid)
            L, Lu, Lv = a * p, a * pu, a * pv
            xh, xu, xv = _sphere_map(u, v, pid)
            C, Cu, Cv = radius * xh, radius * xu, radius * xv
            rr = r[..., None]
            x = (1 - rr) * L + rr * C
            xs = 2 * ((1 - rr) * Lu + rr * Cu)  # d/ds = 2 d/du
            xt = 2 * ((1 - rr) * Lv + rr * Cv)
            xr = C - L
            det = np.abs(np.sum(xs * np.cross(xt, xr), axis=-1))
            return x, det

        return f

    return [centre] + [outer(pid) for pid in range(1, 7)]


def ball_hex_quadrature(m: int, qorder: int = 5, radius: float = 1.0, a: float | None = None) -> Quadrature:
    """The ball of the given radius as 7 blocks x m³ curved hexahedra
    (7 m³ elements), each with the tensor Gauss-Legendre rule of the given
    order mapped through its block: x = P(y0 + h x̂), w = ŵ h³ |det DP|.
    The outer faces lie on the cube-sphere patches of
    ``ellipsoid_quadrature(·, ·, scaling=(R, R, R))``.  A volume quadrature
    for the volume potential (no normals); meta ``order`` is the rule's
    order (the default VDIM interpolation order)."""
    a = 0.5 * radius if a is None else a
    X, W = _cube_rule(qorder)
    h = 1.0 / m
    cells = np.array([(i, j, k) for k in range(m) for j in range(m) for i in range(m)], dtype=np.float64)
    st = (cells[:, None, :] + X[None, :, :]) * h  # (m³, nq, 3)
    coords, weights = [], []
    for block in _ball_blocks(radius, a):
        x, det = block(st[..., 0], st[..., 1], st[..., 2])
        coords.append(x.reshape(-1, 3))
        weights.append((W[None, :] * h ** 3 * det).reshape(-1))
    q = Quadrature(np.concatenate(coords), None, np.concatenate(weights), len(W))
    q.meta.update(shape="ball", radius=radius, order=qorder)
    return q
