"""Host-side quadrature construction (mirrors meshgen + Quadrature)."""
import numpy as np

from inti_b200 import geometry as G


def test_workload_sizes():
    assert len(G.kite_quadrature()) == 1000
    assert G.kite_quadrature().nq == 5
    q = G.p2_sphere_quadrature(36)
    assert len(q) == 62208 and q.nq == 6 and q.nel == 10368
    assert len(G.ellipsoid_quadrature(61, 5)) == 200934


def test_element_blocks_are_contiguous():
    q = G.ellipsoid_quadrature(2, 5)
    tags = q.etype2qtags()
    assert tags.shape == (9, 24)
    assert (tags[:, 3] == np.arange(27, 36)).all()


def test_normals_unit_and_outward():
    for q in (G.kite_quadrature(50, 9), G.ellipsoid_quadrature(4, 5), G.p2_sphere_quadrature(4),
              G.star_quadrature(G.star_coefficients(np.random.default_rng(0)), 4)):
        assert np.allclose(np.linalg.norm(q.normals, axis=1), 1.0)
        c = q.coords - q.coords.mean(0)
        assert np.min(np.sum(c * q.normals, 1)) > 0  # star-shaped about the centroid


def test_p2_sphere_area_and_volume():
    q = G.p2_sphere_quadrature(12)
    assert abs(q.integrate(lambda x: 1.0) - 4 * np.pi) < 2e-4
    vol = np.sum(np.sum(q.coords * q.normals, 1) * q.weights) / 3
    assert abs(vol - 4 / 3 * np.pi) < 2e-4


def test_star_radius_bounds():
    a = G.star_coefficients(np.random.default_rng(7))
    q = G.star_quadrature(a, 6)
    r = np.linalg.norm(q.coords, axis=1)
    assert r.min() >= 0.8 - 1e-9 and r.max() <= 1.2 + 1e-9


def test_kite_perimeter_converges():
    p1 = G.kite_quadrature(200, 9).integrate(lambda x: 1.0)
    p2 = G.kite_quadrature(400, 15).integrate(lambda x: 1.0)
    assert abs(p1 - p2) < 1e-12


def test_gauss_legendre_exactness():
    for n in range(1, 12):
        x, w = G.gauss_legendre(n)
        for p in range(2 * n):
            assert abs(np.sum(w * x**p) - 1.0 / (p + 1)) < 1e-14
