"""Autotuned launch shape of the pair kernel (targets per thread, source
split): operators above 2^26 pairs time their candidates once at creation.
Whatever shape is picked, the product is the same operator: it agrees with
an untuned context's to summation-order rounding and with the oracle's rows."""
import numpy as np
import pytest

import inti_b200 as inti
import oracle as O
from helpers import density, oracle_apply, relerr
from inti_b200 import geometry as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("symmetric", [True, False])
def test_autotuned_shape_gives_the_same_operator(symmetric):
    """Both forms of the square operator: symmetric (split = source blocks
    per work item, untuned default 2 targets per thread) and one-sided."""
    q = G.p2_sphere_quadrature(14)  # 9,408 nodes: 8.9e7 pairs, above the tuning threshold
    op = inti.Helmholtz(k=10.0, dim=3)
    tuned, plain = inti.Context(0), inti.Context(0)
    plain.set_autotune(False)
    for c in (tuned, plain):
        c.set_symmetric(symmetric)
    sigma = density(len(q), True, 5)
    A = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", tuned)
    B = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", plain)
    ta, tb = A.tuning, B.tuning
    assert ta["symmetric"] == tb["symmetric"] == symmetric
    assert ta["targets_per_thread"] in (2, 4) and 1 <= ta["split"] <= 256
    assert tb["targets_per_thread"] == (2 if symmetric else 4)
    # the choice is cached per context and problem shape
    assert inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", tuned).tuning == ta
    ya, yb = A @ sigma, B @ sigma
    assert relerr(ya, yb) < 1e-13
    rows = np.arange(0, len(q), 97)
    assert relerr(ya[rows], oracle_apply(O.HELMHOLTZ, O.SL, 10.0, q, q, sigma, rows=rows)) < 1e-12


def test_small_operators_keep_the_heuristic_shape():
    q = G.p2_sphere_quadrature(4)
    op = inti.Helmholtz(k=10.0, dim=3)
    tuned, plain = inti.Context(0), inti.Context(0)
    plain.set_autotune(False)
    A = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", tuned)
    B = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, None, "fp64", plain)
    assert A.tuning == B.tuning


@pytest.mark.parametrize("kname", ["SL", "DL"])
def test_few_targets_many_source_chunks(ctx, kname):
    """A potential at a few hundred points from 21,600 sources: one or two
    target blocks, so the heuristic cuts the sources into more than 64
    chunks; the product still matches the oracle."""
    q = G.ellipsoid_quadrature(20, 5)
    d = np.random.default_rng(4).standard_normal((300, 3))
    tgt = inti.points(1.7 * d / np.linalg.norm(d, axis=1, keepdims=True))
    op = inti.Helmholtz(k=3.0, dim=3)
    K, okind = (inti.SingleLayerKernel, O.SL) if kname == "SL" else (inti.DoubleLayerKernel, O.DL)
    A = inti.GpuOperator(K(op), tgt, q, None, "fp64", ctx)
    assert A.tuning["split"] > 64
    sigma = density(len(q), True, 8)
    ref = O.apply(O.HELMHOLTZ, okind, 3.0, tgt.coords, None, q.coords, q.normals, q.weights, sigma)
    assert relerr(A @ sigma, ref) < 1e-12
