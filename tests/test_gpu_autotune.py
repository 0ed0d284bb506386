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
    assert ta["targets_per_thread"] in (2, 4) and 1 <= ta["split"] <= 64
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
