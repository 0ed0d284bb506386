"""Target-row sharding of one operator across ranks (one GPU per rank).

Every target row of ``y = (A + δ)σ`` is independent: rank r holds all
sources and computes the contiguous row block ``rows(n, world)[r]``; the
blocks are put back together by one all-gather of y (the exchange step of an
iterative solve, where y feeds the next product).  The correction is
row-partitioned with the same split.  This module holds the host-side
bookkeeping only; the apply itself is the ordinary GPU operator on a target
subset and the gather is the caller's collective.
"""
from __future__ import annotations

import numpy as np

from .geometry import Quadrature


def row_blocks(n: int, world: int) -> list[tuple[int, int]]:
    """Balanced contiguous blocks ``[r0, r1)`` covering ``0..n-1`` (the first
    ``n % world`` blocks one row longer).  Every rank gets a block, possibly
    empty when ``n < world``."""
    if world < 1:
        raise ValueError("world must be >= 1")
    base, extra = divmod(int(n), int(world))
    out, r0 = [], 0
    for r in range(world):
        r1 = r0 + base + (1 if r < extra else 0)
        out.append((r0, r1))
        r0 = r1
    return out


def padded_rows(n: int, world: int) -> int:
    """Rows per rank of the all-gather buffer (the longest block), so that
    every rank sends the same count."""
    return -(-int(n) // int(world))


def target_block(q: Quadrature, r0: int, r1: int) -> Quadrature:
    """Rows ``r0..r1-1`` of q as a target set (coordinates and normals kept;
    no element structure: only the source side needs it)."""
    nrm = None if q.normals is None else q.normals[r0:r1]
    return Quadrature(q.coords[r0:r1], nrm, q.weights[r0:r1], 0)


def slice_csr_rows(indptr, indices, data, r0: int, r1: int):
    """Rows ``r0..r1-1`` of a CSR matrix as a CSR matrix of its own."""
    indptr = np.asarray(indptr)
    a, b = int(indptr[r0]), int(indptr[r1])
    return (indptr[r0:r1 + 1] - a).astype(np.int64), np.asarray(indices)[a:b].copy(), np.asarray(data)[a:b].copy()


def unpad(gathered: np.ndarray, n: int, world: int) -> np.ndarray:
    """Undo the padding of an all-gather of ``padded_rows`` rows per rank."""
    p = padded_rows(n, world)
    blocks = row_blocks(n, world)
    g = np.asarray(gathered).reshape(world, p, *np.asarray(gathered).shape[1:])
    return np.concatenate([g[r, : r1 - r0] for r, (r0, r1) in enumerate(blocks)], axis=0)
