"""Row sharding of one operator over ranks: the host-side bookkeeping of the
multi-GPU mode, run as world_size-2 gloo ranks on the CPU.  Each rank forms
its row block of (A + δD)σ for the kite (the oracle stands in for the GPU
apply here) and the blocks travel through the same padded all-gather the
bench uses; the result must equal the single-process product bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle as O
from inti_b200 import geometry as G
from inti_b200 import shard as SH


def test_row_blocks_cover_and_balance():
    for n, w in [(10, 3), (3, 8), (62208, 8), (1, 1), (0, 2)]:
        b = SH.row_blocks(n, w)
        assert len(b) == w and b[0][0] == 0 and b[-1][1] == n
        assert all(b[i][1] == b[i + 1][0] for i in range(w - 1))
        sizes = [r1 - r0 for r0, r1 in b]
        assert max(sizes) - min(sizes) <= 1 and max(sizes) <= SH.padded_rows(n, w)


def test_slice_csr_rows_roundtrip():
    r = np.random.default_rng(0)
    lens = r.integers(0, 5, 20)
    indptr = np.concatenate([[0], np.cumsum(lens)])
    indices = r.integers(0, 30, indptr[-1]).astype(np.int32)
    data = r.standard_normal(indptr[-1])
    parts = [SH.slice_csr_rows(indptr, indices, data, r0, r1) for r0, r1 in SH.row_blocks(20, 3)]
    assert np.array_equal(np.concatenate([p[1] for p in parts]), indices)
    assert np.array_equal(np.concatenate([p[2] for p in parts]), data)
    assert sum(len(p[0]) - 1 for p in parts) == 20


def _problem():
    q = G.kite_quadrature(40, 9)
    dS, dD = O.bdim(O.LAPLACE, 0.0, q.coords, q.normals, q.weights, q.nq)
    indptr, indices, data = O.block_csr(dD, q.nq, None, len(q))
    sigma = np.random.default_rng(1).standard_normal(len(q))
    return q, (indptr, indices, data), sigma


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q, (indptr, indices, data), sigma = _problem()
        n = len(q)
        r0, r1 = SH.row_blocks(n, world)[rank]
        tq = SH.target_block(q, r0, r1)
        y = O.apply(O.LAPLACE, O.DL, 0.0, tq.coords, tq.normals, q.coords, q.normals, q.weights, sigma)
        ip, ix, dv = SH.slice_csr_rows(indptr, indices, data, r0, r1)
        y = y + O.csr_apply(ip, ix, dv, sigma)
        p = SH.padded_rows(n, world)
        send = torch.zeros(p, dtype=torch.float64)
        send[: r1 - r0] = torch.from_numpy(y)
        recv = torch.zeros(world * p, dtype=torch.float64)
        dist.all_gather(list(recv.view(world, p).unbind(0)), send)  # NCCL: all_gather_into_tensor
        if rank == 0:
            out.put(SH.unpad(recv.numpy(), n, world))
    finally:
        dist.destroy_process_group()


def test_row_sharded_product_matches_single_process():
    q, (indptr, indices, data), sigma = _problem()
    full = O.apply(O.LAPLACE, O.DL, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights, sigma) + \
        O.csr_apply(indptr, indices, data, sigma)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    world = 2
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = out.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.array_equal(got, full)


def _rank_items(rank, world, port, out):
    """The item-shard exchange: each rank holds a share of the pair terms of
    the product over all rows (here: the source columns j with j % world ==
    rank, a stand-in for its work items), rank 0 adds the correction, and one
    all-reduce sums the partials (NCCL all_reduce on the GPUs)."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        q, (indptr, indices, data), sigma = _problem()
        part = np.where(np.arange(len(q)) % world == rank, sigma, 0.0)
        y = O.apply(O.LAPLACE, O.DL, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights, part)
        if rank == 0:
            y = y + O.csr_apply(indptr, indices, data, sigma)
        t = torch.from_numpy(y)
        dist.all_reduce(t)
        if rank == 0:
            out.put(t.numpy())
    finally:
        dist.destroy_process_group()


def test_item_sharded_product_matches_single_process():
    q, (indptr, indices, data), sigma = _problem()
    full = O.apply(O.LAPLACE, O.DL, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights, sigma) + \
        O.csr_apply(indptr, indices, data, sigma)
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    world = 2
    procs = [ctx.Process(target=_rank_items, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    got = out.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert np.max(np.abs(got - full)) <= 1e-13 * np.max(np.abs(full))
