"""Perturbation sharding over ranks: the cyclic distribution of WEST's images
and a two-rank gloo run on CPU whose gathered result equals one rank's (the
operator here is the oracle, as CPU-only ranks have no GPU kernels; the same
sharding through the library's CUDA kernels is tests/test_gpu_multirank.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from west_b200.distribute import PertDistribution, apply_operator_sharded


@pytest.mark.parametrize("nglob,nlevel", [(64, 1), (64, 2), (7, 3), (5, 8)])
def test_cyclic_distribution_covers_every_column_once(nglob, nlevel):
    seen = []
    for r in range(nlevel):
        d = PertDistribution(nglob, nlevel, r)
        cols = d.local_columns()
        assert len(cols) == d.nloc <= d.nlocx
        for il, ig in enumerate(cols):
            assert d.l2g(il) == ig and d.g2l(ig) == (il, r)
        seen.extend(cols.tolist())
    assert sorted(seen) == list(range(nglob))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from oracle import west_oracle as O
    from west_b200.system import build_system, perturbations
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = build_system("tiny")
        dvg = perturbations(s, 5)
        d = PertDistribution(5, world, rank)
        dng, ierr, cols = apply_operator_sharded(lambda v, t: O.apply_operator(s, v, t), dvg, 1e-12, d)
        # gather to rank 0 (test only: apply_operator itself exchanges nothing)
        buf = np.zeros((s.npw, d.nlocx), complex)
        buf[:, :dng.shape[1]] = dng
        parts = [torch.zeros(2 * s.npw * d.nlocx, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(parts, torch.from_numpy(buf.view(np.float64).ravel().copy()))
        if rank == 0:
            full = np.zeros((s.npw, 5), complex)
            for r in range(world):
                blk = parts[r].numpy().view(complex).reshape(s.npw, d.nlocx)
                c = d.local_columns(r)
                full[:, c] = blk[:, :len(c)]
            ref, _ = O.apply_operator(s, dvg, 1e-12)
            out.put(float(np.abs(full - ref).max() / np.abs(ref).max()))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_sharding_matches_single_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert q.get(timeout=10) < 1e-13


@pytest.mark.parametrize("col0,m,nranks", [(0, 4, 2), (5, 7, 2), (8, 3, 4), (16, 1, 3)])
def test_batch_rows_split_the_batch(col0, m, nranks):
    from west_b200.distribute import batch_owner_rows
    rows = [batch_owner_rows(col0, m, nranks, r) for r in range(nranks)]
    assert sorted(sum(rows, [])) == list(range(m))
    for r in range(nranks):
        assert all((col0 + i) % nranks == r for i in rows[r])


def _gather_main(rank, world, port, out):
    import torch
    import torch.distributed as dist
    from west_b200.distribute import batch_owner_rows, gather_batch
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(3)
        ok = True
        for col0, m in ((0, 4), (5, 7), (9, 1)):
            x = torch.randn((m, 11), generator=g, dtype=torch.complex128)    # same on every rank
            rows = batch_owner_rows(col0, m, world, rank)
            local = 2.0 * x[rows] + 1j                                        # this rank's share of the operator
            full = gather_batch(local, col0, m, world, rank)
            ok = ok and bool(torch.equal(full, 2.0 * x + 1j))
        out.put((rank, ok))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_batch_gather():
    """The exchange step of the sharded Davidson apply: each rank's rows of a batch,
    all-gathered, reassemble the batch in its original order on every rank."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: True, 1: True}
