"""Replicas over several processes (gloo on CPU, world size 2 and 3): each
rank solves a round-robin share of the T-matrix columns and rank 0 gathers
the full matrix -- the host logic of the multi-GPU path, with a stand-in
solver whose column j is a known function of j."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from scadyn_b200.replicas import compute_T_matrix_replicated, shard_columns


def test_shards_cover_columns_once():
    for ncol in (1, 7, 16, 448):
        for world in (1, 2, 3, 8):
            seen = []
            sizes = []
            for r in range(world):
                cols = shard_columns(ncol, r, world)
                assert np.all(cols % world == r)
                seen += list(cols)
                sizes.append(len(cols))
            assert sorted(seen) == list(range(ncol))
            assert max(sizes) - min(sizes) <= 1


def test_shards_balance_column_orders():
    """Each rank's share spans every VSWF order: with a cost that grows with
    the order n of column c (2nm columns, order n holds 2(2n+1) of them), the
    round-robin shares of 8 ranks differ by under 5 %, where contiguous runs
    would differ by more than 3x."""
    Nmax = 14
    n_of = np.concatenate([[n] * (2 * n + 1) for n in range(1, Nmax + 1)] * 2)
    cost = n_of.astype(float) ** 2
    ncol = len(cost)
    shares = [cost[shard_columns(ncol, r, 8)].sum() for r in range(8)]
    assert max(shares) / min(shares) < 1.05
    runs = [cost[np.array_split(np.arange(ncol), 8)[r]].sum() for r in range(8)]
    assert max(runs) / min(runs) > 3


class _Stub:
    """compute_T_columns stand-in: column j of the (ncol, ncol) result is
    (j + 1) * [1, 2, ..., ncol] * (1 + 1j)."""

    def compute_T_columns(self, Nmax, cols, **kw):
        n = 2 * ((Nmax + 1) ** 2 - 1)
        cols = np.asarray(cols)
        T = np.outer(np.arange(1, n + 1), cols + 1) * (1 + 1j)
        return T, np.full(len(cols), 7, np.int32)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    T, it = compute_T_matrix_replicated(_Stub(), 3, rank, world)
    if rank == 0:
        q.put(T)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_gather_assembles_full_T(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    T = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    full, _ = _Stub().compute_T_columns(3, np.arange(30))
    assert np.array_equal(T, full)
