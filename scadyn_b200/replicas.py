"""Several GPUs: replicas, one process per GPU.

T-matrix columns are independent solves against a read-only operator
(src/T_matrix.f90:254-268), so every rank builds its own copy of the operator
and solves its share of the columns; the only exchange is one gather of the
column blocks to rank 0 at the end (torch.distributed: NCCL between GPUs,
gloo on CPU for the tests).  There is no collective inside a solve.

Shares are dealt round-robin (rank r takes columns r, r + W, r + 2W, ...):
the cost of a column grows with its VSWF order, and the column loop runs
through the orders in turn, so contiguous runs would give the last ranks
the slowest columns.
"""
from __future__ import annotations

import numpy as np


def shard_columns(ncol: int, rank: int, world: int) -> np.ndarray:
    """This rank's 0-based columns of ncol: rank, rank + world, ... (sizes
    differ by at most one across ranks)."""
    return np.arange(rank, ncol, world, dtype=np.int32)


def gather_columns(T_local: np.ndarray, ncol: int, rank: int, world: int, group=None, device=None):
    """Collect every rank's (nrow, count) column block into the full
    (nrow, ncol) matrix on rank 0 (None elsewhere), each column at its index
    in the round-robin deal.  Blocks travel as float64 pairs padded to the
    largest share."""
    import torch
    import torch.distributed as dist
    nrow = T_local.shape[0]
    width = -(-ncol // world)
    buf = np.zeros((nrow, width), np.complex128)
    buf[:, :T_local.shape[1]] = T_local
    t = torch.from_numpy(np.ascontiguousarray(buf).view(np.float64).copy())
    if device is not None:
        t = t.to(device)
    parts = [torch.zeros_like(t) for _ in range(world)] if rank == 0 else None
    dist.gather(t, gather_list=parts, dst=0, group=group)
    if rank != 0:
        return None
    T = np.zeros((nrow, ncol), np.complex128)
    for r, p in enumerate(parts):
        cols = shard_columns(ncol, r, world)
        T[:, cols] = p.cpu().numpy().view(np.complex128)[:, :len(cols)]
    return T


def compute_T_matrix_replicated(solver, Nmax: int, rank: int, world: int, group=None, device=None, **opts):
    """This rank's columns of compute_T_matrix on its own GPU
    (scd_compute_T_columns), gathered on rank 0: returns (T (2nm, 2nm) on
    rank 0 else None, this rank's iteration counts in its column order)."""
    ncol = 2 * ((Nmax + 1) ** 2 - 1)
    cols = shard_columns(ncol, rank, world)
    if len(cols) > 0:
        T_loc, iters = solver.compute_T_columns(Nmax, cols, **opts)
    else:
        T_loc, iters = np.zeros((ncol, 0), np.complex128), np.zeros(0, np.int32)
    return gather_columns(T_loc, ncol, rank, world, group=group, device=device), iters
