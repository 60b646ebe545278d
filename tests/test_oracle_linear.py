"""The oracle's linear-basis matvec (compute_Ax2 with mesh%order = 1,
src/gmres_module.f90:57-176, and matmul_Acorr, src/sparse_mat.f90:64-92) and
the pseudo-tet view the device uses for it: each (tet, node) basis function is
a pseudo-tet with its own projector column and three unknowns, so the far
field of the linear basis equals the constant-basis far field over 4T
pseudo-tets, and the near zone equals 3x3 blocks between pseudo-tets, applied
one-sided inside a tet (the reference adds no transpose when a == b)."""
import dataclasses

import numpy as np
import pytest
import scipy.sparse

from oracle import oracle as O


@pytest.fixture(scope="module")
def ops(small_op):
    op0 = dataclasses.replace(small_op, nthreads=0)
    return op0, O.linear_from_constant(op0, seed=3)


def crand(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def pseudo_x(x1, T):
    """x(12t + 4c + i) -> pseudo-tet 4t + i, component c."""
    return np.ascontiguousarray(x1.reshape(T, 3, 4).transpose(0, 2, 1).reshape(-1))


def sparse_from(n, rows, cols, vals):
    return scipy.sparse.coo_matrix((vals.ravel(), (rows.ravel(), cols.ravel())), shape=(n, n)).tocsr()


def near_matrix(op1, T):
    """Sparse 12T x 12T near-zone matrix from the 12x12 block list."""
    V = op1.sp_mat.astype(np.complex128).transpose(0, 2, 1)      # V[b, r, c] = V(r, c)
    a = 12 * (op1.sp_ind[:, 0] - 1)[:, None, None] + np.arange(12)[None, :, None]
    c = 12 * (op1.sp_ind[:, 1] - 1)[:, None, None] + np.arange(12)[None, None, :]
    a, c = np.broadcast_to(a, V.shape), np.broadcast_to(c, V.shape)
    off = op1.sp_ind[:, 0] != op1.sp_ind[:, 1]
    rows = np.concatenate([a.ravel(), c[off].ravel()])
    cols = np.concatenate([c.ravel(), a[off].ravel()])
    vals = np.concatenate([V.ravel(), V[off].ravel()])
    return sparse_from(12 * T, rows, cols, vals)


def test_matmul_Acorr_matches_block_assembly(ops):
    _, op1 = ops
    T = op1.geom.T
    rng = np.random.default_rng(7)
    x = crand(rng, 12 * T)
    got = O.matmul_Acorr(T, op1.sp_mat, op1.sp_ind, x)
    want = near_matrix(op1, T) @ x
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-13


def test_linear_far_field_is_constant_far_field_over_pseudo_tets(ops):
    op0, op1 = ops
    T = op0.geom.T
    empty = np.zeros((0, 2), np.int32)
    far1 = dataclasses.replace(op1, sp_mat=np.zeros((0, 12, 12), np.complex64), sp_ind=empty)
    pseudo = O.Operator(op0.geom, op1.S, op1.Sx, op1.Sy, op1.Sz, op1.indS, op0.Fg,
                        np.zeros((0, 3, 3), np.complex64), empty, nthreads=0)
    rng = np.random.default_rng(8)
    x1 = crand(rng, 12 * T)
    y1 = far1.compute_Ax2(x1)
    yp = pseudo.compute_Ax2(pseudo_x(x1, T))
    assert np.linalg.norm(pseudo_x(y1, T) - yp) / np.linalg.norm(yp) < 1e-13


def test_pseudo_tet_near_blocks_one_sided_inside_a_tet(ops):
    """The 3x3 pseudo-tet blocks of every 12x12 block, mirrored only between
    different tets, rebuild the near-zone matrix in pseudo-tet order."""
    _, op1 = ops
    T = op1.geom.T
    V = op1.sp_mat.astype(np.complex128).transpose(0, 2, 1)      # V[b, 4c + i, 4c' + j]
    blk = V.reshape(-1, 3, 4, 3, 4).transpose(0, 2, 4, 1, 3)     # [b, i, j, c, c']
    t1, t2 = (op1.sp_ind[:, 0] - 1), (op1.sp_ind[:, 1] - 1)
    ar4, ar3 = np.arange(4), np.arange(3)
    p = 4 * t1[:, None, None, None, None] + ar4[None, :, None, None, None]
    q = 4 * t2[:, None, None, None, None] + ar4[None, None, :, None, None]
    rows = np.broadcast_to(3 * p + ar3[None, None, None, :, None], blk.shape)
    cols = np.broadcast_to(3 * q + ar3[None, None, None, None, :], blk.shape)
    off = t1 != t2                                                # mirrored between different tets only
    P = sparse_from(12 * T, np.concatenate([rows.ravel(), cols[off].ravel()]),
                    np.concatenate([cols.ravel(), rows[off].ravel()]),
                    np.concatenate([blk.ravel(), blk[off].ravel()]))
    A = near_matrix(op1, T)
    perm = pseudo_x(np.arange(12 * T), T)                   # pseudo index -> original index
    D = P - A[perm][:, perm]
    assert D.count_nonzero() == 0 or abs(D).max() == 0


def test_linear_gmres_converges(ops):
    op0, op1 = ops
    T = op0.geom.T
    rng = np.random.default_rng(9)
    b = crand(rng, 12 * T)
    x, info = op1.gmres(b, tol=1e-8, m=50, cycles=8)
    assert info["converged"]
    r = b - op1.compute_Ax2(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-7
