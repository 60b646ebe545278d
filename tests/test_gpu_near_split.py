"""The FP64 near-zone kernel with split row and column sums
(scd_grid_desc.near_split = 2, the default: two lanes per sum at one
right-hand side, two partial sums per lane at four): the FP64 matvec against
the oracle, solutions against the one-sum kernel (near_split = 1), and
bit-identical columns alone and in batches (the mixed form's complex64
kernels are left unsplit)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_helpers import solver_from_oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _solver(op, split):
    return solver_from_oracle(op, near_split=2 if split else 1)


@pytest.fixture(scope="module")
def split_solver(small_op):
    s = _solver(small_op, True)
    yield s
    s.close()


def test_split_matvec_matches_oracle(split_solver, small_op):
    rng = np.random.default_rng(31)
    x = rng.standard_normal(split_solver.n) + 1j * rng.standard_normal(split_solver.n)
    assert rel(split_solver.compute_Ax2(x), small_op.compute_Ax2(x)) < 1e-11


def test_split_columns_bitwise_equal_single(split_solver, small_op, small_sphere):
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 2)
    T1, it1, X1, _ = split_solver.solve_columns(mat, tol=1e-8, block=1, want_x=True)
    T4, it4, X4, _ = split_solver.solve_columns(mat, tol=1e-8, block=4, want_x=True)
    T16, it16, X16, _ = split_solver.solve_columns(mat, tol=1e-8, block=16, want_x=True)
    assert np.array_equal(it1, it4) and np.array_equal(it1, it16)
    assert np.array_equal(X1, X4) and np.array_equal(X1, X16)
    assert np.array_equal(T1, T4) and np.array_equal(T1, T16)
    x, info = split_solver.gmres(mat[3], tol=1e-8, m=50, cycles=4)
    assert info["iters"] == it1[3] and np.array_equal(x, X1[3])
    # the same solutions as the default kernel, to the GMRES tolerance
    d = _solver(small_op, False)
    try:
        Td, itd, Xd, _ = d.solve_columns(mat, tol=1e-8, block=4, want_x=True)
    finally:
        d.close()
    assert np.abs(it1.astype(int) - itd.astype(int)).max() <= 1
    assert rel(X1, Xd) < 1e-7


def test_split_mixed_batch_invariant(split_solver, small_op, small_sphere):
    from scadyn_b200 import api
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    a = split_solver.solve_columns(mat, tol=1e-8, block=1, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True)
    b = split_solver.solve_columns(mat, tol=1e-8, block=6, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True)
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
