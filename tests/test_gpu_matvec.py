"""Parity of the device matvec and GMRES with the CPU oracle on the same
operator data (complex FP64).  Tolerances: the device merges the three
cross-component convolutions and may use longer FFT lengths than 2N, so
results agree with the reference's six-convolution form to rounding (1e-11
relative)."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

RTOL_MV = 1e-11


def crand(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)




def test_matvec_matches_oracle(small_op, dev_small, rng):
    x = crand(rng, 3 * small_op.geom.T)
    small_op.merged = False
    ref = small_op.compute_Ax2(x)
    y = dev_small.compute_Ax2(x)
    assert rel(y, ref) < RTOL_MV


def test_matvec_is_linear(dev_small, rng, small_op):
    n = 3 * small_op.geom.T
    x1, x2 = crand(rng, n), crand(rng, n)
    a = 0.3 - 1.7j
    y = dev_small.compute_Ax2(x1 + a * x2)
    y2 = dev_small.compute_Ax2(x1) + a * dev_small.compute_Ax2(x2)
    assert rel(y, y2) < 1e-13


def test_matvec_deterministic(dev_small, rng, small_op):
    x = crand(rng, 3 * small_op.geom.T)
    a = dev_small.compute_Ax2(x)
    b = dev_small.compute_Ax2(x)
    assert np.array_equal(a, b)


def test_matvec_unit_vectors(dev_small, small_op):
    """A few columns of A: unit vectors hit single scatter entries."""
    n = 3 * small_op.geom.T
    for i in (0, 1, n // 2, n - 1):
        e = np.zeros(n, np.complex128)
        e[i] = 1.0
        assert rel(dev_small.compute_Ax2(e), small_op.compute_Ax2(e)) < RTOL_MV


def test_gmres_matches_oracle_iteration_count(small_op, dev_small, small_sphere):
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 2)
    for col in (0, 5, 9):
        xr, ir = small_op.gmres(mat[col], tol=1e-6, m=50, cycles=4)
        x, info = dev_small.gmres(mat[col], tol=1e-6, m=50, cycles=4)
        assert info["iters"] == ir["iters"]
        assert info["converged"]
        assert abs(info["relres"] - ir["relres"]) <= 1e-6 * ir["relres"]
        assert rel(x, xr) < 1e-9


def test_gmres_restart_path(small_op, dev_small, small_sphere):
    """Small Krylov dimension forces restarts (src/gmres_module.f90:305-314)."""
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    xr, ir = small_op.gmres(mat[2], tol=1e-9, m=3, cycles=6)
    x, info = dev_small.gmres(mat[2], tol=1e-9, m=3, cycles=6)
    assert info["iters"] == ir["iters"]
    assert rel(x, xr) < 1e-9


def test_gmres_zero_rhs(dev_small, small_op):
    x, info = dev_small.gmres(np.zeros(3 * small_op.geom.T, np.complex128), tol=1e-6)
    assert np.all(x == 0)


def test_solve_columns_T_matches_oracle(small_op, dev_small, small_sphere):
    Nmax = 2
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, Nmax)
    ncol = mat.shape[0]
    Tc, iters, X, rc = dev_small.solve_columns(mat, tol=1e-8, want_x=True)
    Xr = np.zeros_like(mat)
    for c in range(ncol):
        Xr[c], info = small_op.gmres(mat[c], tol=1e-8, m=50, cycles=4)
        assert iters[c] == info["iters"]
    Tr = O.T_assemble(mat, Xr)
    assert rel(Tc, Tr) < 1e-9
    assert rel(X, Xr) < 1e-9


def test_batched_columns_bitwise_equal_single(small_op, dev_small, small_sphere):
    """Slots solved together give the same bits as one column at a time and
    as scd_gmres (per-column arithmetic does not depend on the batch)."""
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 2)
    T1, it1, X1, _ = dev_small.solve_columns(mat, tol=1e-8, block=1, want_x=True)
    T4, it4, X4, _ = dev_small.solve_columns(mat, tol=1e-8, block=4, want_x=True)
    T16, it16, X16, _ = dev_small.solve_columns(mat, tol=1e-8, block=16, want_x=True)
    assert np.array_equal(it1, it4) and np.array_equal(it1, it16)
    assert np.array_equal(X1, X4) and np.array_equal(X1, X16)
    assert np.array_equal(T1, T4) and np.array_equal(T1, T16)
    for c in (0, 7):
        x, info = dev_small.gmres(mat[c], tol=1e-8, m=50, cycles=4)
        assert info["iters"] == it1[c]
        assert np.array_equal(x, X1[c])


def test_batched_restarts_match_oracle(small_op, dev_small, small_sphere):
    """Small Krylov dimension: slots restart at different ticks."""
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    Tc, it, X, rc = dev_small.solve_columns(mat, tol=1e-9, m=3, cycles=8, block=6, want_x=True)
    for c in range(mat.shape[0]):
        xr, info = small_op.gmres(mat[c], tol=1e-9, m=3, cycles=8)
        assert it[c] == info["iters"]
        assert rel(X[c], xr) < 1e-9


def test_mixed_precision_matches_fp64_oracle(small_op, dev_small, small_sphere):
    """Complex64 inner GMRES + FP64 refinement reaches the FP64 answer: the
    T-matrix relative error against the oracle's FP64 solve stays below 1e-6
    (the target is <= 1e-5)."""
    from scadyn_b200 import api
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 2)
    Tm, itm, Xm, rc = dev_small.solve_columns(mat, tol=1e-9, block=8, precision=api.PREC_MIXED,
                                              inner_tol=1e-4, max_outer=10, want_x=True)
    assert rc == api.SCD_OK
    Xr = np.zeros_like(mat)
    for c in range(mat.shape[0]):
        Xr[c], _ = small_op.gmres(mat[c], tol=1e-11, m=50, cycles=8)
    Tr = O.T_assemble(mat, Xr)
    assert rel(Tm, Tr) < 1e-6
    assert rel(Xm, Xr) < 1e-6
    # the FP64 residual of every column meets the outer tolerance
    for c in (0, 4):
        r = mat[c] - small_op.compute_Ax2(Xm[c])
        assert np.linalg.norm(r) / np.linalg.norm(mat[c]) < 1e-8


def test_mixed_precision_batch_invariant(dev_small, small_op, small_sphere):
    from scadyn_b200 import api
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    a = dev_small.solve_columns(mat, tol=1e-8, block=1, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True)
    b = dev_small.solve_columns(mat, tol=1e-8, block=6, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True)
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(a[2], b[2])
