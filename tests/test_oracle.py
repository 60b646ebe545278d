"""The CPU oracle checked against an independent numpy/scipy restatement and
against physics (Mie series, reciprocity).  No GPU needed."""
import numpy as np
import pytest

from oracle import oracle as O
from tests import np_restate as R


def crand(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def test_pinv_matches_numpy(rng):
    A = rng.standard_normal((98, 27)) + 1j * rng.standard_normal((98, 27))
    # Fortran (98,27) column-major == C array (27,98)
    Af = np.ascontiguousarray(A.T)
    P = O.pinv(Af)                       # memory (27,98) Fortran -> C (98,27)
    ref = np.linalg.pinv(A)              # (27,98)
    np.testing.assert_allclose(P.T, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_fft1d_matches_numpy(rng):
    for L in (8, 12, 20, 34, 64, 68):
        x = crand(rng, L)
        y = np.ascontiguousarray(x.copy())
        O.lib().orc_fft1d(L, O._p(y), -1)
        np.testing.assert_allclose(y, np.fft.fft(x), atol=1e-12 * L)


def test_pruned_fft_convolution_is_exact(rng):
    N = (6, 5, 4)
    Px, Py, Pz = 2 * N[0], 2 * N[1], 2 * N[2]
    A = np.zeros((Pz, Py, Px), np.complex128)
    A[: N[2], : N[1], : N[0]] = crand(rng, N[0] * N[1] * N[2]).reshape(N[2], N[1], N[0])
    F = crand(rng, Px * Py * Pz).reshape(Pz, Py, Px)
    a = O.fft3d_pruned(A, inverse=False)
    b = O.fft3d_pruned(F * a, inverse=True)
    full = np.fft.ifftn(F * np.fft.fftn(A)) * (Px * Py * Pz)
    np.testing.assert_allclose(b[: N[2], : N[1], : N[0]], full[: N[2], : N[1], : N[0]],
                               atol=1e-11 * np.abs(full).max())


def test_build_G_matches_numpy(small_op):
    g = small_op.geom
    Fg = small_op.Fg                                 # (2Nz,2Ny,2Nx)
    ref = R.build_G(g.Nx, g.Ny, g.Nz, g.delta, g.min_coord, g.k)
    np.testing.assert_allclose(Fg.transpose(2, 1, 0), ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_geometry_invariants(small_op):
    g = small_op.geom
    assert g.Nx % 2 == 0 and g.Ny % 2 == 0 and g.Nz % 2 == 0
    assert g.N_cubes == np.prod(g.cube_dims)
    tets = g.tetras[g.tetras > 0]
    assert np.array_equal(np.sort(tets), np.arange(1, g.T + 1))
    # every tet's box nodes are the 27 nodes of its cube (indS == etopol_box of the cube)
    cube_of = np.zeros(g.T + 1, int)
    for c in range(g.N_cubes):
        for t in g.tetras[c]:
            if t:
                cube_of[t] = c
    np.testing.assert_array_equal(small_op.indS, g.etopol_box[cube_of[1:]])


def test_near_zone_count_is_symmetric_half(small_op):
    ind = small_op.sp_ind
    assert np.all(ind[:, 1] >= ind[:, 0])
    pairs = set(map(tuple, ind.tolist()))
    assert len(pairs) == ind.shape[0]                 # no duplicate block
    diag = ind[ind[:, 0] == ind[:, 1]]
    assert diag.shape[0] == small_op.geom.T           # one self block per tet


def test_near_zone_self_block_carries_inverse_contrast(small_op, small_sphere):
    """Self blocks hold 1/(eps-1) I plus an eps-independent part
    (src/precorrection.f90:226-231): changing eps moves only that term."""
    g = small_op.geom
    eps2 = 3.1 + 0.2j
    g2 = O.Geometry(small_sphere.coord, small_sphere.etopol,
                    np.full(g.T, eps2), k=g.k, grid_size=1.8)
    sp2, ind2 = g2.nearzone(small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, fp64=True)
    sp1, ind1 = g.nearzone(small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, fp64=True)
    np.testing.assert_array_equal(ind1, ind2)
    d = np.where(ind1[:, 0] == ind1[:, 1])[0]
    diff = sp2[d] - sp1[d]
    want = (1 / (eps2 - 1) - 1 / (2.25 + 0.01j - 1)) * np.eye(3)
    np.testing.assert_allclose(diff, np.broadcast_to(want, diff.shape), atol=1e-12)
    off = np.where(ind1[:, 0] != ind1[:, 1])[0]
    np.testing.assert_array_equal(sp2[off], sp1[off])
    # the stored complex64 blocks are the FP64 blocks rounded (src/precorrection.f90:251)
    np.testing.assert_array_equal(small_op.sp_mat, sp1.astype(np.complex64))


@pytest.mark.parametrize("merged", [False, True])
def test_compute_Ax2_matches_numpy(small_op, rng, merged):
    g = small_op.geom
    x = crand(rng, 3 * g.T)
    small_op.merged = merged
    y = small_op.compute_Ax2(x)
    small_op.merged = False
    ref = R.compute_Ax2(x, small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, small_op.indS,
                        small_op.Fg, small_op.sp_mat, small_op.sp_ind, g.k, g.Nx, g.Ny, g.Nz, merged=merged)
    np.testing.assert_allclose(y, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_merged_convolutions_agree_with_six(small_op, rng):
    x = crand(rng, 3 * small_op.geom.T)
    small_op.merged = False
    a = small_op.compute_Ax2(x)
    small_op.merged = True
    b = small_op.compute_Ax2(x)
    small_op.merged = False
    assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-13


def test_gmres_matches_numpy_restatement(small_op, small_sphere):
    g = small_op.geom
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, g.k, 2)
    rhs = mat[3]
    x, info = small_op.gmres(rhs, tol=1e-8, m=6, cycles=4)
    xr, ir = R.gmres(small_op.compute_Ax2, rhs, 1e-8, 6, 4)
    assert info["iters"] == ir["iters"]
    np.testing.assert_allclose(info["history"], ir["history"], rtol=1e-7)
    np.testing.assert_allclose(x, xr, rtol=0, atol=1e-10 * np.abs(xr).max())


def test_calc_MN_matches_scipy():
    k = 2.3e7
    Po = np.array([1.1e-8, -0.7e-8, 0.45e-8])
    MM, NN = O.calc_MN(6, k, Po)
    MMr, NNr = R.calc_MN(6, k, Po)
    np.testing.assert_allclose(MM, MMr, rtol=0, atol=1e-12 * np.abs(MMr).max())
    np.testing.assert_allclose(NN, NNr, rtol=0, atol=1e-12 * np.abs(NNr).max())


def test_cspherebessel_matches_scipy():
    from scipy.special import spherical_jn
    for z in (0.3, 2.0, 7.5, 15.0):
        j, _ = O.cspherebessel(12, z)
        np.testing.assert_allclose(j, spherical_jn(np.arange(13), z), rtol=1e-10, atol=1e-14)


def test_jvie_T_matrix_matches_mie_series(small_op, small_sphere):
    """Physics pin: T of a 1680-tet sphere (h = a/4) agrees with the Mie
    coefficients at discretisation level (src/T_matrix.f90:131-168)."""
    g = small_op.geom
    k = g.k
    Nmax = 2
    nm = (Nmax + 1) ** 2 - 1
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, k, Nmax)
    X = np.zeros_like(mat)
    small_op.nthreads = 0
    for c in range(2 * nm):
        X[c], info = small_op.gmres(mat[c], tol=1e-6, m=50, cycles=4)
        assert info["converged"]
    small_op.nthreads = 1
    T = O.T_assemble(mat, X).T * (1j * k ** 3)
    a_n, b_n = O.mie_T(Nmax, k * small_sphere.a, np.sqrt(2.25 + 0.01j))
    for j in range(nm):
        n = int(np.floor(np.sqrt(j + 1)))
        assert abs(T[j, j] - a_n[n - 1]) < 0.08 * abs(a_n[n - 1])
        assert abs(T[nm + j, nm + j] - b_n[n - 1]) < 0.08 * abs(b_n[n - 1])
    # reciprocity-type symmetry: off-diagonal leakage small against the diagonal
    assert np.abs(T[:nm, :nm] - np.diag(np.diag(T[:nm, :nm]))).max() < 0.05 * abs(a_n[0])
