"""Device-side operator construction (build_grid, build_G, projectors, near
zone, VSWF right-hand sides) against the CPU oracle, complex FP64."""
import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import api

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def dev_setup(small_sphere, small_op):
    m = small_sphere
    d = api.grid_from_mesh(m.coord, m.etopol, grid_size=1.8)
    s = api.Solver.from_desc(d)
    s.set_wavenumber(small_op.geom.k)
    s.set_mesh(m.coord, m.etopol, m.param)
    s.build_G()
    proj = s.pfft_projection_const()
    s.compute_near_zone_interactions_const(api.STORE_C128)
    yield s, proj
    s.close()


def test_grid_from_mesh_matches_build_grid(small_sphere, small_op):
    d = api.grid_from_mesh(small_sphere.coord, small_sphere.etopol, grid_size=1.8)
    g = small_op.geom
    assert (d.Nx, d.Ny, d.Nz) == (g.Nx, g.Ny, g.Nz)
    assert d.delta == g.delta
    assert tuple(d.min_coord) == tuple(g.min_coord)


def test_projectors_match_oracle(dev_setup, small_op):
    s, (S, Sx, Sy, Sz, indS) = dev_setup
    np.testing.assert_array_equal(indS, small_op.indS)
    for a, b in ((S, small_op.S), (Sx, small_op.Sx), (Sy, small_op.Sy), (Sz, small_op.Sz)):
        assert rel(a, b) < 1e-9


def test_near_zone_matches_oracle(dev_setup, small_op):
    s, _ = dev_setup
    sp, ind = s.get_nearzone()
    sp64, ind64 = small_op.geom.nearzone(small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, fp64=True)
    o = np.lexsort((ind64[:, 1], ind64[:, 0]))
    np.testing.assert_array_equal(ind, ind64[o])
    ref = sp64[o]
    err = np.abs(sp - ref).max() / np.abs(ref).max()
    assert err < 1e-9, err


def test_device_operator_matvec_matches_oracle(dev_setup, small_op, rng):
    s, _ = dev_setup
    x = rng.standard_normal(3 * small_op.geom.T) + 1j * rng.standard_normal(3 * small_op.geom.T)
    small_op.merged = False
    # the oracle operator with FP64 near zone
    sp64, ind64 = small_op.geom.nearzone(small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, fp64=True)
    op64 = O.Operator(small_op.geom, small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, small_op.indS,
                      small_op.Fg, sp64, ind64)
    assert rel(s.compute_Ax2(x), op64.compute_Ax2(x)) < 1e-9


def test_vswf_rhs_matches_oracle(dev_setup, small_sphere, small_op):
    s, _ = dev_setup
    for Nmax in (1, 3, 6):
        mat = s.vswf2constant(Nmax)
        ref = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, Nmax)
        assert rel(mat, ref) < 1e-12, Nmax


def test_green_host_and_device_agree(small_sphere):
    """Fg passed from the host (power-of-two 2N) equals the device-built one."""
    from scadyn_b200 import geometry
    m = small_sphere
    gs = geometry.cell_size_for_grid(m.coord, m.etopol, 16)
    g = O.Geometry(m.coord, m.etopol, m.param, k=1.0 / m.a, grid_size=gs)
    assert max(g.Nx, g.Ny, g.Nz) == 16
    S, Sx, Sy, Sz, indS = g.projectors()
    Fg = g.build_G()
    sp, ind = g.nearzone(S, Sx, Sy, Sz)
    op = O.Operator(g, S, Sx, Sy, Sz, indS, Fg, sp, ind)
    from tests.gpu_helpers import solver_from_oracle
    a = solver_from_oracle(op, fg_from_host=True)
    b = solver_from_oracle(op, fg_from_host=False)
    x = np.random.default_rng(5).standard_normal(3 * g.T) + 0j
    ya, yb, yr = a.compute_Ax2(x), b.compute_Ax2(x), op.compute_Ax2(x)
    assert rel(ya, yr) < 1e-11
    assert rel(yb, yr) < 1e-11
    a.close()
    b.close()


def test_full_device_T_matrix_matches_oracle(dev_setup, small_sphere, small_op):
    """T from the device-built operator and device RHS vs the oracle's own
    setup and solve: agreement to the GMRES tolerance."""
    s, _ = dev_setup
    k = small_op.geom.k
    Td, iters = s.compute_T_matrix(1, tol=1e-10)
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, k, 1)
    sp64, ind64 = small_op.geom.nearzone(small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, fp64=True)
    op64 = O.Operator(small_op.geom, small_op.S, small_op.Sx, small_op.Sy, small_op.Sz, small_op.indS,
                      small_op.Fg, sp64, ind64)
    X = np.zeros_like(mat)
    for c in range(mat.shape[0]):
        X[c], _ = op64.gmres(mat[c], tol=1e-10)
    T = O.T_assemble(mat, X).T * (1j * k ** 3)
    assert rel(Td, T) < 1e-8
    # a column range returns the same columns
    Tpart, _ = s.compute_T_matrix(1, col0=2, ncol=3, tol=1e-10)
    assert rel(Tpart, Td[:, 2:5]) < 1e-12


@pytest.mark.parametrize("block", [1, 3])
def test_T_columns_round_robin_share(dev_setup, block):
    """scd_compute_T_columns over a replica's round-robin share, listed out of
    order, returns the same bits as those columns of scd_compute_T_matrix
    (columns are batch-invariant); a repeated or out-of-range index is
    SCD_BAD_ARG."""
    s, _ = dev_setup
    Nmax = 2
    kw = dict(tol=1e-10, m=50, cycles=8, block=block)
    Tfull, itf = s.compute_T_matrix(Nmax, **kw)
    cols = np.arange(1, Tfull.shape[1], 3)[::-1].copy()
    Tc, itc = s.compute_T_columns(Nmax, cols, **kw)
    assert np.array_equal(Tc, Tfull[:, cols])
    assert np.array_equal(itc, itf[cols])
    with pytest.raises(api.ScadynError) as e:
        s.compute_T_columns(Nmax, [0, 0], **kw)
    assert e.value.code == api.SCD_BAD_ARG
    with pytest.raises(api.ScadynError):
        s.compute_T_columns(Nmax, [Tfull.shape[1]], **kw)


@pytest.mark.parametrize("precision", [api.PREC_FP64, api.PREC_MIXED])
def test_solve_columns_in_blocks_reproduce_T_matrix(dev_setup, small_op, precision):
    """The column loop run by the host in two blocks (scd_solve_columns over
    columns 0..4 and 5..nmat-1 of the whole mat, T_matrix.f90:254-268) returns
    T_mat(:, col) = mat^H x over all nmat rows (T_matrix.f90:260); times i k^3
    (T_matrix.f90:271-275) the blocks are scd_compute_T_matrix's full T.  The
    resident matrix of scd_set_rhs_matrix serves a call with mat = NULL the
    same way.  Columns are batch-invariant, so the two agree to rounding of
    the scaling only."""
    s, _ = dev_setup
    k = small_op.geom.k
    Nmax = 2
    mat = s.vswf2constant(Nmax)                  # (nmat, n)
    nmat = mat.shape[0]
    kw = dict(tol=1e-10, m=50, cycles=8, block=4, precision=precision, inner_tol=1e-4, max_outer=10)
    Tfull, _ = s.compute_T_matrix(Nmax, **kw)     # (nmat, nmat), scaled
    Ta, ita, _, rca = s.solve_columns(mat, col0=0, ncol=5, **kw)
    s.set_rhs_matrix(mat)
    Tb, itb, _, rcb = s.solve_columns(None, col0=5, ncol=nmat - 5, nmat=nmat, **kw)
    assert rca == api.SCD_OK and rcb == api.SCD_OK
    assert Ta.shape == (5, nmat) and Tb.shape == (nmat - 5, nmat)
    Tblocks = np.concatenate([Ta, Tb]).T          # (nmat rows, nmat columns), unscaled
    assert rel(1j * k ** 3 * Tblocks, Tfull) < 1e-13
