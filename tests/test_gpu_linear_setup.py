"""Linear-basis (mesh%order = 1) operator construction on the device --
pfft_projection_lin (src/projection.f90:170-338) and
compute_near_zone_interactions_lin (src/precorrection.f90:268-725) -- against
the CPU oracle, and the order-1 matvec on the device-built operator.  An
816-tet sphere at ka = 1."""
import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import api

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def mesh():
    from scadyn_b200 import meshgen
    return meshgen.sphere(3, seed=1, eps=2.25 + 0.01j)


@pytest.fixture(scope="module")
def oracle_lin(mesh):
    k = 1.0 / mesh.a
    return O.setup_lin(mesh, k, grid_size=1.8, fp64_near=True)


def _device(mesh, k, storage):
    d = api.grid_from_mesh(mesh.coord, mesh.etopol, grid_size=1.8)
    d.order = 1
    s = api.Solver.from_desc(d)
    s.set_wavenumber(k)
    s.set_mesh(mesh.coord, mesh.etopol, mesh.param)
    s.build_G()
    proj = s.pfft_projection_lin()
    s.compute_near_zone_interactions_lin(storage)
    return s, proj


@pytest.fixture(scope="module")
def dev128(mesh, oracle_lin):
    s, proj = _device(mesh, oracle_lin.geom.k, api.STORE_C128)
    yield s, proj
    s.close()


def test_projectors_lin_match_oracle(dev128, oracle_lin):
    _, (S, Sx, Sy, Sz, indS) = dev128
    assert S.shape == oracle_lin.S.shape
    for got, want in zip((S, Sx, Sy, Sz), (oracle_lin.S, oracle_lin.Sx, oracle_lin.Sy, oracle_lin.Sz)):
        assert rel(got, want) < 1e-8
    assert (indS == oracle_lin.indS).all()


def test_nearzone_lin_c128_matches_oracle(dev128, oracle_lin):
    s, _ = dev128
    sp, ind = s.get_nearzone()
    assert sp.shape == oracle_lin.sp_mat.shape
    order = np.lexsort((oracle_lin.sp_ind[:, 1], oracle_lin.sp_ind[:, 0]))
    assert (ind == oracle_lin.sp_ind[order]).all()
    assert rel(sp, oracle_lin.sp_mat[order]) < 1e-9


def test_nearzone_lin_c64_matches_oracle(mesh, oracle_lin):
    s, _ = _device(mesh, oracle_lin.geom.k, api.STORE_C64)
    try:
        sp, ind = s.get_nearzone()
        order = np.lexsort((oracle_lin.sp_ind[:, 1], oracle_lin.sp_ind[:, 0]))
        assert rel(sp, oracle_lin.sp_mat[order].astype(np.complex64).astype(np.complex128)) < 1e-6
    finally:
        s.close()


def test_matvec_on_device_built_operator(dev128, oracle_lin):
    s, _ = dev128
    rng = np.random.default_rng(21)
    x = rng.standard_normal(s.n) + 1j * rng.standard_normal(s.n)
    assert rel(s.compute_Ax2(x), oracle_lin.compute_Ax2(x)) < 1e-9


@pytest.mark.parametrize("precision,block", [(api.PREC_FP64, 1), (api.PREC_FP64, 4), (api.PREC_MIXED, 4)])
def test_solve_columns_on_device_built_operator(dev128, oracle_lin, precision, block):
    """The batched column solver (FP64 one at a time, FP64 batched, mixed batched) on
    the device-built linear operator: matH X against the oracle's GMRES solutions."""
    s, _ = dev128
    rng = np.random.default_rng(22)
    ncol = 4
    mat = rng.standard_normal((ncol, s.n)) + 1j * rng.standard_normal((ncol, s.n))
    Tc, iters, X, rc = s.solve_columns(mat, tol=1e-8, m=50, cycles=8, block=block, precision=precision,
                                       inner_tol=1e-4, want_x=True)
    assert rc == api.SCD_OK
    Xr = np.array([oracle_lin.gmres(mat[c], tol=1e-8, m=50, cycles=8)[0] for c in range(ncol)])
    assert rel(X, Xr) < 1e-6
    Tr = np.conj(mat) @ Xr.T                 # Tr[r, c] = mat_r^H x_c
    assert rel(Tc.T, Tr) < 1e-6
