"""Committed fixtures (tests/golden/sphere1680.npz, made by
tests/golden/make_golden.py from the CPU oracle): the oracle must keep
reproducing them (CPU), and the device path must match them (GPU) -- grid,
projectors, near-zone blocks, one matvec, GMRES iteration counts and the
T-matrix of a 1680-tet sphere at ka = 1."""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "sphere1680.npz"))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# ------------------------------------------------------------ oracle (CPU)
def test_oracle_geometry_and_green(small_op):
    g = small_op.geom
    assert [g.Nx, g.Ny, g.Nz] == list(G["grid"])
    assert g.delta == float(G["delta"])
    assert np.array_equal(np.array(g.min_coord), G["min_coord"])
    Nx, Ny, Nz = G["grid"]
    assert rel(small_op.Fg[:Nz + 1, :Ny + 1, :Nx + 1], G["Fg_octant"]) < 1e-13


def test_oracle_projectors_and_near_zone(small_op):
    n = G["S"].shape[0]
    for name in ("S", "Sx", "Sy", "Sz"):
        assert rel(getattr(small_op, name)[:n], G[name]) < 1e-13
    assert np.array_equal(small_op.indS[:n], G["indS"])
    nb = G["sp_ind"].shape[0]
    assert small_op.sp_ind.shape[0] == int(G["nblocks"])
    assert np.array_equal(small_op.sp_ind[:nb], G["sp_ind"])
    assert np.array_equal(small_op.sp_mat[:nb], G["sp_mat"])


def test_oracle_matvec_and_T(small_op, small_sphere):
    small_op.merged = False
    assert rel(small_op.compute_Ax2(G["x"]), G["Ax"]) < 1e-13
    k = float(G["k"])
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, k, int(G["Nmax"]))
    X = np.zeros_like(mat)
    for c in range(mat.shape[0]):
        X[c], info = small_op.gmres(mat[c], tol=1e-10, m=50, cycles=4)
        assert info["iters"] == G["iters"][c]
    T = O.T_assemble(mat, X).T * (1j * k ** 3)
    assert rel(T, G["T"]) < 1e-12


# ------------------------------------------------------------ device (GPU)
@pytest.fixture(scope="module")
def dev_built():
    from scadyn_b200 import api
    d = api.grid_from_mesh(G["coord"], G["etopol"], grid_size=float(G["grid_size"]))
    s = api.Solver.from_desc(d)
    s.set_wavenumber(float(G["k"]))
    s.set_mesh(G["coord"], G["etopol"], G["param"])
    s.build_G()
    s.pfft_projection_const()
    s.compute_near_zone_interactions_const(api.STORE_C64)
    yield s, d
    s.close()


@pytest.mark.gpu
def test_device_grid_and_projectors(dev_built):
    s, d = dev_built
    assert [d.Nx, d.Ny, d.Nz] == list(G["grid"])
    S, Sx, Sy, Sz, indS = s.get_projectors()
    n = G["S"].shape[0]
    for got, name in zip((S, Sx, Sy, Sz), ("S", "Sx", "Sy", "Sz")):
        assert rel(got[:n], G[name]) < 1e-9
    assert np.array_equal(indS[:n], G["indS"])


@pytest.mark.gpu
def test_device_near_zone(dev_built):
    s, _ = dev_built
    sp, ind = s.get_nearzone()
    assert ind.shape[0] == int(G["nblocks"])
    # the device exports in (tet_T, tet_B) order; the fixture keeps the
    # oracle's first blocks in its own traversal order
    pos = {(int(t), int(b)): i for i, (t, b) in enumerate(ind)}
    sel = np.array([pos[(int(t), int(b))] for t, b in G["sp_ind"]])
    # both built in FP64 and rounded to complex64: equal to complex64 rounding
    assert rel(sp[sel], G["sp_mat"].astype(np.complex128)) < 1e-6


@pytest.mark.gpu
def test_device_matvec_and_T(dev_built):
    s, _ = dev_built
    assert rel(s.compute_Ax2(G["x"]), G["Ax"]) < 1e-6
    T, iters = s.compute_T_matrix(int(G["Nmax"]), tol=1e-10, m=50, cycles=4, block=16)
    assert rel(T, G["T"]) < 1e-6
    assert np.abs(iters.astype(int) - G["iters"].astype(int)).max() <= 1


@pytest.mark.gpu
def test_oracle_operator_on_device_matches_golden_matvec(small_op):
    """The oracle's operator data run through the CUDA matvec reproduce the
    golden Ax to rounding."""
    from tests.gpu_helpers import solver_from_oracle
    s = solver_from_oracle(small_op)
    try:
        assert rel(s.compute_Ax2(G["x"]), G["Ax"]) < 1e-11
    finally:
        s.close()
