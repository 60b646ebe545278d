"""Committed linear-basis fixtures (tests/golden/sphere336_linear.npz, made by
tests/golden/make_golden_linear.py from the CPU oracle): the oracle must keep
reproducing them (CPU), and the device-built linear operator must match them
(GPU) -- projectors, 12x12 near-zone
blocks and one order-1 matvec of a 336-tet sphere at ka = 1."""
import os

import numpy as np
import pytest

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "sphere336_linear.npz"))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


class _Mesh:
    coord, etopol, param, a = G["coord"], G["etopol"], G["param"], float(G["a"])


@pytest.fixture(scope="module")
def lin_op():
    return O.setup_lin(_Mesh, float(G["k"]), grid_size=float(G["grid_size"]), nthreads=0)


def test_oracle_reproduces_linear_fixture(lin_op):
    n = G["S"].shape[0]
    for name in ("S", "Sx", "Sy", "Sz"):
        assert rel(getattr(lin_op, name)[:n], G[name]) < 1e-12
    assert np.array_equal(lin_op.indS[:n], G["indS"])
    nb = G["sp_ind"].shape[0]
    assert lin_op.sp_ind.shape[0] == int(G["nblocks"])
    assert np.array_equal(lin_op.sp_ind[:nb], G["sp_ind"])
    assert rel(lin_op.sp_mat[:nb].astype(np.complex128), G["sp_mat"].astype(np.complex128)) < 1e-6
    assert rel(lin_op.compute_Ax2(G["x"]), G["Ax"]) < 1e-9


@pytest.mark.gpu
def test_device_linear_operator_matches_fixture():
    from scadyn_b200 import api
    d = api.grid_from_mesh(G["coord"], G["etopol"], grid_size=float(G["grid_size"]))
    d.order = 1
    s = api.Solver.from_desc(d)
    try:
        s.set_wavenumber(float(G["k"]))
        s.set_mesh(G["coord"], G["etopol"], G["param"])
        s.build_G()
        S, Sx, Sy, Sz, indS = s.pfft_projection_lin()
        n = G["S"].shape[0]
        for got, name in zip((S, Sx, Sy, Sz), ("S", "Sx", "Sy", "Sz")):
            assert rel(got[:n], G[name]) < 1e-8
        assert np.array_equal(indS[:n], G["indS"])
        s.compute_near_zone_interactions_lin(api.STORE_C64)
        sp, ind = s.get_nearzone()
        assert sp.shape[0] == int(G["nblocks"])
        # the device exports in (tet_T, tet_B) order; the fixture keeps the
        # oracle's first blocks in its own traversal order
        pos = {(int(t), int(b)): i for i, (t, b) in enumerate(ind)}
        sel = np.array([pos[(int(t), int(b))] for t, b in G["sp_ind"]])
        assert rel(sp[sel], G["sp_mat"].astype(np.complex128)) < 1e-6
        assert rel(s.compute_Ax2(G["x"]), G["Ax"]) < 1e-6
    finally:
        s.close()
