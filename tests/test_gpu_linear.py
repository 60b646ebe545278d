"""Linear basis (mesh%order = 1) on the device, as pseudo-tets: the matvec
against the oracle's compute_Ax2 with order 1 (src/gmres_module.f90:57-176,
matmul_Acorr src/sparse_mat.f90:64-92) on the same operator data, complex64
and complex128 near-zone storage, and GMRES against the oracle's (same
iteration count).  The operator is the seeded linear-basis operator the
oracle derives from the 1680-tet sphere."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from tests.gpu_helpers import solver_from_oracle

pytestmark = pytest.mark.gpu


def crand(rng, n):
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def op1(small_op):
    return O.linear_from_constant(dataclasses.replace(small_op, nthreads=0), seed=3)


@pytest.mark.parametrize("c128", [False, True])
def test_linear_matvec_matches_oracle(op1, c128):
    op = op1 if not c128 else dataclasses.replace(op1, sp_mat=op1.sp_mat.astype(np.complex128))
    s = solver_from_oracle(op)
    try:
        rng = np.random.default_rng(11)
        x = crand(rng, 12 * op.geom.T)
        assert rel(s.compute_Ax2(x), op.compute_Ax2(x)) < 1e-11
    finally:
        s.close()


def test_linear_gmres_matches_oracle(op1):
    s = solver_from_oracle(op1)
    try:
        rng = np.random.default_rng(12)
        b = crand(rng, 12 * op1.geom.T)
        x, info = s.gmres(b, tol=1e-8, m=50, cycles=8)
        xr, ir = op1.gmres(b, tol=1e-8, m=50, cycles=8)
        assert info["iters"] == ir["iters"]
        assert rel(x, xr) < 1e-8
    finally:
        s.close()


def test_linear_T_matrix_refused(op1):
    from scadyn_b200 import api
    s = solver_from_oracle(op1)
    try:
        with pytest.raises(api.ScadynError):
            s.compute_T_matrix(2)
    finally:
        s.close()
