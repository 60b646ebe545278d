"""Generates tests/golden/sphere336_linear.npz: the CPU oracle's linear-basis
(mesh%order = 1) set-up and matvec on a fixed seeded case, regression fixtures
for the oracle and the device.

As with sphere1680.npz, the reference cannot be compiled here and ships no
golden vectors: these pin the oracle to its own committed outputs, which
tests/test_oracle_linear_setup.py ties to brute-force quadrature and numpy
restatements.

Case: sphere(2.5) lattice mesh (336 tets, seed 1, eps 2.25+0.01i), ka = 1,
build_grid cell_size 1.8, linear basis, M_ex = 2, near zone stored in
complex64 as the reference does.

    python tests/golden/make_golden_linear.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from scadyn_b200 import meshgen  # noqa: E402

NT_PROJ = 16          # tets whose four projector columns are kept
NB_NEAR = 96          # 12x12 blocks kept (first in (tet_T, tet_B) order)


def main():
    mesh = meshgen.sphere(2.5, seed=1, eps=2.25 + 0.01j)
    k = 1.0 / mesh.a
    op = O.setup_lin(mesh, k, grid_size=1.8, nthreads=0)
    g = op.geom
    rng = np.random.default_rng(20241)
    n = 12 * g.T
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Ax = op.compute_Ax2(x)
    np.savez_compressed(
        os.path.join(HERE, "sphere336_linear.npz"),
        coord=mesh.coord, etopol=mesh.etopol, param=mesh.param, a=mesh.a, k=k, grid_size=1.8,
        S=op.S[:4 * NT_PROJ], Sx=op.Sx[:4 * NT_PROJ], Sy=op.Sy[:4 * NT_PROJ], Sz=op.Sz[:4 * NT_PROJ],
        indS=op.indS[:4 * NT_PROJ], sp_mat=op.sp_mat[:NB_NEAR], sp_ind=op.sp_ind[:NB_NEAR],
        nblocks=op.sp_ind.shape[0], x=x, Ax=Ax)
    print("wrote", os.path.join(HERE, "sphere336_linear.npz"))


if __name__ == "__main__":
    main()
