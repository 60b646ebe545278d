"""Generates tests/golden/sphere1680.npz: per-stage outputs of the CPU oracle
on a fixed seeded case, the regression fixtures the CPU and GPU tests check.

The reference (Fortran, FFTW, LAPACK) cannot be compiled here and ships no
golden vectors, so these fixtures pin the oracle to its own committed outputs
(and, through test_oracle.py, to numpy/scipy restatements and the Mie
series); they are not outputs of the reference itself.

Case: sphere(4) lattice mesh (1680 tets, seed 1, eps 2.25+0.01i), ka = 1,
build_grid cell_size 1.8, constant basis, M_ex = 2, near zone stored in
complex64 as the reference does.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from scadyn_b200 import meshgen  # noqa: E402

NT_PROJ = 64          # projector columns kept (first tets)
NB_NEAR = 512         # near-zone blocks kept (first in (tet_T, tet_B) order)
NMAX = 2


def main():
    mesh = meshgen.sphere(4, seed=1, eps=2.25 + 0.01j)
    k = 1.0 / mesh.a
    op = O.setup(mesh, k, grid_size=1.8, nthreads=0)
    g = op.geom
    rng = np.random.default_rng(20240)
    x = rng.standard_normal(3 * g.T) + 1j * rng.standard_normal(3 * g.T)
    Ax = op.compute_Ax2(x)
    mat = O.vswf2constant(mesh.coord, mesh.etopol, k, NMAX)
    X = np.zeros_like(mat)
    iters = np.zeros(mat.shape[0], np.int32)
    for c in range(mat.shape[0]):
        X[c], info = op.gmres(mat[c], tol=1e-10, m=50, cycles=4)
        iters[c] = info["iters"]
    T = O.T_assemble(mat, X).T * (1j * k ** 3)
    Nx, Ny, Nz = g.Nx, g.Ny, g.Nz
    np.savez_compressed(
        os.path.join(HERE, "sphere1680.npz"),
        coord=mesh.coord, etopol=mesh.etopol, param=mesh.param, a=mesh.a, k=k, grid_size=1.8,
        grid=np.array([Nx, Ny, Nz]), delta=g.delta, min_coord=np.array(g.min_coord),
        S=op.S[:NT_PROJ], Sx=op.Sx[:NT_PROJ], Sy=op.Sy[:NT_PROJ], Sz=op.Sz[:NT_PROJ], indS=op.indS[:NT_PROJ],
        Fg_octant=op.Fg[:Nz + 1, :Ny + 1, :Nx + 1] if op.Fg.ndim == 3 else op.Fg,
        sp_mat=op.sp_mat[:NB_NEAR], sp_ind=op.sp_ind[:NB_NEAR], nblocks=op.sp_ind.shape[0],
        x=x, Ax=Ax, Nmax=NMAX, T=T, iters=iters)
    print("wrote", os.path.join(HERE, "sphere1680.npz"))


if __name__ == "__main__":
    main()
