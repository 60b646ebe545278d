"""Energy balance of the T-matrix (tr_T, src/mie.f90:728-759): extinction
-2 pi / k^2 Re tr T and scattering 2 pi / k^2 sum |T|^2 of the oracle's JVIE
T-matrix on an ellipsoid.  A lossless body (real eps) neither absorbs nor
gains beyond discretisation level (|Cabs| / Cext < 1e-2; 2.6e-3 at this mesh);
with Im eps = 0.1 absorption appears (Cabs / Cext about 0.15)."""
import dataclasses

import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import meshgen


def cross_sections(eps, Nmax=3):
    mesh = meshgen.ellipsoid(4, ratios=(1.0, 0.75, 0.55), seed=5, eps=eps)
    k = 1.4 / mesh.a
    op = dataclasses.replace(O.setup(mesh, k, grid_size=1.8, fp64_near=True, nthreads=0), nthreads=0)
    mat = O.vswf2constant(mesh.coord, mesh.etopol, k, Nmax)
    X = np.array([op.gmres(mat[c], tol=1e-11, m=50, cycles=12)[0] for c in range(mat.shape[0])])
    T = O.T_assemble(mat, X).T * (1j * k ** 3)          # compute_T_matrix scaling (src/T_matrix.f90:271)
    nm = mat.shape[0] // 2
    return O.tr_T(T[:nm, :nm], T[nm:, nm:], T[:nm, nm:], T[nm:, :nm], k)


@pytest.mark.parametrize("eps,lo,hi", [(2.6 + 0.0j, -1e-2, 1e-2), (2.6 + 0.1j, 0.05, 0.3)])
def test_absorption_matches_material_loss(eps, lo, hi):
    cext, csca, cabs, _ = cross_sections(eps)
    assert cext > 0 and csca > 0
    assert lo < cabs / cext < hi
