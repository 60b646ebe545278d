"""Physics pin of the oracle under mesh refinement: the T-matrix of the
constant-basis JVIE (src/T_matrix.f90:240-277 over the operator of
src/precorrection.f90:131-264 and src/projection.f90:17-166) approaches the
Mie series of the sphere (src/mie.f90) as the tets shrink.

The electric-dipole coefficient a_1 is dominated by the volume integral and
the self and near-zone terms, and its error falls with h: about 5.7 %, 4.3 %
and 2.2 % at h = a/3, a/4 and a/6 (816, 1680 and 5472 tets, ka = 1,
eps = 2.25 + 0.01i, pFFT cell 1.8 h).  A wrong sign or factor in one face
term of the singular integrals would leave an error floor there that does
not move with h.  The magnetic-dipole coefficient b_1 stays within about 2 %
at every h; its floor moves with the pFFT cell (1.0 to 2.0 % for cells of
1.2 to 2.5 h at h = a/6), so it is set by the far-field approximation, not
by the singular integrals.  Runs on the CPU in about 20 s."""
import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import meshgen

EPS = 2.25 + 0.01j


def _dipole_errors(nres):
    mesh = meshgen.sphere(nres, seed=1, eps=EPS)
    k = 1.0 / mesh.a
    op = O.setup(mesh, k, grid_size=1.8, nthreads=0)
    op.nthreads = 0
    nm = 3                                   # Nmax = 1: m = -1, 0, 1
    mat = O.vswf2constant(mesh.coord, mesh.etopol, k, 1)
    X = np.zeros_like(mat)
    for c in range(2 * nm):
        X[c], info = op.gmres(mat[c], tol=1e-8, m=50, cycles=10)
        assert info["converged"], (nres, c)
    T = O.T_assemble(mat, X).T * (1j * k ** 3)
    a_n, b_n = O.mie_T(1, k * mesh.a, np.sqrt(EPS))
    ea = max(abs(T[j, j] - a_n[0]) / abs(a_n[0]) for j in range(nm))
    eb = max(abs(T[nm + j, nm + j] - b_n[0]) / abs(b_n[0]) for j in range(nm))
    return ea, eb


@pytest.fixture(scope="module")
def errors():
    return {n: _dipole_errors(n) for n in (3, 4, 6)}


def test_electric_dipole_error_falls_with_h(errors):
    ea = [errors[n][0] for n in (3, 4, 6)]
    assert ea[0] > ea[1] > ea[2], ea
    assert ea[0] / ea[2] > 1.8, ea            # about first order in h (h ratio 2)
    assert ea[2] < 0.03, ea


def test_magnetic_dipole_within_far_field_floor(errors):
    eb = [errors[n][1] for n in (3, 4, 6)]
    assert max(eb) < 0.03, eb
