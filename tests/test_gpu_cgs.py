"""Classical Gram-Schmidt for the complex64 inner solves
(scd_solve_opts.gram_schmidt = SCD_GS_CLASSICAL, the default) against modified
Gram-Schmidt (SCD_GS_MODIFIED) on the same context: mixed-precision T-matrices
agree to 1e-6, both meet the FP64 residual, iteration counts stay within 20%,
and results are batch-invariant.  The FP64 form always uses MGS."""
import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import api

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_cgs_T_matches_mgs(dev_small, small_op, small_sphere):
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 2)
    kw = dict(tol=1e-9, block=16, precision=api.PREC_MIXED, inner_tol=1e-4, max_outer=10, want_x=True)
    Ta, ita, Xa, rca = dev_small.solve_columns(mat, gram_schmidt=api.GS_MODIFIED, **kw)
    Tb, itb, Xb, rcb = dev_small.solve_columns(mat, gram_schmidt=api.GS_CLASSICAL, **kw)
    assert rca == api.SCD_OK and rcb == api.SCD_OK
    assert rel(Tb, Ta) < 1e-6
    for c in (0, 5, mat.shape[0] - 1):
        r = mat[c] - small_op.compute_Ax2(Xb[c])
        assert np.linalg.norm(r) / np.linalg.norm(mat[c]) < 1e-8
    assert itb.sum() <= 1.2 * ita.sum() + 16


@pytest.mark.parametrize("gs", [api.GS_CLASSICAL, api.GS_MODIFIED])
def test_gram_schmidt_batch_invariant(dev_small, small_op, small_sphere, gs):
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    kw = dict(tol=1e-8, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True, gram_schmidt=gs)
    x1 = dev_small.solve_columns(mat, block=1, **kw)
    x2 = dev_small.solve_columns(mat, block=6, **kw)
    assert np.array_equal(x1[1], x2[1])
    assert np.array_equal(x1[2], x2[2])


def test_fp64_form_unaffected(dev_small, small_op, small_sphere):
    """The FP64 form keeps MGS: identical results whatever gram_schmidt says."""
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    ra = dev_small.solve_columns(mat, tol=1e-8, block=4, want_x=True, gram_schmidt=api.GS_MODIFIED)
    rb = dev_small.solve_columns(mat, tol=1e-8, block=4, want_x=True, gram_schmidt=api.GS_CLASSICAL)
    assert np.array_equal(ra[1], rb[1]) and np.array_equal(ra[2], rb[2])
