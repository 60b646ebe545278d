"""The tensor-core near zone of the complex64 matvec (scd_grid_desc.near_kernel:
SCD_NEAR_TENSOR_SPLIT, SCD_NEAR_TENSOR_MERGED -- the default with complex64
storage -- and SCD_NEAR_TENSOR_WIDE, 32 right-hand sides per pass) against the
CUDA-core kernel (SCD_NEAR_CUDA_CORES) on the same operator: mixed-precision
T-matrices agree to 1e-6 and both meet the FP64 residual, iteration counts
stay within 20%, results are batch-invariant, and the pipeline never times
out.  Two grid cell sizes give groups below and above 64 rows (M = 64 and
M = 128 accumulators); the wide schedule runs with more than 32 columns in
flight, so that full and partial passes both occur."""
import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import api
from tests.gpu_helpers import solver_from_oracle

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module",
                params=[(1.8, api.NEAR_TENSOR_SPLIT), (3.2, api.NEAR_TENSOR_SPLIT),
                        (1.8, api.NEAR_DEFAULT), (3.2, api.NEAR_TENSOR_MERGED),
                        (1.8, api.NEAR_TENSOR_WIDE), (3.2, api.NEAR_TENSOR_WIDE)],
                ids=["1.8", "3.2", "1.8-default", "3.2-merged", "1.8-wide", "3.2-wide"])
def ops(request, small_sphere):
    grid_size, kernel = request.param
    k = 1.0 / small_sphere.a
    op = O.setup(small_sphere, k, grid_size=grid_size, nthreads=0)
    a = solver_from_oracle(op, near_kernel=api.NEAR_CUDA_CORES)
    b = solver_from_oracle(op, near_kernel=kernel)
    yield op, a, b
    a.close()
    b.close()


def test_tensor_near_zone_T_matches_cuda_core(ops, small_sphere):
    op, a, b = ops
    wide = b.desc.near_kernel == api.NEAR_TENSOR_WIDE
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, op.geom.k, 4 if wide else 2)
    kw = dict(tol=1e-9, block=48 if wide else 16, precision=api.PREC_MIXED, inner_tol=1e-4, max_outer=10,
              want_x=True)
    Ta, ita, Xa, rca = a.solve_columns(mat, **kw)
    Tb, itb, Xb, rcb = b.solve_columns(mat, **kw)
    assert rca == api.SCD_OK and rcb == api.SCD_OK
    assert rel(Tb, Ta) < 1e-6
    for c in (0, 5, mat.shape[0] - 1):
        r = mat[c] - op.compute_Ax2(Xb[c])
        assert np.linalg.norm(r) / np.linalg.norm(mat[c]) < 1e-8
    assert itb.sum() <= 1.2 * ita.sum() + 16


def test_tensor_near_zone_batch_invariant(ops, small_sphere):
    op, _, b = ops
    wide = b.desc.near_kernel == api.NEAR_TENSOR_WIDE
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, op.geom.k, 4 if wide else 1)
    if wide:
        mat = mat[:40]
    kw = dict(tol=1e-8, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True)
    x1 = b.solve_columns(mat, block=1, **kw)
    x2 = b.solve_columns(mat, block=mat.shape[0], **kw)
    assert np.array_equal(x1[1], x2[1])
    assert np.array_equal(x1[2], x2[2])


def test_tensor_near_zone_profile_runs(ops):
    _, _, b = ops
    t = b.profile_matvec(reps=3, nrhs=40, precision=api.PREC_MIXED)
    assert t["matvecs"] >= 3 and t["nearzone_ms"] > 0


def test_complex128_storage_keeps_cuda_cores(small_sphere):
    """With complex128 near-zone storage the default falls back to the CUDA-core
    kernel, and an explicit tensor-core request is refused."""
    k = 1.0 / small_sphere.a
    op = O.setup(small_sphere, k, grid_size=1.8, fp64_near=True, nthreads=0)
    s = solver_from_oracle(op)
    try:
        mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, k, 1)
        _, _, _, rc = s.solve_columns(mat, tol=1e-8, block=6, precision=api.PREC_MIXED, inner_tol=1e-3)
        assert rc == api.SCD_OK
    finally:
        s.close()
    s = solver_from_oracle(op, near_kernel=api.NEAR_TENSOR_MERGED)
    try:
        with pytest.raises(api.ScadynError) as e:
            s.solve_columns(mat, tol=1e-8, block=6, precision=api.PREC_MIXED, inner_tol=1e-3)
        assert e.value.code == api.SCD_BAD_ARG
    finally:
        s.close()


def test_wide_and_merged_schedules_give_the_same_bits(small_sphere):
    """The wide schedule (32 right-hand sides per tensor-core pass, 16 for the
    rest) and the merged one (16 per pass) form every output element from the
    same products in the same order, so a column solved with either has the
    same bits: 40 columns at once take a 32-wide and a 16-wide pass, and the
    batch shrinks through both as columns finish."""
    k = 1.0 / small_sphere.a
    op = O.setup(small_sphere, k, grid_size=1.8, nthreads=0)
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, k, 4)[:40]
    kw = dict(tol=1e-8, block=40, precision=api.PREC_MIXED, inner_tol=1e-3, want_x=True)
    out = []
    for kernel in (api.NEAR_TENSOR_MERGED, api.NEAR_TENSOR_WIDE):
        s = solver_from_oracle(op, near_kernel=kernel)
        try:
            out.append(s.solve_columns(mat, **kw))
        finally:
            s.close()
    assert np.array_equal(out[0][1], out[1][1])
    assert np.array_equal(out[0][2], out[1][2])
