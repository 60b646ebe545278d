"""Failure detection without a GPU fault: bounded device waits return an
error status (SCD_TIMEOUT) and leave the device usable; a NaN right-hand
side ends its column with SCD_NAN; an iteration cap ends with
SCD_NOT_CONVERGED and the last iterate; bad arguments are refused on the
host."""
import numpy as np
import pytest

from oracle import oracle as O
from scadyn_b200 import api


@pytest.fixture(scope="module")
def dev(small_op):
    from tests.gpu_helpers import solver_from_oracle
    s = solver_from_oracle(small_op)
    yield s
    s.close()


@pytest.mark.gpu
def test_bounded_waits_report_timeout_and_device_stays_usable(dev, small_op):
    lib = api.load_library()
    assert lib.scd_selftest_waits(0) == api.SCD_TIMEOUT
    x = np.ones(3 * small_op.geom.T, np.complex128)
    small_op.merged = False
    y = dev.compute_Ax2(x)
    ref = small_op.compute_Ax2(x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-11


@pytest.mark.gpu
def test_nan_rhs_reports_nan(dev, small_op):
    rhs = np.ones(3 * small_op.geom.T, np.complex128)
    rhs[17] = np.nan
    with pytest.raises(api.ScadynError) as e:
        dev.gmres(rhs, tol=1e-8, m=20, cycles=2)
    assert e.value.code == api.SCD_NAN


@pytest.mark.gpu
def test_iteration_cap_reports_not_converged(dev, small_op, small_sphere):
    mat = O.vswf2constant(small_sphere.coord, small_sphere.etopol, small_op.geom.k, 1)
    x, info = dev.gmres(mat[0], tol=1e-30, m=5, cycles=2)
    assert not info["converged"]
    assert info["iters"] == 10
    assert np.all(np.isfinite(x))


@pytest.mark.gpu
def test_bad_arguments_refused(dev, small_op):
    rhs = np.ones(3 * small_op.geom.T, np.complex128)
    for kw in (dict(m=0), dict(m=api.SCD_M_MAX + 1), dict(cycles=0), dict(tol=-1.0)):
        args = dict(tol=1e-8, m=20, cycles=2)
        args.update(kw)
        with pytest.raises(api.ScadynError) as e:
            dev.gmres(rhs, **args)
        assert e.value.code == api.SCD_BAD_ARG


def test_selftest_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert api.load_library().scd_selftest_waits(0) == api.SCD_NO_DEVICE
