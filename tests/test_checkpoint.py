"""Checkpoint and resume of a T-matrix solve at block granularity: an
interrupted solve resumes where it stopped and assembles the same T; a
checkpoint of a different problem is ignored; every finished block is logged
as one JSON line.  A stand-in solver replaces the device (host logic only)."""
import json

import numpy as np
import pytest

from scadyn_b200.checkpoint import solve_T_with_checkpoints


class _Stub:
    def __init__(self, fail_after=None, problem="mesh-a"):
        self.calls = []
        self.fail_after = fail_after
        self.problem = problem

    def problem_key(self):
        return {"source": self.problem, "k": 1.0}

    def compute_T_matrix(self, Nmax, col0=0, ncol=None, **kw):
        if self.fail_after is not None and len(self.calls) >= self.fail_after:
            raise RuntimeError("interrupted")
        self.calls.append((col0, ncol))
        n = 2 * ((Nmax + 1) ** 2 - 1)
        cols = np.arange(col0, col0 + ncol)
        return np.outer(np.arange(1, n + 1), cols + 1) * (1 - 2j), np.full(ncol, 3, np.int32)


def test_interrupted_solve_resumes(tmp_path):
    path = str(tmp_path / "T.npz")
    log = str(tmp_path / "T.jsonl")
    with pytest.raises(RuntimeError):
        solve_T_with_checkpoints(_Stub(fail_after=2), 4, path, block=10, log=log, tol=1e-6)
    s = _Stub()
    T, it, solved = solve_T_with_checkpoints(s, 4, path, block=10, log=log, tol=1e-6)
    full, _ = _Stub().compute_T_matrix(4, 0, 48)
    assert np.array_equal(T, full)
    assert s.calls[0] == (20, 10) and solved == 3          # blocks 0 and 1 came from the checkpoint
    lines = [json.loads(x) for x in open(log)]
    assert [x["col0"] for x in lines] == [0, 10, 20, 30, 40]
    assert lines[-1]["done"] == 48


def test_other_problem_is_not_resumed(tmp_path):
    path = str(tmp_path / "T.npz")
    solve_T_with_checkpoints(_Stub(), 3, path, block=8, tol=1e-6)
    s = _Stub()
    solve_T_with_checkpoints(s, 3, path, block=8, tol=1e-8)   # different options: start over
    assert s.calls[0] == (0, 8)
    s2 = _Stub()
    _, _, solved = solve_T_with_checkpoints(s2, 3, path, block=8, tol=1e-8)   # same: nothing left
    assert solved == 0 and not s2.calls
    s3 = _Stub(problem="mesh-b")                                        # same Nmax and options, other mesh
    solve_T_with_checkpoints(s3, 3, path, block=8, tol=1e-8)
    assert s3.calls[0] == (0, 8)


def test_unknown_problem_needs_a_tag(tmp_path):
    class _Anonymous(_Stub):
        problem_key = None
    s = _Anonymous()
    s.problem_key = lambda: None
    with pytest.raises(ValueError):
        solve_T_with_checkpoints(s, 2, str(tmp_path / "T.npz"), block=8)
    T, _, solved = solve_T_with_checkpoints(s, 2, str(tmp_path / "T.npz"), block=8, tag="sphere ka=1")
    assert solved == 2


class _Timed(_Stub):
    def __init__(self):
        super().__init__()
        self.resets = 0

    def timing(self, reset=False):
        self.resets += bool(reset)
        return {"matvec_ms": 1.5, "matvecs": 7}


def test_log_carries_device_phases(tmp_path):
    log = str(tmp_path / "T.jsonl")
    s = _Timed()
    solve_T_with_checkpoints(s, 2, str(tmp_path / "T.npz"), block=8, log=log)
    lines = [json.loads(x) for x in open(log)]
    assert len(lines) == 2 and s.resets == 2
    assert lines[0]["device"] == {"matvec_ms": 1.5, "matvecs": 7} and lines[0]["iters_max"] == 3


class _Profiled(_Timed):
    def profile_matvec(self, reps, nrhs, precision):
        assert (nrhs, precision) == (1, 0)
        return {"nearzone_ms": 0.5, "matvec_ms": 1.0}

    def nearzone_bytes(self):
        return 3_000_000_000


def test_log_carries_near_zone_roofline_once(tmp_path):
    log = str(tmp_path / "T.jsonl")
    solve_T_with_checkpoints(_Profiled(), 2, str(tmp_path / "T.npz"), block=8, log=log, hbm_gbs=6000.0)
    lines = [json.loads(x) for x in open(log)]
    assert lines[0]["near_zone_roofline"] == {"near_zone_ms": 0.5, "gb_per_s": 6000.0, "frac_of_hbm": 1.0}
    assert "near_zone_roofline" not in lines[1]
