"""Column-granular checkpoint and resume of a T-matrix solve.

The reference's unit of restart is one wavelength: T_empty creates the T-matrix
file once and leaves an existing one alone (src/h5io.f90:562-599, called from
src/main.f90:35), and the single-T mode solves the wavelength `whichbar` and
writes it into its slot of that file (src/T_matrix.f90:45-47,78,
src/h5io.f90:682-830); a long solve (1350 columns at Nmax 25) that stops
midway is lost.  Here the columns are solved in blocks through
compute_T_matrix's column range, and after every block the solved columns and
a manifest (problem key, block list, per-column iterations) are written
atomically to one .npz file, so an interrupted solve resumes at block
granularity.  A JSON line of per-block metrics (columns/s, iterations, the
solver's per-phase device milliseconds when it keeps them, and once the near
zone's achieved bandwidth and HBM-roofline fraction) can be appended to a log.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np


def _key(Nmax, opts, tag, problem):
    return json.dumps({"Nmax": int(Nmax), "opts": {k: opts[k] for k in sorted(opts)}, "tag": tag,
                       "problem": problem}, sort_keys=True)


def _save(path, T, done, iters, key):
    tmp = path + ".tmp.npz"
    np.savez(tmp, T=T, done=done, iters=iters, key=np.array(key))
    os.replace(tmp, path)


def near_zone_roofline(solver, hbm_gbs=None, reps=5):
    """Achieved near-zone bandwidth of `solver` (profile_matvec at one FP64
    right-hand side; the kernel reads every stored tile once per matvec) and,
    given the HBM peak in GB/s, its roofline fraction."""
    t = solver.profile_matvec(reps, 1, 0)
    gbs = solver.nearzone_bytes() / (t["nearzone_ms"] * 1e-3) / 1e9
    out = {"near_zone_ms": round(t["nearzone_ms"], 4), "gb_per_s": round(gbs, 1)}
    if hbm_gbs:
        out["frac_of_hbm"] = round(gbs / hbm_gbs, 4)
    return out


def solve_T_with_checkpoints(solver, Nmax, path, block=64, tag="", log=None, hbm_gbs=None, problem=None, **opts):
    """T (2nm, 2nm) of `solver` (anything with compute_T_matrix(Nmax, col0,
    ncol, **opts) -> (T_cols, iters)), resuming from `path` when it holds a
    checkpoint of the same problem: the same Nmax, options, tag and problem
    identity -- `problem`, or else the solver's problem_key() (unknowns, grid,
    wavenumber and a digest of the mesh or operator it was set up from).  A
    solve whose identity is unknown needs a non-empty tag, so that a
    checkpoint of another mesh or wavelength is never mixed into it.
    Returns (T, iters, blocks solved in this call).  With a log and a solver
    that profiles (profile_matvec, nearzone_bytes), the first record also
    carries the near zone's achieved bandwidth, as a fraction of hbm_gbs when
    given."""
    ncol = 2 * ((Nmax + 1) ** 2 - 1)
    if problem is None and hasattr(solver, "problem_key"):
        problem = solver.problem_key()
    if problem is None and not tag:
        raise ValueError("a checkpoint needs the problem's identity: pass problem=..., a non-empty tag, "
                         "or a solver with problem_key()")
    roof = None
    if log and hasattr(solver, "profile_matvec") and hasattr(solver, "nearzone_bytes"):
        roof = near_zone_roofline(solver, hbm_gbs)
    key = _key(Nmax, opts, tag, problem)
    T = np.zeros((ncol, ncol), np.complex128)
    done = np.zeros(ncol, bool)
    iters = np.zeros(ncol, np.int32)
    if os.path.exists(path):
        d = np.load(path)
        if str(d["key"]) == key and d["T"].shape == T.shape:
            T, done, iters = d["T"].copy(), d["done"].copy(), d["iters"].copy()
    solved = 0
    for c0 in range(0, ncol, block):
        n = min(block, ncol - c0)
        if done[c0:c0 + n].all():
            continue
        timed = hasattr(solver, "timing")
        if timed:
            solver.timing(reset=True)
        t = time.time()
        Tc, it = solver.compute_T_matrix(Nmax, col0=c0, ncol=n, **opts)
        secs = time.time() - t
        T[:, c0:c0 + n] = Tc
        iters[c0:c0 + n] = it
        done[c0:c0 + n] = True
        _save(path, T, done, iters, key)
        solved += 1
        if log:
            rec = {"col0": c0, "ncol": n, "seconds": round(secs, 3), "columns_per_s": round(n / max(secs, 1e-9), 4),
                   "iters_mean": float(np.mean(it)), "iters_max": int(np.max(it)), "done": int(done.sum()),
                   "of": ncol}
            if timed:
                rec["device"] = {k: v for k, v in solver.timing().items()}
            if roof is not None:
                rec["near_zone_roofline"] = roof
                roof = None
            with open(log, "a") as f:
                f.write(json.dumps(rec) + "\n")
    return T, iters, solved
