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
granularity.  A JSON line of per-block metrics (columns/s, iterations, and the
solver's per-phase device milliseconds when it keeps them) can be appended to a
log.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np


def _key(Nmax, opts, tag):
    return json.dumps({"Nmax": int(Nmax), "opts": {k: opts[k] for k in sorted(opts)}, "tag": tag}, sort_keys=True)


def _save(path, T, done, iters, key):
    tmp = path + ".tmp.npz"
    np.savez(tmp, T=T, done=done, iters=iters, key=np.array(key))
    os.replace(tmp, path)


def solve_T_with_checkpoints(solver, Nmax, path, block=64, tag="", log=None, **opts):
    """T (2nm, 2nm) of `solver` (anything with compute_T_matrix(Nmax, col0,
    ncol, **opts) -> (T_cols, iters)), resuming from `path` when it holds a
    checkpoint of the same problem (same Nmax, options and tag).  Returns
    (T, iters, blocks solved in this call)."""
    ncol = 2 * ((Nmax + 1) ** 2 - 1)
    key = _key(Nmax, opts, tag)
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
            with open(log, "a") as f:
                f.write(json.dumps(rec) + "\n")
    return T, iters, solved
