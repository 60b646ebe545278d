"""Autotuning of the solve's kernel choices, with a cache.

The reference picks its FFT plans at run time (FFTW plans made per length,
src/possu.f90:82-89); this is the counterpart for the device path.  Two
levels:

- ``tune_matvec``: the matvec kernels of one context -- near-zone kernel
  (CUDA cores, tensor cores split or merged), fused or three-pass y-z FFT,
  anterpolation and interpolation spans -- timed by the library itself
  (``scd_tune_matvec``) for a right-hand-side count and precision, applied to
  the context and cached by problem shape;
- ``tune_slots``: the batched solver's slots (columns in flight) and the
  mixed form's inner Krylov dimension, timed on a short sample of columns.

The cache is a JSON file keyed by the problem's shape (grid nodes, FFT
lengths, tets, near-zone storage, right-hand sides, precision): a later
context of the same shape applies the stored choice without timing.
"""
from __future__ import annotations

import json
import os
import time

from . import api


def _load(path):
    if path and os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    return {}


def _store(path, cache):
    if not path:
        return
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def shape_key(solver, what, **extra):
    d = solver.desc
    parts = [what, f"grid={d.Nx}x{d.Ny}x{d.Nz}", f"tets={solver.T}", f"order={solver.order}",
             f"fft={d.fft_lengths}", f"near={d.near_kernel}"]
    parts += [f"{k}={extra[k]}" for k in sorted(extra)]
    return ";".join(parts)


_memory = {}


def tune_matvec(solver, nrhs, precision=api.PREC_MIXED, cache=None, reps=10):
    """Choose and apply the fastest matvec kernel setting of `solver` for
    `nrhs` right-hand sides; returns the setting (with its matvec time and
    the defaults' time) and whether it came from the cache."""
    key = shape_key(solver, "matvec", nrhs=nrhs, precision=precision)
    store = _load(cache)
    hit = store.get(key) or _memory.get(key)
    if hit:
        solver.apply_tuning(hit)
        return dict(hit), True
    t = solver.tune_matvec(nrhs, precision, reps)
    _memory[key] = t
    store[key] = t
    _store(cache, store)
    return t, False


def tune_slots(solver, Nmax, sample_cols=32, slots=(16, 32, 64), inner_m=(20, 30), cache=None, col0=0, **opts):
    """Choose the batched solver's slot count and the mixed form's inner
    Krylov dimension by timing `sample_cols` columns (from col0) for each
    pair; returns (choice, columns/s of every pair, from cache)."""
    key = shape_key(solver, "slots", Nmax=Nmax, sample=sample_cols,
                    opts=",".join(f"{k}={opts[k]}" for k in sorted(opts)))
    store = _load(cache)
    hit = store.get(key) or _memory.get(key)
    if hit:
        return dict(hit["choice"]), hit["rates"], True
    rates = {}
    best, best_rate = None, -1.0
    for ns in slots:
        for m in inner_m:
            kw = dict(opts, m=m, block=min(ns, sample_cols), precision=api.PREC_MIXED)
            solver.timing(reset=True)
            t = time.time()
            solver.compute_T_matrix(Nmax, col0=col0, ncol=sample_cols, **kw)
            ms = solver.timing(reset=True)["accum_ms"] or (time.time() - t) * 1e3
            rate = sample_cols / (ms / 1e3)
            rates[f"slots={ns},m={m}"] = round(rate, 4)
            if rate > best_rate:
                best, best_rate = {"slots": ns, "inner_m": m}, rate
    rec = {"choice": best, "rates": rates}
    _memory[key] = rec
    store[key] = rec
    _store(cache, store)
    return dict(best), rates, False
