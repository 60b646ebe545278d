"""Python binding of the request loop (include/scadyn_server.h).

A :class:`Server` owns one GPU; requests (a mesh with per-tet permittivity, a
wavenumber, a VSWF order and solve options) are submitted at any time and
admitted by an HBM budget.  Requests with the same operator key share a
resident pool (the operator is built once, their columns are solved in the
same batched slots); pools solve concurrently on their own CUDA streams and
stay resident when idle.  Every request returns its full T-matrix, and a
request's result does not depend on what else runs beside it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import api
from .api import ScadynError, SolveOpts

REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = range(5)

EXPORTS = ["scd_server_create", "scd_server_submit", "scd_server_estimate", "scd_server_poll", "scd_server_wait",
           "scd_server_result", "scd_server_cancel", "scd_server_stats_get", "scd_server_error",
           "scd_server_destroy"]


class Request(C.Structure):
    _fields_ = [("Nv", C.c_int32), ("T", C.c_int32), ("coord", C.c_void_p), ("etopol", C.c_void_p),
                ("param", C.c_void_p), ("k", C.c_double), ("grid_size", C.c_double), ("Nmax", C.c_int32),
                ("storage_prec", C.c_int32), ("opts", SolveOpts)]


class Stats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("completed", C.c_int64), ("failed", C.c_int64),
                ("cancelled", C.c_int64), ("columns", C.c_int64), ("queued", C.c_int32), ("running", C.c_int32),
                ("peak_running", C.c_int32), ("bytes_in_use", C.c_int64), ("peak_bytes", C.c_int64),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("busy_s", C.c_double),
                ("pools_built", C.c_int64), ("pool_reuses", C.c_int64), ("pools_resident", C.c_int32)]


_bound = False


def _lib():
    global _bound
    lib = api.load_library()
    if not _bound:
        vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        sig = {
            "scd_server_create": ([C.POINTER(vp), i32, i64, i32], C.c_int),
            "scd_server_submit": ([vp, C.POINTER(Request), C.POINTER(i64)], C.c_int),
            "scd_server_estimate": ([C.POINTER(Request), C.POINTER(i64)], C.c_int),
            "scd_server_poll": ([vp, i64, C.POINTER(i32), C.POINTER(i32), C.POINTER(dbl)], C.c_int),
            "scd_server_wait": ([vp, i64, dbl], C.c_int),
            "scd_server_result": ([vp, i64, vp, vp], C.c_int),
            "scd_server_cancel": ([vp, i64], C.c_int),
            "scd_server_stats_get": ([vp, C.POINTER(Stats)], C.c_int),
            "scd_server_error": ([vp, i64], C.c_char_p),
            "scd_server_destroy": ([vp], C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = res
        _bound = True
    return lib


def ncols(Nmax):
    return 2 * ((Nmax + 1) ** 2 - 1)


class Server:
    def __init__(self, device=0, hbm_budget=150e9, max_running=0):
        """max_running bounds the pools solving at once; 0 leaves it to the
        HBM budget."""
        self.lib = _lib()
        self.srv = C.c_void_p()
        rc = self.lib.scd_server_create(C.byref(self.srv), device, int(hbm_budget), max_running)
        if rc:
            raise ScadynError(rc, "scd_server_create")
        self._keep = {}
        self._nmax = {}

    def _request(self, mesh, k, grid_size, Nmax, tol=1e-6, m=50, cycles=12, block=16,
                 precision=api.PREC_FP64, inner_tol=1e-4, max_outer=10, storage=api.STORE_C64,
                 gram_schmidt=api.GS_DEFAULT):
        coord = np.ascontiguousarray(mesh.coord, np.float64)
        etopol = np.ascontiguousarray(mesh.etopol, np.int32)
        param = np.ascontiguousarray(mesh.param, np.complex128)
        r = Request(coord.shape[0], etopol.shape[0], coord.ctypes.data, etopol.ctypes.data, param.ctypes.data,
                    float(k), float(grid_size), int(Nmax), int(storage),
                    SolveOpts(tol, m, cycles, block, precision, inner_tol, max_outer, gram_schmidt))
        return r, (coord, etopol, param)

    def estimate(self, mesh, k, grid_size, Nmax, **opts):
        r, keep = self._request(mesh, k, grid_size, Nmax, **opts)
        b = C.c_int64()
        rc = self.lib.scd_server_estimate(C.byref(r), C.byref(b))
        if rc:
            raise ScadynError(rc, "scd_server_estimate")
        return int(b.value)

    def submit(self, mesh, k, grid_size, Nmax, **opts):
        r, keep = self._request(mesh, k, grid_size, Nmax, **opts)
        rid = C.c_int64()
        rc = self.lib.scd_server_submit(self.srv, C.byref(r), C.byref(rid))
        if rc:
            raise ScadynError(rc, "scd_server_submit")
        self._nmax[rid.value] = int(Nmax)
        return rid.value

    def poll(self, rid):
        st, status, lat = C.c_int32(), C.c_int32(), C.c_double()
        rc = self.lib.scd_server_poll(self.srv, rid, C.byref(st), C.byref(status), C.byref(lat))
        if rc:
            raise ScadynError(rc, "scd_server_poll")
        return st.value, status.value, lat.value

    def wait(self, rid, timeout=3600.0):
        rc = self.lib.scd_server_wait(self.srv, rid, float(timeout))
        if rc:
            raise ScadynError(rc, "scd_server_wait")

    def result(self, rid):
        """(T (ncol, ncol) with T[r, c], iterations per column, status)."""
        n = ncols(self._nmax[rid])
        Tf = np.zeros((n, n), np.complex128)   # column-major (ncol, ncol): Tf[c, r] = T(r, c)
        it = np.zeros(n, np.int32)
        rc = self.lib.scd_server_result(self.srv, rid, Tf.ctypes.data, it.ctypes.data)
        if rc not in (api.SCD_OK, api.SCD_NOT_CONVERGED):
            raise ScadynError(rc, "scd_server_result: " + self.error(rid))
        return Tf.T.copy(), it, rc

    def cancel(self, rid):
        return self.lib.scd_server_cancel(self.srv, rid)

    def error(self, rid):
        return (self.lib.scd_server_error(self.srv, rid) or b"").decode()

    def stats(self):
        s = Stats()
        self.lib.scd_server_stats_get(self.srv, C.byref(s))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def close(self):
        if self.srv:
            self.lib.scd_server_destroy(self.srv)
            self.srv = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
