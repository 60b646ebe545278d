"""Host-side mirror of scadyn's solver interface over the C ABI of
``libscadyn_gpu.so`` (include/scadyn_gpu.h).

Names follow the reference: ``compute_Ax2`` (src/gmres_module.f90:57),
``gmres`` (:180), ``compute_T_matrix`` (src/T_matrix.f90:240), ``build_G``
(src/build_G.f90), ``pfft_projection_const`` (src/projection.f90:17),
``compute_near_zone_interactions_const`` (src/precorrection.f90:131),
``vswf2constant`` (src/T_matrix.f90:280).  Arrays use the reference's Fortran
layouts, stored C-contiguous with the shape reversed (``S`` is ``(T, 27)``
memory of Fortran ``S(27, T)``).

There is no CPU fallback: importing succeeds without a GPU, but every call
that computes needs the CUDA library and a device and raises otherwise.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libscadyn_gpu.so")

SCD_OK, SCD_NOT_CONVERGED, SCD_NAN, SCD_OOM, SCD_BAD_ARG, SCD_TIMEOUT, SCD_CUDA_ERROR, SCD_NOT_READY, SCD_NO_DEVICE = range(9)
STORE_C64, STORE_C128 = 32, 64
PREC_FP64, PREC_MIXED = 0, 1
SCD_M_MAX = 63
FFT_DEFAULT, FFT_POW2, FFT_SMOOTH = 0, 1, 2
NEAR_DEFAULT, NEAR_CUDA_CORES, NEAR_TENSOR_SPLIT, NEAR_TENSOR_MERGED, NEAR_TENSOR_WIDE = 0, 1, 2, 3, 4
GS_DEFAULT, GS_MODIFIED, GS_CLASSICAL = 0, 1, 2
FFT_PASSES_DEFAULT, FFT_PASSES_FUSED_YZ, FFT_PASSES_THREE = 0, 1, 2

_NAMES = {0: "SCD_OK", 1: "SCD_NOT_CONVERGED", 2: "SCD_NAN", 3: "SCD_OOM", 4: "SCD_BAD_ARG",
          5: "SCD_TIMEOUT", 6: "SCD_CUDA_ERROR", 7: "SCD_NOT_READY", 8: "SCD_NO_DEVICE"}

# every symbol declared in include/scadyn_gpu.h
EXPORTS = [
    "scd_create", "scd_destroy", "scd_last_error", "scd_set_wavenumber", "scd_set_green",
    "scd_set_projectors", "scd_set_nearzone", "scd_grid_from_mesh", "scd_set_mesh",
    "scd_build_projectors", "scd_build_nearzone", "scd_get_projectors", "scd_nearzone_count",
    "scd_get_nearzone", "scd_matvec", "scd_gmres", "scd_set_rhs_matrix", "scd_solve_columns", "scd_vswf_rhs",
    "scd_get_timing", "scd_compute_T_matrix", "scd_profile_matvec", "scd_nearzone_bytes",
    "scd_column_latency", "scd_T_assemble_noalloc", "scd_selftest_waits", "scd_tune_matvec", "scd_apply_tuning",
    "scd_solve_sweep", "scd_compute_T_columns", "scd_check_matvec_repeat",
]


class ScadynError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_NAMES.get(code, code)}: {msg}")
        self.code = code


class GridDesc(C.Structure):
    _fields_ = [("Nx", C.c_int32), ("Ny", C.c_int32), ("Nz", C.c_int32), ("delta", C.c_double),
                ("min_coord", C.c_double * 3), ("T", C.c_int32), ("order", C.c_int32),
                ("M_ex", C.c_int32), ("near_zone", C.c_int32), ("device", C.c_int32),
                ("fft_lengths", C.c_int32), ("near_kernel", C.c_int32), ("near_split", C.c_int32),
                ("fft_passes", C.c_int32)]


class SolveOpts(C.Structure):
    _fields_ = [("tol", C.c_double), ("m", C.c_int32), ("cycles", C.c_int32), ("block", C.c_int32),
                ("precision", C.c_int32), ("inner_tol", C.c_double), ("max_outer", C.c_int32),
                ("gram_schmidt", C.c_int32)]


class Timing(C.Structure):
    _fields_ = [("matvec_ms", C.c_double), ("nearzone_ms", C.c_double), ("fft_ms", C.c_double),
                ("gather_ms", C.c_double), ("arnoldi_ms", C.c_double), ("last_call_ms", C.c_double),
                ("accum_ms", C.c_double), ("launches", C.c_int64), ("matvecs", C.c_int64),
                ("arnoldi_steps", C.c_int64), ("near_kernel_ms", C.c_double)]


class Tuning(C.Structure):
    _fields_ = [("nrhs", C.c_int32), ("precision", C.c_int32), ("near_kernel", C.c_int32), ("fft_passes", C.c_int32),
                ("scatter_span", C.c_int32), ("gather_span", C.c_int32), ("matvec_ms", C.c_double),
                ("default_ms", C.c_double)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Load libscadyn_gpu.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ScadynError(SCD_NOT_READY, f"{path} is missing: run scadyn_b200.build.build() (nvcc, sm_100a)")
    lib = C.CDLL(path)
    vp, i32, i64, dbl = C.c_void_p, C.c_int32, C.c_int64, C.c_double
    sig = {
        "scd_create": ([C.POINTER(vp), C.POINTER(GridDesc)], C.c_int),
        "scd_destroy": ([vp], C.c_int),
        "scd_last_error": ([vp], C.c_char_p),
        "scd_set_wavenumber": ([vp, dbl], C.c_int),
        "scd_set_green": ([vp, vp], C.c_int),
        "scd_set_projectors": ([vp, i32, i32, vp, vp, vp, vp, vp], C.c_int),
        "scd_set_nearzone": ([vp, i64, vp, vp, i32], C.c_int),
        "scd_grid_from_mesh": ([i32, vp, i32, vp, dbl, i32, C.POINTER(GridDesc)], C.c_int),
        "scd_set_mesh": ([vp, i32, vp, vp, vp], C.c_int),
        "scd_build_projectors": ([vp], C.c_int),
        "scd_build_nearzone": ([vp, i32], C.c_int),
        "scd_get_projectors": ([vp, vp, vp, vp, vp, vp], C.c_int),
        "scd_nearzone_count": ([vp], C.c_int64),
        "scd_get_nearzone": ([vp, i64, vp, vp], C.c_int),
        "scd_matvec": ([vp, vp, vp], C.c_int),
        "scd_gmres": ([vp, vp, vp, dbl, i32, i32, C.POINTER(i32), C.POINTER(dbl)], C.c_int),
        "scd_set_rhs_matrix": ([vp, i32, vp], C.c_int),
        "scd_solve_columns": ([vp, i32, vp, i32, i32, vp, C.POINTER(SolveOpts), vp, vp], C.c_int),
        "scd_vswf_rhs": ([vp, i32, vp], C.c_int),
        "scd_get_timing": ([vp, C.POINTER(Timing), i32], C.c_int),
        "scd_compute_T_matrix": ([vp, i32, C.POINTER(SolveOpts), i32, i32, vp, vp], C.c_int),
        "scd_compute_T_columns": ([vp, i32, C.POINTER(SolveOpts), i32, vp, vp, vp], C.c_int),
        "scd_profile_matvec": ([vp, i32, i32, i32], C.c_int),
        "scd_tune_matvec": ([vp, i32, i32, i32, C.POINTER(Tuning)], C.c_int),
        "scd_apply_tuning": ([vp, C.POINTER(Tuning)], C.c_int),
        "scd_solve_sweep": ([vp, i32, vp, C.POINTER(SolveOpts), vp, vp, vp], C.c_int),
        "scd_nearzone_bytes": ([vp], C.c_int64),
        "scd_column_latency": ([vp, i32, vp], C.c_int),
        "scd_T_assemble_noalloc": ([vp, i64, i32, vp, i32, vp, vp], C.c_int),
        "scd_selftest_waits": ([i32], C.c_int),
        "scd_check_matvec_repeat": ([vp, i32, i32, i32, C.POINTER(C.c_int64), C.POINTER(C.c_int64)], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


def _c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)


def grid_from_mesh(coord, etopol, grid_size=1.8, M_ex=2, order=0) -> GridDesc:
    """build_grid (src/geometry.f90:60-125) -> GridDesc; order 1 selects the linear basis."""
    lib = load_library()
    coord = np.ascontiguousarray(coord, np.float64)
    etopol = np.ascontiguousarray(etopol, np.int32)
    d = GridDesc()
    rc = lib.scd_grid_from_mesh(coord.shape[0], _p(coord), etopol.shape[0], _p(etopol), grid_size, M_ex, C.byref(d))
    if rc:
        raise ScadynError(rc, "scd_grid_from_mesh")
    d.order = order
    return d


def T_assemble_noalloc(mat_ptr, n, ncol, X_ptr, ncb, T_ptr, stream=0):
    """T = mat^H X on caller-owned device buffers, allocating nothing
    (scd_T_assemble_noalloc).  Pointers are device addresses (ints)."""
    lib = load_library()
    rc = lib.scd_T_assemble_noalloc(C.c_void_p(mat_ptr), n, ncol, C.c_void_p(X_ptr), ncb, C.c_void_p(T_ptr),
                                    C.c_void_p(stream))
    if rc:
        raise ScadynError(rc, "scd_T_assemble_noalloc")


def solve_sweep(solvers, Nmax, tol=1e-6, m=30, cycles=60, block=32, precision=PREC_MIXED, inner_tol=3e-4,
                max_outer=10, gram_schmidt=GS_DEFAULT):
    """scd_solve_sweep: the T-matrices of every wavelength of a sweep in one
    batched solve (calc_T's wavelength loop, src/T_matrix.f90:36-79).
    solvers[w] holds wavelength w's operator on the same mesh; Nmax[w] its
    VSWF order.  Returns ([T_w (2nm_w, 2nm_w)], [iters_w], [status_w], rc)."""
    lib = load_library()
    nw = len(solvers)
    ctxs = (C.c_void_p * nw)(*[s.ctx.value for s in solvers])
    nm = np.ascontiguousarray(Nmax, np.int32)
    ncol = [2 * ((int(v) + 1) ** 2 - 1) for v in nm]
    Ts = [np.zeros((c, c), np.complex128) for c in ncol]       # memory of Fortran T(2nm, 2nm)
    its = [np.zeros(c, np.int32) for c in ncol]
    Tp = (C.c_void_p * nw)(*[t.ctypes.data for t in Ts])
    Ip = (C.c_void_p * nw)(*[i.ctypes.data for i in its])
    st = np.zeros(nw, np.int32)
    o = SolveOpts(tol, m, cycles, block, precision, inner_tol, max_outer, gram_schmidt)
    rc = lib.scd_solve_sweep(C.cast(ctxs, C.c_void_p), nw, _p(nm), C.byref(o), C.cast(Tp, C.c_void_p),
                             C.cast(Ip, C.c_void_p), _p(st))
    if rc not in (SCD_OK, SCD_NOT_CONVERGED):
        raise ScadynError(rc, "scd_solve_sweep: " + lib.scd_last_error(solvers[0].ctx).decode())
    return [t.T.copy() for t in Ts], its, st, rc


@dataclass
class GridInfo:
    Nx: int
    Ny: int
    Nz: int
    delta: float
    min_coord: tuple
    T: int


class Solver:
    """One device context (scd_ctx) for one mesh and grid."""

    def __init__(self, Nx, Ny, Nz, delta, min_coord, T, device=0, order=0, fft_lengths=FFT_DEFAULT,
                 near_kernel=NEAR_DEFAULT, near_split=0, fft_passes=FFT_PASSES_DEFAULT):
        """order 1 (linear basis): 4 projector columns and 12 unknowns per tet.
        The operator comes from the host (set_projectors, set_nearzone with
        12x12 blocks) or from the mesh on the device (set_mesh,
        pfft_projection_lin, compute_near_zone_interactions_lin); compute_Ax2,
        gmres and solve_columns run on it.  The VSWF right-hand sides and the
        T-matrix entry points are constant-basis only, as in the reference.
        fft_lengths, near_kernel and near_split are the kernel choices of
        scd_grid_desc (0 = the library's default)."""
        self.lib = load_library()
        d = GridDesc()
        d.Nx, d.Ny, d.Nz, d.delta = Nx, Ny, Nz, delta
        for i in range(3):
            d.min_coord[i] = float(min_coord[i])
        d.T, d.order, d.M_ex, d.near_zone, d.device = T, order, 2, 1, device
        d.fft_lengths, d.near_kernel, d.near_split = fft_lengths, near_kernel, near_split
        d.fft_passes = fft_passes
        self.desc = d
        self.order = order
        self.T = (4 if order == 1 else 1) * T      # projector columns (basis functions)
        self.n = 3 * self.T
        h = C.c_void_p()
        rc = self.lib.scd_create(C.byref(h), C.byref(d))
        self.ctx = h
        if rc:
            msg = self.lib.scd_last_error(h).decode() if h.value else "scd_create"
            if h.value:
                self.lib.scd_destroy(h)
                self.ctx = C.c_void_p()
            raise ScadynError(rc, msg)

    @classmethod
    def from_desc(cls, d: GridDesc, device=0):
        return cls(d.Nx, d.Ny, d.Nz, d.delta, list(d.min_coord), d.T, device, order=d.order,
                   fft_lengths=d.fft_lengths, near_kernel=d.near_kernel, near_split=d.near_split,
                   fft_passes=d.fft_passes)

    def _chk(self, rc, what, ok=(SCD_OK,)):
        if rc not in ok:
            raise ScadynError(rc, f"{what}: {self.lib.scd_last_error(self.ctx).decode()}")
        return rc

    def close(self):
        if self.ctx and self.ctx.value:
            self.lib.scd_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --- operator pieces
    def set_wavenumber(self, k):
        self._chk(self.lib.scd_set_wavenumber(self.ctx, float(k)), "set_wavenumber")
        self._k = float(k)

    def problem_key(self):
        """Identity of the problem this context solves, for checkpoints:
        unknowns, grid, wavenumber and a digest of the mesh (set_mesh) or of
        the host projectors (set_projectors) it was set up from; None before
        either is known."""
        src = getattr(self, "_mesh_digest", None) or getattr(self, "_proj_digest", None)
        if src is None or not hasattr(self, "_k"):
            return None
        d = self.desc
        return {"n": int(self.n), "grid": [int(d.Nx), int(d.Ny), int(d.Nz)], "delta": float(d.delta),
                "k": self._k, "source": src}

    def build_G(self, Fg=None):
        """matrices%Fg; None builds it on the device (src/build_G.f90)."""
        if Fg is None:
            self._chk(self.lib.scd_set_green(self.ctx, None), "build_G")
        else:
            Fg = _c128(Fg)
            self._chk(self.lib.scd_set_green(self.ctx, _p(Fg)), "set_green")

    def set_projectors(self, S, Sx, Sy, Sz, indS):
        S, Sx, Sy, Sz = (_c128(a) for a in (S, Sx, Sy, Sz))
        indS = np.ascontiguousarray(indS, np.int32)
        self._chk(self.lib.scd_set_projectors(self.ctx, 27, self.T, _p(S), _p(Sx), _p(Sy), _p(Sz), _p(indS)),
                  "set_projectors")
        h = hashlib.sha256()
        for a in (S, Sx, Sy, Sz, indS):
            h.update(a.tobytes())
        self._proj_digest = "projectors:" + h.hexdigest()

    def set_nearzone(self, sp_mat, sp_ind):
        sp_ind = np.ascontiguousarray(sp_ind, np.int32)
        if sp_mat.dtype == np.complex64:
            sp = np.ascontiguousarray(sp_mat)
            prec = STORE_C64
        else:
            sp = _c128(sp_mat)
            prec = STORE_C128
        self._chk(self.lib.scd_set_nearzone(self.ctx, sp_ind.shape[0], _p(sp), _p(sp_ind), prec), "set_nearzone")

    def set_mesh(self, coord, etopol, param):
        self._coord = np.ascontiguousarray(coord, np.float64)
        self._etopol = np.ascontiguousarray(etopol, np.int32)
        self._param = _c128(param)
        self._chk(self.lib.scd_set_mesh(self.ctx, self._coord.shape[0], _p(self._coord), _p(self._etopol),
                                        _p(self._param)), "set_mesh")
        h = hashlib.sha256()
        for a in (self._coord, self._etopol, self._param):
            h.update(a.tobytes())
        self._mesh_digest = "mesh:" + h.hexdigest()

    def pfft_projection_const(self):
        """Projectors on the device; returns (S, Sx, Sy, Sz, indS) in the reference layout."""
        self._chk(self.lib.scd_build_projectors(self.ctx), "build_projectors")
        return self.get_projectors()

    def get_projectors(self):
        S, Sx, Sy, Sz = (np.zeros((self.T, 27), np.complex128) for _ in range(4))
        indS = np.zeros((self.T, 27), np.int32)
        self._chk(self.lib.scd_get_projectors(self.ctx, _p(S), _p(Sx), _p(Sy), _p(Sz), _p(indS)), "get_projectors")
        return S, Sx, Sy, Sz, indS

    def pfft_projection_lin(self):
        """Linear-basis projectors on the device (src/projection.f90:170-338): (4T, 27) columns."""
        return self.pfft_projection_const()

    def compute_near_zone_interactions_const(self, storage=STORE_C64):
        self._chk(self.lib.scd_build_nearzone(self.ctx, storage), "build_nearzone")

    def compute_near_zone_interactions_lin(self, storage=STORE_C64):
        """Linear-basis 12x12 near-zone blocks on the device (src/precorrection.f90:268-725)."""
        self.compute_near_zone_interactions_const(storage)

    def get_nearzone(self):
        """(sp_mat, sp_ind) ordered by (tet_T, tet_B): (B, 3, 3) blocks, or (B, 12, 12) with the linear basis."""
        B = self.lib.scd_nearzone_count(self.ctx)
        if B < 0:
            raise ScadynError(SCD_NOT_READY, "near zone not set")
        nbk = 12 if self.order == 1 else 3
        sp = np.zeros((B, nbk, nbk), np.complex128)
        ind = np.zeros((B, 2), np.int32)
        self._chk(self.lib.scd_get_nearzone(self.ctx, B, _p(sp), _p(ind)), "get_nearzone")
        return sp, ind

    # --- hot path
    def compute_Ax2(self, x):
        x = _c128(x)
        Ax = np.zeros_like(x)
        self._chk(self.lib.scd_matvec(self.ctx, _p(x), _p(Ax)), "matvec")
        return Ax

    def gmres(self, rhs, tol=1e-5, m=50, cycles=4):
        rhs = _c128(rhs)
        x = np.zeros_like(rhs)
        it = C.c_int32()
        rr = C.c_double()
        rc = self._chk(self.lib.scd_gmres(self.ctx, _p(rhs), _p(x), tol, m, cycles, C.byref(it), C.byref(rr)),
                       "gmres", ok=(SCD_OK, SCD_NOT_CONVERGED))
        return x, {"iters": it.value, "relres": rr.value, "converged": rc == SCD_OK}

    def vswf2constant(self, Nmax):
        nm = (Nmax + 1) ** 2 - 1
        mat = np.zeros((2 * nm, self.n), np.complex128)
        self._chk(self.lib.scd_vswf_rhs(self.ctx, Nmax, _p(mat)), "vswf_rhs")
        return mat

    def set_rhs_matrix(self, mat):
        """The incident matrix (vswf2constant, src/T_matrix.f90:252), mat
        (nmat, n) memory of Fortran mat(n, nmat), kept on the device for
        solve_columns(None, ...)."""
        mat = _c128(mat)
        self._nmat = mat.shape[0]
        self._chk(self.lib.scd_set_rhs_matrix(self.ctx, mat.shape[0], _p(mat)), "set_rhs_matrix")

    def solve_columns(self, mat, col0=0, ncol=None, tol=1e-5, m=50, cycles=4, block=1, precision=PREC_FP64,
                      inner_tol=1e-3, max_outer=10, gram_schmidt=GS_DEFAULT, want_x=False, nmat=None):
        """The column loop of compute_T_matrix over columns col0 .. col0+ncol-1
        of mat (nmat, n) (memory of Fortran mat(n, nmat)), or of the matrix of
        set_rhs_matrix when mat is None.  Returns (Tc, iters, X, rc): Tc
        (ncol, nmat) is the memory of Fortran T_mat(nmat, ncol), i.e.
        Tc[j, r] = T_mat(r, col0+j) = (mat^H x_j)[r] unscaled; X (ncol, n)."""
        if mat is not None:
            mat = _c128(mat)
            nmat = mat.shape[0]
        elif nmat is None:
            nmat = self._nmat
        if ncol is None:
            ncol = nmat - col0
        Tc = np.zeros((ncol, nmat), np.complex128)
        iters = np.zeros(ncol, np.int32)
        X = np.zeros((ncol, self.n), np.complex128) if want_x else None
        o = SolveOpts(tol, m, cycles, block, precision, inner_tol, max_outer, gram_schmidt)
        rc = self._chk(self.lib.scd_solve_columns(self.ctx, nmat, _p(mat), col0, ncol, _p(Tc), C.byref(o),
                                                  _p(iters), _p(X)),
                       "solve_columns", ok=(SCD_OK, SCD_NOT_CONVERGED))
        return Tc, iters, X, rc

    def compute_T_matrix(self, Nmax, col0=0, ncol=None, tol=1e-5, m=50, cycles=4, block=1,
                         precision=PREC_FP64, inner_tol=1e-3, max_outer=10, gram_schmidt=GS_DEFAULT):
        """compute_T_matrix (src/T_matrix.f90:240-277) on device-resident data:
        returns (T (2nm, ncol) with T[:, j] the scaled T column col0+j, iters).
        With all columns, T = [[Taa, Tab], [Tba, Tbb]]."""
        nm = (Nmax + 1) ** 2 - 1
        if ncol is None:
            ncol = 2 * nm - col0
        Tf = np.zeros((ncol, 2 * nm), np.complex128)       # memory of Fortran T(2nm, ncol)
        iters = np.zeros(ncol, np.int32)
        o = SolveOpts(tol, m, cycles, block, precision, inner_tol, max_outer, gram_schmidt)
        self._chk(self.lib.scd_compute_T_matrix(self.ctx, Nmax, C.byref(o), col0, ncol, _p(Tf), _p(iters)),
                  "compute_T_matrix", ok=(SCD_OK, SCD_NOT_CONVERGED))
        return Tf.T, iters

    def compute_T_columns(self, Nmax, cols, tol=1e-5, m=50, cycles=4, block=1, precision=PREC_FP64,
                          inner_tol=1e-3, max_outer=10, gram_schmidt=GS_DEFAULT):
        """compute_T_matrix over the 0-based columns `cols` (any order, each
        once): returns (T (2nm, len(cols)) with T[:, j] the scaled column
        cols[j], iters)."""
        nm = (Nmax + 1) ** 2 - 1
        cols = np.ascontiguousarray(cols, np.int32)
        Tf = np.zeros((len(cols), 2 * nm), np.complex128)
        iters = np.zeros(len(cols), np.int32)
        o = SolveOpts(tol, m, cycles, block, precision, inner_tol, max_outer, gram_schmidt)
        self._chk(self.lib.scd_compute_T_columns(self.ctx, Nmax, C.byref(o), len(cols), _p(cols), _p(Tf),
                                                 _p(iters)),
                  "compute_T_columns", ok=(SCD_OK, SCD_NOT_CONVERGED))
        return Tf.T, iters

    def profile_matvec(self, reps=10, nrhs=1, precision=PREC_FP64):
        self._chk(self.lib.scd_profile_matvec(self.ctx, reps, nrhs, precision), "profile_matvec")
        return self.timing()

    def check_matvec_repeat(self, reps=100, nrhs=1, precision=PREC_MIXED):
        """scd_check_matvec_repeat: (repetitions whose output differed in any
        bit from the first matvec of the same inputs, differing 32-bit words)."""
        br, bw = C.c_int64(0), C.c_int64(0)
        self._chk(self.lib.scd_check_matvec_repeat(self.ctx, reps, nrhs, precision, C.byref(br), C.byref(bw)),
                  "check_matvec_repeat")
        return br.value, bw.value

    def tune_matvec(self, nrhs, precision=PREC_MIXED, reps=10):
        """scd_tune_matvec: time the matvec kernel choices, keep the fastest
        (applied to this context) and return it as a dict."""
        t = Tuning()
        self._chk(self.lib.scd_tune_matvec(self.ctx, nrhs, precision, reps, C.byref(t)), "tune_matvec")
        return {f: getattr(t, f) for f, _ in Tuning._fields_}

    def apply_tuning(self, tuning):
        """scd_apply_tuning with a dict of tune_matvec's fields."""
        t = Tuning(**{f: tuning[f] for f, _ in Tuning._fields_ if f in tuning})
        self._chk(self.lib.scd_apply_tuning(self.ctx, C.byref(t)), "apply_tuning")

    def column_latency(self, ncol):
        ms = np.zeros(ncol, np.float64)
        self._chk(self.lib.scd_column_latency(self.ctx, ncol, _p(ms)), "column_latency")
        return ms

    def nearzone_bytes(self):
        return int(self.lib.scd_nearzone_bytes(self.ctx))

    def nearzone_count(self):
        return int(self.lib.scd_nearzone_count(self.ctx))

    def timing(self, reset=False):
        t = Timing()
        self.lib.scd_get_timing(self.ctx, C.byref(t), int(reset))
        return {f: getattr(t, f) for f, _ in Timing._fields_}
