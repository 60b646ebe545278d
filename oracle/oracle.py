"""ctypes binding of the CPU oracle (``oracle/liborc.so``) — TEST INFRASTRUCTURE.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, to check results.  The oracle restates the reference's
Fortran algorithm (jherrane/scadyn ``src/``); parity against the reference is
UNPINNED (no golden vectors exist upstream).

All arrays use the reference's Fortran layouts, stored C-contiguous with the
shape reversed, e.g. ``S`` is a ``(T, 27)`` complex128 array whose memory is
the Fortran ``S(27, T)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liborc.so")


def build() -> str:
    src = os.path.join(_HERE, "oracle.c")
    if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


class _Geom(C.Structure):
    _fields_ = [
        ("Nv", C.c_int), ("T", C.c_int),
        ("coord", C.c_void_p), ("etopol", C.c_void_p), ("param", C.c_void_p),
        ("grid_size", C.c_double), ("M_ex", C.c_int), ("near_zone", C.c_int), ("k", C.c_double),
        ("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
        ("delta", C.c_double), ("box_delta", C.c_double), ("min_coord", C.c_double * 3),
        ("Nx_cube", C.c_int), ("Ny_cube", C.c_int), ("Nz_cube", C.c_int), ("N_cubes", C.c_int),
        ("etopol_box", C.POINTER(C.c_int32)),
        ("N_tet_cube", C.c_int),
        ("tetras", C.POINTER(C.c_int32)),
    ]


class _Op(C.Structure):
    _fields_ = [
        ("g", C.c_void_p), ("T", C.c_int),
        ("S", C.c_void_p), ("Sx", C.c_void_p), ("Sy", C.c_void_p), ("Sz", C.c_void_p),
        ("indS", C.c_void_p), ("Fg", C.c_void_p),
        ("B", C.c_int64), ("sp32", C.c_void_p), ("sp64", C.c_void_p), ("sp_ind", C.c_void_p),
        ("k", C.c_double), ("merged", C.c_int), ("nthreads", C.c_int), ("order", C.c_int),
    ]


class _Info(C.Structure):
    _fields_ = [("iters", C.c_int), ("matvecs", C.c_int), ("cycles", C.c_int),
                ("converged", C.c_int), ("relres", C.c_double),
                ("history", C.POINTER(C.c_double)), ("history_len", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.orc_nearzone_count.restype = C.c_int64
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a is not None else C.c_void_p(0)


@dataclass
class Geometry:
    """build_grid + build_box + tetras_in_cubes (src/geometry.f90)."""
    coord: np.ndarray
    etopol: np.ndarray
    param: np.ndarray
    k: float
    grid_size: float = 1.8
    M_ex: int = 2
    near_zone: int = 1

    def __post_init__(self):
        self.coord = np.ascontiguousarray(self.coord, dtype=np.float64)
        self.etopol = np.ascontiguousarray(self.etopol, dtype=np.int32)
        self.param = np.ascontiguousarray(self.param, dtype=np.complex128)
        g = _Geom()
        g.Nv = self.coord.shape[0]
        g.T = self.etopol.shape[0]
        g.coord = self.coord.ctypes.data
        g.etopol = self.etopol.ctypes.data
        g.param = self.param.ctypes.data
        g.grid_size = self.grid_size
        g.M_ex = self.M_ex
        g.near_zone = self.near_zone
        g.k = self.k
        rc = lib().orc_geom_build(C.byref(g))
        if rc != 0:
            raise RuntimeError(f"orc_geom_build failed ({rc})")
        self._g = g
        self.Nx, self.Ny, self.Nz = g.Nx, g.Ny, g.Nz
        self.delta, self.box_delta = g.delta, g.box_delta
        self.min_coord = np.array(list(g.min_coord))
        self.N_cubes = g.N_cubes
        self.cube_dims = (g.Nx_cube, g.Ny_cube, g.Nz_cube)
        self.N_tet_cube = g.N_tet_cube
        self.etopol_box = np.ctypeslib.as_array(g.etopol_box, shape=(g.N_cubes, 27)).copy()
        self.tetras = np.ctypeslib.as_array(g.tetras, shape=(g.N_cubes, g.N_tet_cube)).copy()

    @property
    def T(self):
        return self.etopol.shape[0]

    def set_k(self, k: float):
        self.k = k
        self._g.k = k

    def __del__(self):
        try:
            lib().orc_geom_free(C.byref(self._g))
        except Exception:
            pass

    def near_cubes(self, cube1: int) -> np.ndarray:
        out = np.zeros(125, dtype=np.int32)
        n = lib().orc_find_near_cubes(C.byref(self._g), cube1, _p(out))
        return out[:n]

    def projectors(self):
        """pfft_projection_const -> S, Sx, Sy, Sz (T,27) c128 and indS (T,27) int32."""
        T = self.T
        S, Sx, Sy, Sz = (np.zeros((T, 27), np.complex128) for _ in range(4))
        indS = np.zeros((T, 27), np.int32)
        rc = lib().orc_pfft_projection_const(C.byref(self._g), _p(S), _p(Sx), _p(Sy), _p(Sz), _p(indS))
        if rc != 0:
            raise RuntimeError(f"projection failed ({rc})")
        return S, Sx, Sy, Sz, indS

    def nearzone(self, S, Sx, Sy, Sz, fp64: bool = False, nthreads: int = 0):
        """compute_near_zone_interactions_const -> (sp_mat (B,3,3) [memory (3,3,B)], sp_ind (B,2))."""
        B = lib().orc_nearzone_count(C.byref(self._g))
        sp32 = None if fp64 else np.zeros((B, 3, 3), np.complex64)
        sp64 = np.zeros((B, 3, 3), np.complex128) if fp64 else None
        ind = np.zeros((B, 2), np.int32)
        rc = lib().orc_nearzone_const(C.byref(self._g), _p(S), _p(Sx), _p(Sy), _p(Sz), C.c_int64(B),
                                      _p(sp32), _p(sp64), _p(ind), nthreads)
        if rc != 0:
            raise RuntimeError(f"nearzone failed ({rc})")
        return (sp64 if fp64 else sp32), ind

    def projectors_lin(self):
        """pfft_projection_lin -> S, Sx, Sy, Sz (4T,27) c128 and indS (4T,27) int32; row 4t+n is node n of tet t."""
        T4 = 4 * self.T
        S, Sx, Sy, Sz = (np.zeros((T4, 27), np.complex128) for _ in range(4))
        indS = np.zeros((T4, 27), np.int32)
        rc = lib().orc_pfft_projection_lin(C.byref(self._g), _p(S), _p(Sx), _p(Sy), _p(Sz), _p(indS))
        if rc != 0:
            raise RuntimeError(f"linear projection failed ({rc})")
        return S, Sx, Sy, Sz, indS

    def nearzone_lin(self, S, Sx, Sy, Sz, fp64: bool = False, nthreads: int = 0):
        """compute_near_zone_interactions_lin -> (sp_mat (B,12,12) [memory (12,12,B)], sp_ind (B,2))."""
        B = lib().orc_nearzone_count(C.byref(self._g))
        sp32 = None if fp64 else np.zeros((B, 12, 12), np.complex64)
        sp64 = np.zeros((B, 12, 12), np.complex128) if fp64 else None
        ind = np.zeros((B, 2), np.int32)
        rc = lib().orc_nearzone_lin(C.byref(self._g), _p(S), _p(Sx), _p(Sy), _p(Sz), C.c_int64(B),
                                    _p(sp32), _p(sp64), _p(ind), nthreads)
        if rc != 0:
            raise RuntimeError(f"linear near zone failed ({rc})")
        return (sp64 if fp64 else sp32), ind

    def build_G(self):
        """build_G -> Fg (2Nz, 2Ny, 2Nx) c128 (memory of Fortran Fg(2Nx,2Ny,2Nz))."""
        Fg = np.zeros((2 * self.Nz, 2 * self.Ny, 2 * self.Nx), np.complex128)
        lib().orc_build_G(C.byref(self._g), _p(Fg))
        return Fg


@dataclass
class Operator:
    geom: Geometry
    S: np.ndarray
    Sx: np.ndarray
    Sy: np.ndarray
    Sz: np.ndarray
    indS: np.ndarray
    Fg: np.ndarray
    sp_mat: np.ndarray
    sp_ind: np.ndarray
    merged: bool = False
    nthreads: int = 1
    order: int = 0          # 1: linear basis, S (4T, 27), sp_mat (B, 12, 12), 12 unknowns per tet

    def _op(self):
        o = _Op()
        o.g = C.addressof(self.geom._g)
        o.T = self.S.shape[0] // (4 if self.order == 1 else 1)   # tets (projector columns / basis functions per tet)
        o.S, o.Sx, o.Sy, o.Sz = (a.ctypes.data for a in (self.S, self.Sx, self.Sy, self.Sz))
        o.indS = self.indS.ctypes.data
        o.Fg = self.Fg.ctypes.data
        o.B = self.sp_ind.shape[0]
        if self.sp_mat.dtype == np.complex64:
            o.sp32, o.sp64 = self.sp_mat.ctypes.data, None
        else:
            o.sp32, o.sp64 = None, self.sp_mat.ctypes.data
        o.sp_ind = self.sp_ind.ctypes.data
        o.k = self.geom.k
        o.merged = int(self.merged)
        o.nthreads = self.nthreads
        o.order = int(self.order)
        return o

    def compute_Ax2(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        Ax = np.zeros_like(x)
        o = self._op()
        lib().orc_compute_Ax2(C.byref(o), _p(x), _p(Ax))
        return Ax

    def gmres(self, rhs: np.ndarray, tol: float = 1e-5, m: int = 50, cycles: int = 4):
        rhs = np.ascontiguousarray(rhs, dtype=np.complex128)
        x = np.zeros_like(rhs)
        hist = np.zeros(m * cycles + 1, np.float64)
        info = _Info()
        info.history = hist.ctypes.data_as(C.POINTER(C.c_double))
        info.history_len = hist.shape[0]
        o = self._op()
        lib().orc_gmres(C.byref(o), _p(rhs), _p(x), C.c_double(tol), m, cycles, C.byref(info))
        return x, {"iters": info.iters, "matvecs": info.matvecs, "cycles": info.cycles,
                   "converged": bool(info.converged), "relres": info.relres,
                   "history": hist[: info.history_len].copy()}


def mgs_terms(V: np.ndarray, w: np.ndarray) -> np.ndarray:
    """One Arnoldi step's modified Gram-Schmidt of w (in place) against the
    rows of V (i, n), as orc_gmres does it; returns the coefficients h."""
    V = np.ascontiguousarray(V, np.complex128)
    h = np.zeros(V.shape[0], np.complex128)
    f = lib().orc_mgs_terms
    f.argtypes = [C.c_size_t, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    f(V.shape[1], V.shape[0], _p(V), _p(w), _p(h))
    return h


def linear_from_constant(op, seed=0):
    """A linear-basis (order 1) operator on the geometry of a constant-basis
    one, for parity of the order-1 matvec: each tet's projector column is
    split over its 4 nodes with seeded weights (one column per basis function,
    same box nodes, as pfft_projection_lin stores them, src/projection.f90:
    170-338), and each 3x3 near-zone block V becomes the 12x12 block
    V(c, c') * m(i, j), m seeded and not symmetric (self blocks included)."""
    rng = np.random.default_rng(seed)
    T = op.geom.T
    w = 0.25 + 0.05 * rng.standard_normal((T, 4, 4))          # per tet and node, one weight per projector kind

    def split(P, kind):
        return np.ascontiguousarray((P[:, None, :] * w[:, :, kind, None]).reshape(4 * T, 27))

    S1, Sx1, Sy1, Sz1 = (split(P, q) for q, P in enumerate((op.S, op.Sx, op.Sy, op.Sz)))
    indS1 = np.ascontiguousarray(np.repeat(op.indS, 4, axis=0))
    B = op.sp_ind.shape[0]
    m = (np.eye(4)[None] + 0.1 * (rng.standard_normal((B, 4, 4)) + 1j * rng.standard_normal((B, 4, 4)))) / 2
    V = op.sp_mat.astype(np.complex128)       # memory (3,3,B): V[b, c', c] = V(c, c')
    # 12x12 block, memory (12,12,B): A[b, 4c'+j, 4c+i] = V(c, c') m(i, j)
    A = np.einsum("bdc,bij->bdjci", V, m).reshape(B, 12, 12)
    sp12 = np.ascontiguousarray(A.astype(op.sp_mat.dtype))
    return Operator(op.geom, S1, Sx1, Sy1, Sz1, indS1, op.Fg, sp12, op.sp_ind.copy(), merged=op.merged,
                    nthreads=op.nthreads, order=1)


def matmul_Acorr(T, sp_mat, sp_ind, x):
    """matmul_Acorr (12x12 blocks, src/sparse_mat.f90:64-92)."""
    x = np.ascontiguousarray(x, dtype=np.complex128)
    Ax = np.zeros(12 * T, np.complex128)
    sp32 = sp_mat if sp_mat.dtype == np.complex64 else None
    sp64 = sp_mat if sp_mat.dtype == np.complex128 else None
    lib().orc_matmul_Acorr(T, C.c_int64(sp_ind.shape[0]), _p(sp32), _p(sp64), _p(sp_ind), _p(x), _p(Ax))
    return Ax


def matmul_Acorr_const(T, sp_mat, sp_ind, x, nthreads=1):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    Ax = np.zeros(3 * T, np.complex128)
    sp32 = sp_mat if sp_mat.dtype == np.complex64 else None
    sp64 = sp_mat if sp_mat.dtype == np.complex128 else None
    lib().orc_matmul_Acorr_const(T, C.c_int64(sp_ind.shape[0]), _p(sp32), _p(sp64), _p(sp_ind), _p(x), _p(Ax), nthreads)
    return Ax


def fft3d(A: np.ndarray, sign: int = -1) -> np.ndarray:
    A = np.ascontiguousarray(A, dtype=np.complex128).copy()
    Pz, Py, Px = A.shape
    lib().orc_fft3d(Px, Py, Pz, _p(A), sign)
    return A


def fft3d_pruned(A: np.ndarray, inverse: bool) -> np.ndarray:
    A = np.ascontiguousarray(A, dtype=np.complex128).copy()
    Pz, Py, Px = A.shape
    lib().orc_fft3d_pruned(Px, Py, Pz, _p(A), int(inverse))
    return A


def pinv(A: np.ndarray) -> np.ndarray:
    """A given as Fortran (M,N) -> numpy array of shape (N, M) [memory (M,N)]."""
    A = np.ascontiguousarray(A, dtype=np.complex128)
    N, M = A.shape
    out = np.zeros((M, N), np.complex128)
    lib().orc_pinv(M, N, _p(A), _p(out))
    return out


class _Z(C.Structure):
    _fields_ = [("re", C.c_double), ("im", C.c_double)]


def _z(v):
    return _Z(float(np.real(v)), float(np.imag(v)))


def vswf2constant(coord, etopol, k, Nmax):
    """vswf2constant -> mat, a (2nm, 3T) array (memory of Fortran mat(3T, 2nm))."""
    T = etopol.shape[0]
    nm = (Nmax + 1) ** 2 - 1
    mat = np.zeros((2 * nm, 3 * T), np.complex128)
    fn = lib().orc_vswf2constant
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int, _Z, C.c_int, C.c_void_p]
    fn(_p(np.ascontiguousarray(coord, np.float64)), _p(np.ascontiguousarray(etopol, np.int32)),
       T, _z(k), Nmax, _p(mat))
    return mat


def calc_MN(Nmax, k, Po):
    nm = (Nmax + 1) ** 2 - 1
    MM = np.zeros((nm, 3), np.complex128)
    NN = np.zeros((nm, 3), np.complex128)
    fn = lib().orc_calc_MN
    fn.argtypes = [C.c_int, _Z, C.c_void_p, C.c_void_p, C.c_void_p]
    P = np.ascontiguousarray(Po, np.float64)
    fn(Nmax, _z(k), _p(P), _p(MM), _p(NN))
    return MM, NN


def cspherebessel(n, z):
    csj = np.zeros(n + 1, np.complex128)
    csy = np.zeros(n + 1, np.complex128)
    fn = lib().orc_cspherebessel
    fn.argtypes = [C.c_int, _Z, C.c_void_p, C.c_void_p]
    fn(n, _z(z), _p(csj), _p(csy))
    return csj, csy


def mie_T(Nmax, ka, m):
    a = np.zeros(Nmax, np.complex128)
    b = np.zeros(Nmax, np.complex128)
    fn = lib().orc_mie_T
    fn.argtypes = [C.c_int, C.c_double, _Z, C.c_void_p, C.c_void_p]
    fn(Nmax, ka, _z(m), _p(a), _p(b))
    return a, b


def T_assemble(mat, X):
    """T_cols = mat^H X; mat memory (n, ncol), X memory (n, ncol)."""
    mat = np.ascontiguousarray(mat, np.complex128)
    X = np.ascontiguousarray(X, np.complex128)
    ncol, n = mat.shape
    out = np.zeros((ncol, ncol), np.complex128)
    lib().orc_T_assemble(n, ncol, _p(mat), _p(X), _p(out))
    return out          # memory of Fortran T(ncol, ncol): out[c, r] = T(r, c)


def tr_T(Taa, Tbb, Tab, Tba, k):
    crs = np.zeros(4)
    nm = Taa.shape[0]
    args = [np.ascontiguousarray(t, np.complex128) for t in (Taa, Tbb, Tab, Tba)]
    lib().orc_tr_T(nm, *[_p(a) for a in args], C.c_double(k), _p(crs))
    return crs


def setup(mesh, k, grid_size=1.8, fp64_near=False, nthreads=0):
    """Full per-wavelength setup: geometry, projectors, Green grid, near zone."""
    g = Geometry(mesh.coord, mesh.etopol, mesh.param, k=k, grid_size=grid_size)
    S, Sx, Sy, Sz, indS = g.projectors()
    Fg = g.build_G()
    sp, ind = g.nearzone(S, Sx, Sy, Sz, fp64=fp64_near, nthreads=nthreads)
    return Operator(g, S, Sx, Sy, Sz, indS, Fg, sp, ind)


def setup_lin(mesh, k, grid_size=1.8, fp64_near=False, nthreads=0):
    """Per-wavelength setup with the linear basis (mesh%order = 1): geometry,
    pfft_projection_lin, Green grid, compute_near_zone_interactions_lin."""
    g = Geometry(mesh.coord, mesh.etopol, mesh.param, k=k, grid_size=grid_size)
    S, Sx, Sy, Sz, indS = g.projectors_lin()
    Fg = g.build_G()
    sp, ind = g.nearzone_lin(S, Sx, Sy, Sz, fp64=fp64_near, nthreads=nthreads)
    return Operator(g, S, Sx, Sy, Sz, indS, Fg, sp, ind, order=1)


def analytical_integration(tri, r):
    """analytical_integration (src/singularity_subtraction.f90:15-108) at one
    point: [int_tri 1/R dS, int_tri R dS]; tri (3,3)."""
    out = np.zeros(2, np.float64)
    lib().orc_analytical_integration(_p(np.ascontiguousarray(tri, np.float64)),
                                     _p(np.ascontiguousarray(r, np.float64)), _p(out))
    return out


def int_V_G(rf, k, B):
    """singularity_subtraction_int_V_G (src/singularity_subtraction.f90:112-189)
    at one point: int_B G(rf, r') dV'; B (4,3)."""
    f = lib().orc_int_V_G
    f.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
    f.restype = _Z
    z = f(_p(np.ascontiguousarray(rf, np.float64)), float(k), _p(np.ascontiguousarray(B, np.float64)))
    return complex(z.re, z.im)


def int_S_G(rf, k, tri):
    """singularity_subtraction_int_S_G (src/singularity_subtraction.f90:193-243)
    at one point: int_tri G(rf, r') dS'; tri (3,3)."""
    f = lib().orc_int_S_G
    f.argtypes = [C.c_void_p, C.c_double, C.c_void_p]
    f.restype = _Z
    z = f(_p(np.ascontiguousarray(rf, np.float64)), float(k), _p(np.ascontiguousarray(tri, np.float64)))
    return complex(z.re, z.im)


def int_V_GN(rf, k, B):
    """singularity_subtraction_int_V_GN at one point: int_B G(rf, r') N_j(r') dV', j = 1..4; B (4,3)."""
    out = np.zeros(4, np.complex128)
    lib().orc_int_V_GN(_p(np.ascontiguousarray(rf, np.float64)), C.c_double(k),
                       _p(np.ascontiguousarray(B, np.float64)), _p(out))
    return out


def int_S_GN(rf, k, tri):
    """singularity_subtraction_int_S_GN at one point: int_tri G(rf, r') N_l(r') dS', l = 1..3; tri (3,3)."""
    out = np.zeros(3, np.complex128)
    lib().orc_int_S_GN(_p(np.ascontiguousarray(rf, np.float64)), C.c_double(k),
                       _p(np.ascontiguousarray(tri, np.float64)), _p(out))
    return out


def gradshape(tc):
    """gradshape: dN (4,3), row n = gradient of the shape function of vertex n."""
    out = np.zeros((4, 3), np.float64)
    lib().orc_gradshape(_p(np.ascontiguousarray(tc, np.float64)), _p(out))
    return out
