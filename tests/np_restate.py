"""Independent numpy/scipy restatement of selected reference routines.

Used by the tests to cross-check the C oracle (``oracle/oracle.c``); both
restate jherrane/scadyn's Fortran from its source:

* ``build_G``            src/build_G.f90:1-66 (numpy FFT instead of FFTW)
* ``compute_Ax2``        src/gmres_module.f90:57-176 with sparse_T_matmul /
                         sparse_eps_matmul (src/sparse.f90:13-77), the pruned
                         FFT convolution written as a full zero-padded FFT
                         convolution (the pruning in src/possu.f90:140-289 is
                         exact), and matmul_Acorr_const (src/sparse_mat.f90:96-123)
* ``gmres``              src/gmres_module.f90:180-325
* ``calc_MN``            src/mie.f90:408-496 via scipy.special
"""
from __future__ import annotations

import numpy as np


def build_G(Nx, Ny, Nz, delta, min_coord, k):
    kk, ll, mm = np.meshgrid(np.arange(Nx), np.arange(Ny), np.arange(Nz), indexing="ij")
    nodes = np.stack([min_coord[0] + delta * kk, min_coord[1] + delta * ll, min_coord[2] + delta * mm], -1)
    R = np.sqrt(((nodes - nodes[0, 0, 0]) ** 2).sum(-1))
    with np.errstate(divide="ignore", invalid="ignore"):
        G = np.where(R > 0, np.exp(1j * k * R) / (4 * np.pi * R), 0)
    A = np.zeros((2 * Nx, 2 * Ny, 2 * Nz), np.complex128)
    ix = np.r_[np.arange(Nx), 2 * Nx - np.arange(1, Nx)]
    iy = np.r_[np.arange(Ny), 2 * Ny - np.arange(1, Ny)]
    iz = np.r_[np.arange(Nz), 2 * Nz - np.arange(1, Nz)]
    sx = np.r_[np.arange(Nx), np.arange(1, Nx)]
    sy = np.r_[np.arange(Ny), np.arange(1, Ny)]
    sz = np.r_[np.arange(Nz), np.arange(1, Nz)]
    A[np.ix_(ix, iy, iz)] = G[np.ix_(sx, sy, sz)]
    A[0, 0, 0] = 0
    return np.fft.fftn(A)          # (2Nx, 2Ny, 2Nz), x first


def _conv(src_xyz, Fg_xyz, Nx, Ny, Nz):
    A = np.zeros(Fg_xyz.shape, np.complex128)
    A[:Nx, :Ny, :Nz] = src_xyz
    A = np.fft.ifftn(Fg_xyz * np.fft.fftn(A))
    return A[:Nx, :Ny, :Nz]


def compute_Ax2(x, S, Sx, Sy, Sz, indS, Fg_zyx, sp_mat, sp_ind, k, Nx, Ny, Nz, merged=False):
    """x (3T,), S* (T,27), indS (T,27) 1-based, Fg as (2Nz,2Ny,2Nx) memory layout."""
    T = S.shape[0]
    Fg = np.transpose(Fg_zyx, (2, 1, 0))
    X = x.reshape(T, 3)
    node = indS - 1
    ngrid = Nx * Ny * Nz

    def scatter(P, xv):
        g = np.zeros(ngrid, np.complex128)
        np.add.at(g, node.ravel(), (P * xv[:, None]).ravel())
        return g.reshape(Nz, Ny, Nx).transpose(2, 1, 0)

    def gather(P, grid):
        flat = grid.transpose(2, 1, 0).ravel()
        return (P * flat[node]).sum(1)

    Y = [gather(S, _conv(scatter(S, X[:, d]), Fg, Nx, Ny, Nz)) for d in range(3)]
    P = (Sx, Sy, Sz)
    if merged:
        src = sum(scatter(P[d], X[:, d]) for d in range(3))
        r = _conv(src, Fg, Nx, Ny, Nz)
        Y2 = [gather(P[e], r) for e in range(3)]
    else:
        Y2 = [np.zeros(T, np.complex128) for _ in range(3)]
        for d in range(3):
            r = _conv(scatter(P[d], X[:, d]), Fg, Nx, Ny, Nz)
            for e in range(3):
                Y2[e] += gather(P[e], r)
    far = np.stack([Y2[d] - k ** 2 * Y[d] for d in range(3)], 1).ravel()
    return matmul_Acorr_const(sp_mat, sp_ind, x) + far


def matmul_Acorr_const(sp_mat, sp_ind, x):
    """sp_mat (B,3,3) holding Fortran (3,3,B): sp_mat[b, c, r] = val(r, c)."""
    V = sp_mat.astype(np.complex128).transpose(0, 2, 1)     # V[b, r, c]
    a = sp_ind[:, 0] - 1
    b = sp_ind[:, 1] - 1
    X = x.reshape(-1, 3)
    out = np.zeros_like(X)
    np.add.at(out, a, np.einsum("brc,bc->br", V, X[b]))
    off = a != b
    np.add.at(out, b[off], np.einsum("brc,br->bc", V[off], X[a[off]]))
    return out.ravel()


def gmres(matvec, rhs, tol, m, cycles):
    """Restarted GMRES with MGS, conditional re-orthogonalisation and complex
    Givens rotations, as src/gmres_module.f90:180-325."""
    n = rhs.shape[0]
    x = rhs.copy()
    b_norm = np.sqrt(np.vdot(rhs, rhs).real)
    error = np.inf
    iters = 0
    hist = []
    for _ in range(cycles):
        r = rhs - matvec(x)
        V = np.zeros((m + 1, n), np.complex128)
        H = np.zeros((m + 1, m), np.complex128)
        cs = np.zeros(m + 1, np.complex128)
        sn = np.zeros(m + 1, np.complex128)
        g = np.zeros(m + 1, np.complex128)
        V[0] = r / np.sqrt(np.vdot(r, r))
        g[0] = np.sqrt(np.vdot(r, r))
        kdim = m
        for i in range(m):
            w = matvec(V[i])
            iters += 1
            normav = np.sqrt(np.vdot(w, w)).real
            for kk in range(i + 1):
                H[kk, i] = np.vdot(V[kk], w)
                w = w - H[kk, i] * V[kk]
            H[i + 1, i] = np.sqrt(np.vdot(w, w))
            normav2 = H[i + 1, i].real
            V[i + 1] = w
            if normav + np.float32(0.001).astype(np.float64) * normav2 == normav:
                for j in range(i + 1):
                    hr = np.vdot(V[j], V[i + 1])
                    H[j, i] += hr
                    V[i + 1] = V[i + 1] - hr * V[j]
                H[i + 1, i] = np.sqrt(np.vdot(V[i + 1], V[i + 1]))
            if H[i + 1, i] != 0:
                V[i + 1] = V[i + 1] / H[i + 1, i]
            for kk in range(i):
                tmp = cs[kk] * H[kk, i] - sn[kk] * H[kk + 1, i]
                H[kk + 1, i] = sn[kk] * H[kk, i] + np.conj(cs[kk]) * H[kk + 1, i]
                H[kk, i] = tmp
            nu = np.sqrt(abs(H[i, i]) ** 2 + abs(H[i + 1, i]) ** 2)
            if nu != 0:
                cs[i] = np.conj(H[i, i] / nu)
                sn[i] = -H[i + 1, i] / nu
                H[i, i] = cs[i] * H[i, i] - sn[i] * H[i + 1, i]
                H[i + 1, i] = 0
                t1, t2 = g[i], g[i + 1]
                g[i] = cs[i] * t1 - sn[i] * t2
                g[i + 1] = sn[i] * t1 + np.conj(cs[i]) * t2
            error = abs(g[i + 1]) / b_norm
            hist.append(error)
            if error < tol:
                kdim = i + 1
                break
        y = np.linalg.solve(np.triu(H[:kdim, :kdim]), g[:kdim])
        x = x + V[:kdim].T @ y
        if error < tol:
            break
    return x, {"iters": iters, "relres": error, "history": np.array(hist)}


def calc_MN(Nmax, k, Po):
    """Regular VSWFs (Cartesian components) at Po, scadyn's normalisation."""
    from scipy.special import spherical_jn, lpmv, factorial
    r = np.linalg.norm(Po)
    th = np.arccos(Po[2] / r)
    ph = np.arctan2(Po[1], Po[0])
    kr = k * r
    nm = (Nmax + 1) ** 2 - 1
    MM = np.zeros((nm, 3), np.complex128)
    NN = np.zeros((nm, 3), np.complex128)
    H = np.array([[np.sin(th) * np.cos(ph), np.cos(th) * np.cos(ph), -np.sin(ph)],
                  [np.sin(th) * np.sin(ph), np.cos(th) * np.sin(ph), np.cos(ph)],
                  [np.cos(th), -np.sin(th), 0.0]])
    ind = 0
    ct = np.cos(th)
    for n in range(1, Nmax + 1):
        jn = spherical_jn(n, kr)
        jn1 = spherical_jn(n + 1, kr)
        alpha = jn
        beta = np.sqrt(n * (n + 1)) / kr * jn
        gamma = (n + 1) / kr * jn - jn1
        q = np.sqrt(n * (n + 1.0)) / ((2 * n + 1.0) * np.sin(th))
        for m in range(-n, n + 1):
            mm = abs(m)
            cc = np.sqrt((2 * n + 1.0) * factorial(n - mm) / factorial(n + mm) / (4 * np.pi))
            e = np.exp(1j * m * ph)
            Y = lpmv(mm, n, ct) * e
            Y1 = lpmv(mm, n + 1, ct) * e * ((n - mm + 1.0) / (n + 1.0))
            Y2 = 0 if mm == n else lpmv(mm, n - 1, ct) * e * ((n + mm) / n)
            B = np.array([0, Y1 - Y2, 1j * m * (2 * n + 1.0) / (n * (n + 1.0)) * Y]) * q
            Cv = np.array([0, B[2], -B[1]])
            P = np.array([Y, 0, 0])
            MM[ind] = H @ (cc * alpha * Cv)
            NN[ind] = H @ (cc * (beta * P + gamma * B))
            ind += 1
    return MM, NN
