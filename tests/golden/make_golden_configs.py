"""Generates the oracle fixtures of the benchmark configurations C1 and C2.

For the seeded C1 sphere (43k tets, grid 32^3 nodes) and the seeded C2
ellipsoid (150k tets, grid 64x54x40 nodes) -- the meshes ``bench.py`` builds --
the oracle sets up its own operator (``O.setup``: projectors, Green grid,
complex64 near zone as the reference stores it) and solves a few incident
VSWF columns with its restated ``gmres`` (GMRES(50), tol 1e-6).  The fixture
keeps what a GPU run is compared with:

* a fingerprint of the mesh (so a test notices a generator change),
* the unscaled T columns ``mat^H x`` (``T_matrix.f90:260``), the iteration
  counts and the final residuals of those columns,
* samples of the oracle operator: near-zone blocks with their (tet_T, tet_B)
  pairs, projector columns and Green samples.

Usage:  python tests/golden/make_golden_configs.py c1|c2 [nthreads]
(C1 takes a few minutes of CPU, C2 about an hour on 8 threads.)
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

# columns solved per configuration: first and last of the TE (M) and TM (N)
# halves, and a few in between
COLUMNS = {"c1": [0, 7, 30, 48, 60, 95], "c2": [0, 111, 224, 447]}


def mesh_fingerprint(mesh) -> str:
    h = hashlib.sha256()
    for a in (mesh.coord, mesh.etopol, mesh.param):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def near_sample_index(B: int, count: int = 4001) -> np.ndarray:
    return np.unique(np.linspace(0, B - 1, count).round().astype(np.int64))


def proj_sample_index(T: int, count: int = 257) -> np.ndarray:
    return np.unique(np.linspace(0, T - 1, count).round().astype(np.int64))


def main(name: str, nthreads: int = 0) -> str:
    import bench
    from oracle import oracle as O
    from scadyn_b200 import geometry

    cfg = bench.CONFIGS[name]
    mesh = bench.make_mesh(cfg)
    gs = geometry.cell_size_for_grid(mesh.coord, mesh.etopol, cfg["N"])
    k = cfg["ka"] / mesh.a
    t0 = time.time()
    op = O.setup(mesh, k, grid_size=gs, nthreads=nthreads)
    op.nthreads = nthreads
    t_setup = time.time() - t0
    g = op.geom
    print(f"{name}: T={g.T} grid {g.Nx}x{g.Ny}x{g.Nz} B={op.sp_ind.shape[0]} setup {t_setup:.0f}s", flush=True)
    mat = O.vswf2constant(mesh.coord, mesh.etopol, k, cfg["Nmax"])
    cols = COLUMNS[name]
    Tcols, iters, relres, secs = [], [], [], []
    for c in cols:
        t0 = time.time()
        x, info = op.gmres(mat[c], tol=cfg["tol"], m=cfg["m"], cycles=cfg["cycles"])
        secs.append(time.time() - t0)
        Tcols.append(mat.conj() @ x)
        iters.append(info["iters"])
        relres.append(info["relres"])
        print(f"  column {c}: {info['iters']} iterations, relres {info['relres']:.3e}, {secs[-1]:.0f}s", flush=True)
    B = op.sp_ind.shape[0]
    bi = near_sample_index(B)
    ti = proj_sample_index(g.T)
    out = os.path.join(HERE, f"{name}_columns.npz")
    np.savez_compressed(
        out,
        config=name, mesh_sha256=mesh_fingerprint(mesh), n_tet=g.T, grid=np.array([g.Nx, g.Ny, g.Nz]),
        grid_size=gs, k=k, Nmax=cfg["Nmax"], tol=cfg["tol"], m=cfg["m"], cycles=cfg["cycles"],
        columns=np.array(cols), T_cols=np.array(Tcols), iters=np.array(iters), relres=np.array(relres),
        solve_s=np.array(secs), setup_s=t_setup, nthreads=nthreads or os.cpu_count(),
        near_B=B, near_idx=bi, near_pairs=op.sp_ind[bi], near_blocks=op.sp_mat[bi],
        proj_idx=ti, S=op.S[ti], Sx=op.Sx[ti], indS=op.indS[ti],
        Fg_corner=op.Fg[:4, :4, :4].copy(),
    )
    return out


if __name__ == "__main__":
    print(main(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else 0))
