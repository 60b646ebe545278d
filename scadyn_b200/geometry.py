"""Host helpers around build_grid (src/geometry.f90:60-125)."""
from __future__ import annotations

import numpy as np

F13 = float(np.float32(1.0) / np.float32(3.0))   # Fortran default-real 1.0/3.0


def tet_volume_sum(coord, etopol):
    P = coord[etopol - 1]
    p41 = P[:, 3] - P[:, 0]
    cr = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    return float(np.abs(np.einsum("ti,ti->t", p41, cr)).sum() / 6.0)


def cell_size_for_grid(coord, etopol, N_target: int, M_ex: int = 2) -> float:
    """The ``cell_size`` (mesh%grid_size) that makes build_grid give
    N_target nodes on the longest axis.  build_grid sets
    delta = cell_size/M_ex*(V/T)^(1/3), N = ceil(L/delta) + 1, then rounds N
    up to even (+1 if odd, +2 if even); N_target must be even."""
    if N_target % 2:
        raise ValueError("N_target must be even for M_ex = 2")
    L = float((coord.max(0) - coord.min(0)).max())
    T = etopol.shape[0]
    vol = tet_volume_sum(coord, etopol)
    delta = L / (N_target - 2.5)
    return delta * M_ex / (vol / T) ** F13
