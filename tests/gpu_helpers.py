"""Test helpers that connect oracle operator data to the device solver."""
from scadyn_b200 import api


def solver_from_oracle(op, device=0, fg_from_host=False, **choices):
    """Load an oracle operator into a device Solver so that both sides see the
    same operator data (constant or linear basis, op.order).  choices are the
    kernel choices of scd_grid_desc (fft_lengths, near_kernel, near_split)."""
    g = op.geom
    s = api.Solver(g.Nx, g.Ny, g.Nz, g.delta, g.min_coord, g.T, device, order=getattr(op, "order", 0), **choices)
    s.set_wavenumber(g.k)
    s.set_projectors(op.S, op.Sx, op.Sy, op.Sz, op.indS)
    s.build_G(op.Fg if fg_from_host else None)
    s.set_nearzone(op.sp_mat, op.sp_ind)
    return s
