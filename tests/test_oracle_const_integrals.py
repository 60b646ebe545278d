"""The constant-basis near-zone integrals of the oracle, checked independently.

The product path's near zone (compute_near_zone_interactions_const,
src/precorrection.f90:131-264) rests on three singular integrals of
src/singularity_subtraction.f90; each is checked here against brute-force
Gauss quadrature with the singular point at a collapsed corner:

- analytical_integration (:15-108): int_tri 1/R dS and int_tri R dS for
  points off the plane, in the plane inside and outside the triangle;
- singularity_subtraction_int_V_G (:112-189): int_tet G dV with k -> 0
  (where the numerically integrated remainder G - 1/(4 pi R) vanishes) for
  points outside, inside and on a face of the tet, and with k = 1 at
  quadrature level;
- singularity_subtraction_int_S_G (:193-243): int_tri G dS likewise.

Then one 3x3 block of each kind -- self, same box, neighbouring box -- is
restated in numpy from the reference's formula: the grid-mediated
corrections of precorrect_const (:50-82) from compute_pG (:21-46) and the
projectors, integrate_V_V_G (:729-760) as the order-5 tet rule over
int_V_G, integrate_dV_dV_G (:764-806) as the 16 face pairs with n_T n_B^T
and the order-5 triangle rule over int_S_G, the self term 1/(eps-1) I and
the 1/sqrt(vol_T vol_B) scaling; it must equal the oracle's FP64 block to
1e-10.  A sign or transposition slip in any face term would show here, well
below the discretisation-level Mie bound.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_linear_setup import B0, FACE, QT, QW, _gl, bf_S, bf_V, tri_points, vol6


def bf_tri(fun, rf, tri, n=64):
    """int_tri fun(|rf - r'|) dS' split into three triangles with rf's
    projection at a collapsed corner (signed, so it may lie outside)."""
    a, b = tri[1] - tri[0], tri[2] - tri[0]
    nrm = np.cross(a, b)
    nrm /= np.linalg.norm(nrm)
    p = rf - ((rf - tri[0]) @ nrm) * nrm
    u, wu = _gl(n)
    U, V = np.meshgrid(u, u, indexing="ij")
    WU, WV = np.meshgrid(wu, wu, indexing="ij")
    out = 0.0
    for e in range(3):
        q1, q2 = tri[(e + 1) % 3], tri[(e + 2) % 3]
        area2 = np.linalg.norm(np.cross(q1 - p, q2 - p))
        if area2 < 1e-14:
            continue
        sgn = np.sign(np.cross(q1 - p, q2 - p) @ nrm)
        xi, eta = U, V * (1 - U)
        P = q1 + np.multiply.outer(xi, p - q1) + np.multiply.outer(eta, q2 - q1)
        w = WU * WV * (1 - U) * area2 * sgn
        out += (fun(np.linalg.norm(rf - P, axis=-1)) * w).sum()
    return out


TRI = B0[list(FACE[0])]


@pytest.mark.parametrize("r", [[0.4, 0.5, 0.9], [1.2, -0.3, 0.4], "inside", "outside"])
def test_analytical_integration(r):
    c = TRI.mean(0)
    if r == "inside":
        r = c + 0.2 * (TRI[0] - c)
    elif r == "outside":
        r = c + 2.5 * (TRI[1] - c)
    r = np.array(r, float)
    got = O.analytical_integration(TRI, r)
    want = [bf_tri(lambda R: 1 / R, r, TRI), bf_tri(lambda R: R, r, TRI)]
    assert abs(got[0] - want[0]) < 1e-9 * abs(want[0])
    assert abs(got[1] - want[1]) < 1e-9 * abs(want[1])


@pytest.mark.parametrize("rf", [[1.5, 1.2, 1.1], [0.3, 0.32, 0.28], [0.2, 0.25, 0.3], "face"])
def test_int_V_G(rf):
    if rf == "face":
        rf = B0[list(FACE[2])].mean(0)
    rf = np.array(rf, float)
    k0 = 1e-7
    got, want = O.int_V_G(rf, k0, B0), bf_V(rf, k0, B0).sum()
    assert abs(got.real - want.real) < 1e-8 * abs(want.real)
    got, want = O.int_V_G(rf, 1.0, B0), bf_V(rf, 1.0, B0).sum()
    assert abs(got - want) < 1e-4 * abs(want)


@pytest.mark.parametrize("rf", [[1.5, 1.2, 1.1], [0.2, 0.3, 0.9], [0.1, 0.1, 0.1], "in-plane"])
def test_int_S_G(rf):
    if rf == "in-plane":
        c = TRI.mean(0)
        rf = c + 0.1 * (TRI[1] - c)
    rf = np.array(rf, float)
    k0 = 1e-7
    got, want = O.int_S_G(rf, k0, TRI), bf_S(rf, k0, TRI, n=64).sum()
    assert abs(got.real - want.real) < 1e-8 * abs(want.real)
    got, want = O.int_S_G(rf, 1.0, TRI), bf_S(rf, 1.0, TRI, n=64).sum()
    assert abs(got - want) < 1e-4 * abs(want)


# ------------------------------------------------------------ block restatement
def _node(g, i):
    i = i - 1
    return g.min_coord + g.delta * np.array([i % g.Nx, (i // g.Nx) % g.Ny, i // (g.Nx * g.Ny)])


def block_np(op, mesh, tT, tB):
    """compute_near_zone_interactions_const's block for tets tT <= tB (1-based)."""
    g, k = op.geom, op.geom.k
    cube = lambda t: int(np.nonzero((g.tetras == t).any(axis=1))[0][0])
    tb, bb = g.etopol_box[cube(tT)], g.etopol_box[cube(tB)]
    rT = np.array([_node(g, i) for i in tb])
    rB = np.array([_node(g, i) for i in bb])
    R = np.linalg.norm(rT[:, None] - rB[None], axis=-1)
    same = tb[:, None] == bb[None]
    G = np.where(same, 0, np.exp(1j * k * R) / (4 * np.pi * np.where(same, 1, R)))     # compute_pG
    Tc, Bc = mesh.coord[mesh.etopol[tT - 1] - 1], mesh.coord[mesh.etopol[tB - 1] - 1]
    vT, vB = vol6(Tc) / 6, vol6(Bc) / 6
    sv = np.sqrt(vT * vB)
    PT = [op.Sx[tT - 1], op.Sy[tT - 1], op.Sz[tT - 1]]
    PB = [op.Sx[tB - 1], op.Sy[tB - 1], op.Sz[tB - 1]]
    acorr = (op.S[tT - 1] @ (G @ op.S[tB - 1])) * sv                                      # precorrect_const
    corr2 = np.array([[PT[r] @ (G @ PB[c]) for c in range(3)] for r in range(3)]) * sv
    lam = np.stack([1 - QT.sum(1), QT[:, 0], QT[:, 1], QT[:, 2]], 1)
    Pt, wt = lam @ Tc, QW * 6 * vT                                                        # linmap_tet
    intVV = sum(w * O.int_V_G(p, k, Bc) for p, w in zip(Pt, wt))                         # integrate_V_V_G
    alok2 = np.zeros((3, 3), complex)                                                     # integrate_dV_dV_G
    for ft in range(4):
        Pp, wp, nT = tri_points(Tc[list(FACE[ft])])
        for fb in range(4):
            Btri = Bc[list(FACE[fb])]
            _, _, nB = tri_points(Btri)
            s = sum(w * O.int_S_G(p, k, Btri) for p, w in zip(Pp, wp))
            alok2 += np.outer(nT, nB) * s
    eps = mesh.param[tT - 1]
    blk = np.eye(3) * (1 / (eps - 1) if tT == tB else 0) + (-k * k * (intVV - acorr) * np.eye(3)
                                                           + (alok2 - corr2)) / np.sqrt(vT * vB)
    return blk


def test_block_restatement_matches_oracle(small_sphere, small_op):
    m, op = small_sphere, small_op
    sp, ind = op.geom.nearzone(op.S, op.Sx, op.Sy, op.Sz, fp64=True)
    g = op.geom
    cube = {}
    for c in range(g.tetras.shape[0]):
        for t in g.tetras[c]:
            if t:
                cube[int(t)] = c
    pick = {}
    for b, (tT, tB) in enumerate(ind):
        kind = "self" if tT == tB else ("same box" if cube[int(tT)] == cube[int(tB)] else "neighbour")
        pick.setdefault(kind, b)
        if len(pick) == 3:
            break
    assert set(pick) == {"self", "same box", "neighbour"}
    for kind, b in pick.items():
        tT, tB = (int(v) for v in ind[b])
        want = sp[b].T                    # memory (3,3,B): sp[b][c][r] = block(r, c)
        got = block_np(op, m, tT, tB)
        err = np.abs(got - want).max() / np.abs(want).max()
        assert err < 1e-10, (kind, err)
