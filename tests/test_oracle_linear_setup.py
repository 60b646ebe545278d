"""Oracle restatement of the linear-basis set-up (mesh%order = 1).

pfft_projection_lin (src/projection.f90:170-338) and
compute_near_zone_interactions_lin (src/precorrection.f90:268-725, with
src/singularity_subtraction_N.f90) in oracle/oracle.c are checked three ways:

- the analytic parts of singularity_subtraction_int_V_GN / _int_S_GN against
  brute-force Gauss quadrature of N_j / (4 pi R) (k -> 0, where the numerical
  remainder G - 1/(4 pi R) vanishes), for points off, inside and on the element;
- the projectors against an independent numpy restatement, and their sum over
  the four nodes of a tet against the constant-basis projection with the same
  order-5 rules (the shape functions sum to one, their gradients to zero);
- the 12x12 blocks against a numpy restatement of the block assembly (aloks,
  integrate_NN/V_V/dV_V/V_dV/dV_dV, precorrect_lin) for self, same-box and
  neighbouring-box pairs.
"""
import numpy as np
import pytest

from oracle import oracle as O

# published order-5 rules in the reference's point order (Keast 24-point tetrahedron rule,
# 7-point degree-5 triangle rule; src/integration_points.f90)
_A = [(3.561913862225449e-01, 2.146028712591517e-01), (8.779781243961660e-01, 4.067395853461134e-02),
      (3.298632957317306e-02, 3.223378901422757e-01)]
_W4 = [6.653791709694644e-03, 1.679535175886776e-03, 9.226196923942397e-03]
_QT, _QW = [], []
for (_a, _b), _w in zip(_A, _W4):
    for _p in [(_a, _b, _b), (_b, _b, _b), (_b, _b, _a), (_b, _a, _b)]:
        _QT.append(_p)
        _QW.append(_w)
_c, _d, _e = 6.366100187501753e-02, 2.696723314583159e-01, 6.030056647916491e-01
for _p in [(_d, _c, _c), (_c, _d, _c), (_c, _c, _d), (_e, _c, _c), (_c, _e, _c), (_c, _c, _e),
           (_c, _d, _e), (_d, _e, _c), (_e, _c, _d), (_c, _e, _d), (_d, _c, _e), (_e, _d, _c)]:
    _QT.append(_p)
    _QW.append(8.035714285714281e-03)
QT, QW = np.array(_QT), np.array(_QW)
_t0, _a1, _b1, _a2, _b2 = 3.333333333333330e-01, 5.971587178977000e-02, 4.701420641051150e-01, 7.974269853530870e-01, 1.012865073234560e-01
QR = np.array([(_t0, _t0), (_a1, _b1), (_b1, _b1), (_b1, _a1), (_a2, _b2), (_b2, _b2), (_b2, _a2)])
QRW = np.array([1.125e-01] + [6.619707639425300e-02] * 3 + [6.296959027241350e-02] * 3)
FACE = [(1, 2, 3), (0, 3, 2), (0, 1, 3), (0, 2, 1)]          # tetra_face, src/common.f90:296-322
SHP_T = np.stack([1 - QT.sum(1), QT[:, 0], QT[:, 1], QT[:, 2]], 1)   # (24, 4)
SHP_R = np.stack([1 - QR.sum(1), QR[:, 0], QR[:, 1]], 1)             # (7, 3)


def green(r, p, k):
    R = np.linalg.norm(r - p, axis=-1)
    return np.exp(1j * k * R) / (4 * np.pi * R)


def vol6(tc):
    return abs(np.linalg.det(np.stack([tc[1] - tc[0], tc[2] - tc[0], tc[3] - tc[0]])))


def gradshape(tc):
    J = np.stack([tc[1] - tc[0], tc[2] - tc[0], tc[3] - tc[0]], axis=1)
    Ji = np.linalg.inv(J)
    dN = np.zeros((4, 3))
    dN[1:] = Ji
    dN[0] = -Ji.sum(0)
    return dN


def tri_points(tri):
    a, b = tri[1] - tri[0], tri[2] - tri[0]
    n = np.cross(a, b)
    n /= np.linalg.norm(n)
    ww1 = np.sqrt((a @ a) * (b @ b) - (a @ b) ** 2)
    return tri[0] + np.outer(QR[:, 0], a) + np.outer(QR[:, 1], b), QRW * ww1, n


# ------------------------------------------------------------ brute force
def _gl(n):
    x, w = np.polynomial.legendre.leggauss(n)
    return (x + 1) / 2, w / 2


def _bf_tet(rf, k, tc, n=28):
    """int_tet G N_j dV with a collapsed Gauss rule whose singular corner is vertex 1 of tc."""
    u, wu = _gl(n)
    U, V, W = np.meshgrid(u, u, u, indexing="ij")
    WU, WV, WW = np.meshgrid(wu, wu, wu, indexing="ij")
    xi, eta, zeta = U, V * (1 - U), W * (1 - U) * (1 - V)
    J = (1 - U) ** 2 * (1 - V)
    lam = np.stack([1 - xi - eta - zeta, xi, eta, zeta])
    P = np.einsum("vijk,vd->ijkd", lam, tc)
    return P, WU * WV * WW * J * vol6(tc)


def bf_V(rf, k, B):
    """int_B G(rf, r') N_j(r') dV' split into four tets with rf at a corner (exact for rf inside)."""
    out = np.zeros(4, complex)
    Binv = np.linalg.inv(np.stack([B[1] - B[0], B[2] - B[0], B[3] - B[0]], axis=1))
    for f in range(4):
        sub = np.array([B[FACE[f][0]], rf, B[FACE[f][1]], B[FACE[f][2]]])
        if vol6(sub) < 1e-14:
            continue
        # the cone from rf over face f counts negatively when rf lies beyond the face
        e1, e2 = B[FACE[f][1]] - B[FACE[f][0]], B[FACE[f][2]] - B[FACE[f][0]]
        sgn = np.sign(np.cross(e1, e2) @ (rf - B[FACE[f][0]])) * np.sign(np.cross(e1, e2) @ (B[f] - B[FACE[f][0]]))
        P, w = _bf_tet(rf, k, sub)
        w = w * sgn
        lam = np.einsum("de,ijke->ijkd", Binv, P - B[0])
        N = np.stack([1 - lam.sum(-1), lam[..., 0], lam[..., 1], lam[..., 2]])
        G = green(rf, P, k)
        out += (G[None] * N * w[None]).sum(axis=(1, 2, 3))
    return out


def bf_S(rf, k, tri, n=48):
    """int_tri G(rf, r') N_l(r') dS' split into three triangles with rf's projection at a corner."""
    a, b = tri[1] - tri[0], tri[2] - tri[0]
    nrm = np.cross(a, b)
    nrm /= np.linalg.norm(nrm)
    p = rf - ((rf - tri[0]) @ nrm) * nrm
    M = np.linalg.pinv(np.stack([a, b], axis=1))
    u, wu = _gl(n)
    U, V = np.meshgrid(u, u, indexing="ij")
    WU, WV = np.meshgrid(wu, wu, indexing="ij")
    out = np.zeros(3, complex)
    for e in range(3):
        q1, q2 = tri[(e + 1) % 3], tri[(e + 2) % 3]
        area2 = np.linalg.norm(np.cross(q1 - p, q2 - p))
        # signed: the projection may lie outside the triangle
        sgn = np.sign(np.cross(q1 - p, q2 - p) @ nrm)
        if area2 < 1e-14:
            continue
        xi, eta = U, V * (1 - U)
        # collapsed corner (U = 1) at p, where 1/R is singular
        P = q1 + np.multiply.outer(xi, p - q1) + np.multiply.outer(eta, q2 - q1)
        w = WU * WV * (1 - U) * area2 * sgn
        st = np.einsum("de,ije->ijd", M, P - tri[0])
        N = np.stack([1 - st[..., 0] - st[..., 1], st[..., 0], st[..., 1]])
        out += (green(rf, P, k)[None] * N * w[None]).sum(axis=(1, 2))
    return out


B0 = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.2, 1.0, 0.1], [0.1, 0.2, 1.0]])


@pytest.mark.parametrize("rf", [[1.5, 1.2, 1.1], [0.6, 0.6, 0.6], [0.5, 0.5, -0.3], [0.325, 0.33, 0.275],
                                [0.2, 0.25, 0.3]])
def test_int_V_GN_analytic_part(rf):
    rf = np.array(rf)
    got = O.int_V_GN(rf, 1e-7, B0)
    want = bf_V(rf, 1e-7, B0)
    assert np.abs(got.real - want.real).max() / np.abs(want.real).max() < 1e-8


@pytest.mark.parametrize("rf", [[1.5, 1.2, 1.1], [0.6, 0.6, 0.6], [0.2, 0.3, 0.9], [0.1, 0.1, 0.1]])
def test_int_S_GN_analytic_part(rf):
    rf = np.array(rf)
    tri = B0[list(FACE[0])]
    got = O.int_S_GN(rf, 1e-7, tri)
    want = bf_S(rf, 1e-7, tri)
    assert np.abs(got.real - want.real).max() / np.abs(want.real).max() < 1e-8


def test_int_S_GN_in_plane():
    """rf in the triangle's plane (w0 = 0, the |w0| <= 1e-10 branch), inside it."""
    tri = B0[list(FACE[0])]
    rf = tri.mean(0) + 0.1 * (tri[1] - tri.mean(0))
    got = O.int_S_GN(rf, 1e-7, tri)
    want = bf_S(rf, 1e-7, tri, n=64)
    assert np.abs(got.real - want.real).max() / np.abs(want.real).max() < 1e-8


def test_int_GN_full_green_quadrature_level():
    """With k > 0 the remainder is integrated by the order-5 rules: agreement at quadrature level."""
    for rf in ([1.5, 1.2, 1.1], [0.6, 0.6, 0.6]):
        rf = np.array(rf)
        got, want = O.int_V_GN(rf, 1.0, B0), bf_V(rf, 1.0, B0)
        assert np.abs(got - want).max() / np.abs(want).max() < 1e-4


def test_gradshape():
    dN = O.gradshape(B0)
    assert np.allclose(dN, gradshape(B0), rtol=0, atol=1e-13)
    # gradients of barycentric coordinates: dN_n . (v_m - v_0) = delta_nm - delta_n0
    E = B0 - B0[0]
    assert np.allclose(dN @ E.T, np.eye(4) - np.eye(4)[:, :1], atol=1e-13)


# ------------------------------------------------------------- projectors
@pytest.fixture(scope="module")
def lin_setup():
    from scadyn_b200 import meshgen
    m = meshgen.sphere(3, seed=1, eps=2.25 + 0.01j)
    k = 1.0 / m.a
    g = O.Geometry(m.coord, m.etopol, m.param, k=k, grid_size=1.8)
    P = g.projectors_lin()
    sp, ind = g.nearzone_lin(*P[:4], fp64=True)
    return m, k, g, P, sp, ind


def _node(g, i):
    i = i - 1
    return g.min_coord + g.delta * np.array([i % g.Nx, (i // g.Nx) % g.Ny, i // (g.Nx * g.Ny)])


def _box(g, tc):
    M = np.floor((tc.mean(0) - g.min_coord) / g.box_delta).astype(int)
    cx, cy, _ = g.cube_dims
    return M[0] + cx * M[1] + cx * cy * M[2] + 1


def _samples():
    v = [-1, -0.5, 0, 0.5, 1]
    P = [(v[ix], v[iy], -1) for iy in range(4, -1, -1) for ix in range(5)]
    P += [(v[ix], v[iy], 1) for iy in range(5) for ix in range(5)]
    P += [(v[ix], -1, v[iz]) for iz in range(1, 4) for ix in range(5)]
    P += [(v[ix], 1, v[iz]) for iz in range(3, 0, -1) for ix in range(5)]
    P += [(-1, v[iy], v[iz]) for iz in range(1, 4) for iy in range(3, 0, -1)]
    P += [(1, v[iy], v[iz]) for iz in range(1, 4) for iy in range(1, 4)]
    return np.array(P, float)


def test_projectors_lin_restated(lin_setup):
    m, k, g, (S, Sx, Sy, Sz, indS), _, _ = lin_setup
    T = m.n_tet
    Ps = 2 * g.box_delta * _samples()
    tc0 = m.coord[m.etopol[0] - 1]
    bn = g.etopol_box[_box(g, tc0) - 1]
    cpc = _node(g, bn[0]) + g.box_delta / 2
    W = np.array([[green(Ps[q] + cpc, _node(g, u), k) for u in bn] for q in range(98)])
    WW = O.pinv(np.ascontiguousarray(W.T)).T           # (27, 98)
    for t in (0, 5, 77, 300, T - 1):
        tc = m.coord[m.etopol[t] - 1]
        vol = vol6(tc) / 6
        bt = g.etopol_box[_box(g, tc) - 1]
        r = Ps + _node(g, bt[0]) + g.box_delta / 2
        Pb, wb = SHP_T @ tc, QW * 6 * vol
        G = green(r[:, None, :], Pb[None], k)           # (98, 24)
        Q = (G * wb) @ SHP_T                              # (98, 4)
        Q2 = np.zeros((3, 98, 4), complex)
        for f in range(4):
            Pt, wt, n = tri_points(tc[list(FACE[f])])
            q2 = (green(r[:, None, :], Pt[None], k) * wt) @ SHP_R
            for l in range(3):
                Q2[:, :, FACE[f][l]] += n[:, None] * q2[None, :, l]
        dN = gradshape(tc)
        want = [WW @ Q / np.sqrt(vol)]
        want += [(WW @ Q2[d] - WW @ (Q.sum(1)[:, None] * dN[:, d][None])) / np.sqrt(vol) for d in range(3)]
        for got, w in zip((S, Sx, Sy, Sz), want):
            blk = got[4 * t:4 * t + 4].T
            assert np.abs(blk - w).max() / np.abs(w).max() < 1e-7
        assert (indS[4 * t:4 * t + 4] == bt[None]).all()
        # the four columns sum to the constant-basis projector with the same order-5 rules
        const5 = WW @ (G @ wb) / np.sqrt(vol)
        assert np.abs(S[4 * t:4 * t + 4].sum(0) - const5).max() / np.abs(const5).max() < 1e-9


# ----------------------------------------------------------------- blocks
def block_lin(m, k, g, P, tT, tB):
    """One 12x12 block V(4c+n, 4c'+n') for 0-based tets tT <= tB, restated with numpy."""
    S, Sx, Sy, Sz, _ = P
    Tc, Bc = m.coord[m.etopol[tT] - 1], m.coord[m.etopol[tB] - 1]
    volT, volB = vol6(Tc) / 6, vol6(Bc) / 6
    dNT, dNB = gradshape(Tc), gradshape(Bc)
    # compute_pG of the two boxes
    nt = g.etopol_box[_box(g, Tc) - 1]
    nb = g.etopol_box[_box(g, Bc) - 1]
    G = np.zeros((27, 27), complex)
    for a in range(27):
        for b in range(27):
            if nt[a] != nb[b]:
                G[a, b] = green(_node(g, nt[a]), _node(g, nb[b]), k)
    # precorrect_lin
    corr, corr2 = np.zeros((12, 12), complex), np.zeros((12, 12), complex)
    PT = [A[4 * tT:4 * tT + 4] for A in (S, Sx, Sy, Sz)]
    PB = [A[4 * tB:4 * tB + 4] for A in (S, Sx, Sy, Sz)]
    for i1 in range(4):
        gv = [G @ PB[s][i1] for s in range(4)]
        for i2 in range(4):
            a0 = gv[0] @ PT[0][i2]
            for c in range(3):
                corr[4 * c + i2, 4 * c + i1] = a0
            for r in range(3):
                for c in range(3):
                    corr2[4 * r + i2, 4 * c + i1] = gv[1 + c] @ PT[1 + r][i2]
    sv = np.sqrt(volT * volB)
    corr, corr2 = corr * sv, corr2 * sv
    Pt, wt = SHP_T @ Tc, QW * 6 * volT
    alok = np.zeros((12, 12), complex)
    if tT == tB:
        NN = np.einsum("i,ia,ib->ab", wt, SHP_T, SHP_T)
        for c in range(3):
            alok[4 * c:4 * c + 4, 4 * c:4 * c + 4] = NN
    IV = np.array([O.int_V_GN(p, k, Bc) for p in Pt])                 # (24, 4)
    GNN = np.einsum("i,ia,ib->ab", wt, SHP_T, IV)
    Bf = [tri_points(Bc[list(FACE[f])]) for f in range(4)]

    def J(rf):
        out = np.zeros(12, complex)
        for f in range(4):
            iS = O.int_S_GN(rf, k, Bc[list(FACE[f])])
            for l in range(3):
                for c in range(3):
                    out[4 * c + FACE[f][l]] += iS[l] * Bf[f][2][c]
        return out

    II4 = np.zeros(12, complex)
    alok2 = np.zeros((12, 12), complex)
    for ft in range(4):
        Ptt, wtt, Tn = tri_points(Tc[list(FACE[ft])])
        intN = np.zeros(4, complex)
        II = np.zeros((3, 4, 4), complex)
        for i in range(7):
            Is = O.int_V_GN(Ptt[i], k, Bc).sum()
            Ji = J(Ptt[i])
            for l in range(3):
                intN[FACE[ft][l]] += Is * SHP_R[i, l] * wtt[i]
                for c in range(3):
                    II[c, FACE[ft][l], :] += Ji[4 * c:4 * c + 4] * SHP_R[i, l] * wtt[i]
        for r in range(3):
            II4[4 * r:4 * r + 4] += intN * Tn[r]
            for c in range(3):
                alok2[4 * r:4 * r + 4, 4 * c:4 * c + 4] += II[c] * Tn[r]
    II5 = sum(J(Pt[i]) * wt[i] for i in range(24))
    ddT, ddB = dNT.T.reshape(12), dNB.T.reshape(12)                    # dd(4c + n) = dN_n[c]
    alok1 = np.kron(np.eye(3), GNN)
    alok3 = np.outer(ddT, ddB) * GNN.sum()
    alok4 = np.outer(II4, ddB)
    alok5 = np.outer(ddT, II5)
    ep = m.param[tT]
    return (alok / (ep - 1) + (-k * k * (alok1 - corr) + (alok2 + alok3 - alok4 - alok5) - corr2)) / np.sqrt(volB * volT)


def test_nearzone_lin_restated(lin_setup):
    m, k, g, P, sp, ind = lin_setup
    assert np.isfinite(sp).all()
    pairs = {}
    for b, (t1, t2) in enumerate(ind):
        pairs[(t1 - 1, t2 - 1)] = b
    # a self pair, a same-box pair and a pair in neighbouring boxes
    tets = np.unique(ind[:, 0])
    chosen = [(tets[3] - 1, tets[3] - 1)]
    same = [(a - 1, b - 1) for a, b in ind if a != b and _box(g, m.coord[m.etopol[a - 1] - 1]) == _box(g, m.coord[m.etopol[b - 1] - 1])]
    diff = [(a - 1, b - 1) for a, b in ind if _box(g, m.coord[m.etopol[a - 1] - 1]) != _box(g, m.coord[m.etopol[b - 1] - 1])]
    chosen += [same[len(same) // 2], diff[len(diff) // 3]]
    for tT, tB in chosen:
        want = block_lin(m, k, g, P, tT, tB)
        got = sp[pairs[(tT, tB)]].T                                    # memory (12,12,B) -> V[row, col]
        assert np.abs(got - want).max() / np.abs(want).max() < 1e-9, (tT, tB)


def test_nearzone_lin_pairs_match_constant(lin_setup):
    """The linear assembly visits the constant-basis tet pairs, in the same order."""
    m, k, g, P, sp, ind = lin_setup
    Sc = g.projectors()
    _, indc = g.nearzone(*Sc[:4])
    assert (ind == indc).all()


def test_linear_operator_solves(lin_setup):
    """GMRES on the assembled linear-basis operator converges (order-1 compute_Ax2)."""
    m, k, g, P, sp, ind = lin_setup
    op = O.Operator(g, *P, g.build_G(), sp.astype(np.complex64), ind, order=1, nthreads=0)
    rng = np.random.default_rng(5)
    n = 12 * m.n_tet
    rhs = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    x, info = op.gmres(rhs, tol=1e-6, m=50, cycles=6)
    assert info["converged"], info["relres"]
    r = op.compute_Ax2(x) - rhs
    assert np.linalg.norm(r) / np.linalg.norm(rhs) < 1e-5


def test_self_blocks_nearly_symmetric(lin_setup):
    """The operator is complex-symmetric; a self block V(T, T) applied one-sided must be
    symmetric up to its quadrature (the singular double integrals are not evaluated
    symmetrically, as for the constant basis).  A sign or transposition slip between
    integrate_dV_V_GNN and integrate_V_dV_GNN, or in the (component, node) order of
    integrate_dV_dV_GNN, would make it O(1) asymmetric."""
    m, k, g, P, sp, ind = lin_setup
    V = np.transpose(sp, (0, 2, 1))                  # V[b, row, col]
    own = ind[:, 0] == ind[:, 1]
    asym = np.array([np.linalg.norm(v - v.T) / np.linalg.norm(v) for v in V[own]])
    assert own.sum() == m.n_tet
    assert asym.max() < 5e-3, asym.max()


def test_linear_T_matrix_matches_mie_series(small_sphere):
    """Physics pin of the whole linear-basis operator (projectors, 12x12 near zone,
    order-1 compute_Ax2): a T-matrix solved in the linear basis agrees with the Mie
    coefficients at discretisation level, as the constant basis does.  The reference
    defines no linear-basis T-matrix, so the right-hand sides here are the VSWFs
    projected on the basis functions N_n / sqrt(vol) (24-point rule), the counterpart
    of vswf2constant's centroid values times sqrt(vol)."""
    m = small_sphere
    k, Nmax = 1.0 / m.a, 2
    nm = (Nmax + 1) ** 2 - 1
    op = O.setup_lin(m, k, grid_size=1.8, nthreads=0)
    op.nthreads = 0
    T = m.n_tet
    mat = np.zeros((2 * nm, 12 * T), complex)
    for t in range(T):
        tc = m.coord[m.etopol[t] - 1]
        vol = vol6(tc) / 6
        Pq, w = SHP_T @ tc, QW * 6 * vol
        for i in range(24):
            MM, NN = O.calc_MN(Nmax, k, Pq[i])
            f = SHP_T[i] * w[i] / np.sqrt(vol)             # per node
            for c in range(3):
                mat[:nm, 12 * t + 4 * c:12 * t + 4 * c + 4] += np.outer(MM[:, c], f)
                mat[nm:, 12 * t + 4 * c:12 * t + 4 * c + 4] += np.outer(NN[:, c], f)
    X = np.zeros_like(mat)
    for c in range(2 * nm):
        X[c], info = op.gmres(mat[c], tol=1e-6, m=50, cycles=6)
        assert info["converged"]
    Tl = (np.conj(mat) @ X.T) * (1j * k ** 3)
    a_n, b_n = O.mie_T(Nmax, k * m.a, np.sqrt(2.25 + 0.01j))
    for j in range(nm):
        n = int(np.floor(np.sqrt(j + 1)))
        assert abs(Tl[j, j] - a_n[n - 1]) < 0.08 * abs(a_n[n - 1])
        assert abs(Tl[nm + j, nm + j] - b_n[n - 1]) < 0.08 * abs(b_n[n - 1])
    assert np.abs(Tl[:nm, :nm] - np.diag(np.diag(Tl[:nm, :nm]))).max() < 0.05 * abs(a_n[0])
