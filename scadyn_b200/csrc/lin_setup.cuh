// Linear basis (mesh%order = 1) set-up integrals, host and device.
//
// One 12x12 near-zone block of compute_near_zone_interactions_lin
// (src/precorrection.f90:268-371) between test tet T and basis tet B:
//   V = (alok/(eps_T - 1) + (-k^2 (alok1 - corr) + (alok2 + alok3 - alok4 - alok5) - corr2)) / sqrt(vol_T vol_B)
// with rows and columns 4c + n (component c, node n):
//   alok   = diag_c  int_T N_a N_b                     (integrate_NN, self pairs only, :375-405)
//   alok1  = diag_c  GNN(a, b),  GNN(a, b) = int_T N_a int_B G N_b   (integrate_V_V_GNN, :409-445)
//   alok2  = sum over faces of T and B of n_T,r n_B,c int int N_a G N_b   (integrate_dV_dV_GNN, :528-617)
//   alok3  = dN_T,a[r] dN_B,b[c] sum(GNN)               (aloks, :689-717)
//   alok4  = II4(4r + a) dN_B,b[c], II4 = sum over faces of T of n_r int N_a int_B G   (integrate_dV_V_GNN, :449-524)
//   alok5  = dN_T,a[r] II5(4c + b), II5 = int_T sum over faces of B of n_c int N_b G  (integrate_V_dV_GNN, :621-685)
//   corr, corr2 = the grid-mediated part through the projectors (precorrect_lin, :86-127)
// The inner integrals are singularity_subtraction_int_V_GN / _int_S_GN
// (src/singularity_subtraction_N.f90:140-294): 1/R is subtracted, integrated
// analytically (analytical_integration_N, :15-136) and the remainder is
// integrated with the order-5 rules.
//
// The work of a block is split in three phases so that a warp can share it:
//   lin_point  (260 items): the inner integrals at the 52 test points (24 in
//              T, 7 on each face of T), 16 values per point in a scratch row;
//   lin_small  (40 items):  GNN, II4, II5 from the scratch;
//   lin_entry  (144 items): one entry of the block.
// The quadrature tables come from an accessor Q with t5(i, c) (xi, eta, zeta,
// w) and r5(i, c) (xi, eta, w), so a host program runs the same arithmetic.
#pragma once
#include "geom.cuh"

// Gr (src/common.f90:271-279): exp(ikR) / (4 pi R)
SCD_HD cd green_hd(V3 rf, V3 rp, double k) {
    const double R = vdist(rf, rp);
    const double d = 4.0 * PI * R;
    double s, c;
#ifdef __CUDA_ARCH__
    sincos(k * R, &s, &c);
#else
    s = std::sin(k * R);
    c = std::cos(k * R);
#endif
    return cmk(c / d, s / d);
}

// gradshape (src/common.f90:454-492): gradients of the barycentric shape functions
SCD_HD void gradshape_hd(const V3 *t, V3 *dN) {
    const V3 e1 = vsub(t[1], t[0]), e2 = vsub(t[2], t[0]), e3 = vsub(t[3], t[0]);
    const V3 c1 = vcross(e2, e3), c2 = vcross(e3, e1), c3 = vcross(e1, e2);
    const double det = vdot(e1, c1);
    dN[1] = V3{c1.x / det, c1.y / det, c1.z / det};
    dN[2] = V3{c2.x / det, c2.y / det, c2.z / det};
    dN[3] = V3{c3.x / det, c3.y / det, c3.z / det};
    dN[0] = V3{-dN[1].x - dN[2].x - dN[3].x, -dN[1].y - dN[2].y - dN[3].y, -dN[1].z - dN[2].z - dN[3].z};
}

SCD_HD V3 bary_point(const V3 *t, double x, double y, double z) {
    const double w = 1 - x - y - z;
    return V3{t[0].x * w + t[1].x * x + t[2].x * y + t[3].x * z, t[0].y * w + t[1].y * x + t[2].y * y + t[3].y * z,
              t[0].z * w + t[1].z * x + t[2].z * y + t[3].z * z};
}

SCD_HD void face_tri(const V3 *t, int f, V3 *tri) {
    tri[0] = t[face_vertex(f, 0)];
    tri[1] = t[face_vertex(f, 1)];
    tri[2] = t[face_vertex(f, 2)];
}

// analytical_integration_N: out[nm-1][l] = int_tri N_l R^(2 nm - 3) dS,
// nm = 1..NP, N_l the shape function of triangle vertex l
template <int NP>
SCD_HD void analytic_tri_N(const V3 *tri, V3 n, V3 r, double (*out)[3]) {
    double Kl[NP + 1], Il[3] = {0, 0, 0}, tl[3], hhl[3], Inl[NP + 1][3];
    V3 mv[3];
    for (int q = 0; q <= NP; ++q) Kl[q] = 0.0;
    const double w0 = vdot(vsub(r, tri[0]), n);
    for (int m = 0; m <= NP; ++m) {
        const int nexp = 2 * m - 1;
        for (int l = 0; l < 3; ++l) {
            // edge l runs from vertex l1 to l2, opposite vertex l0 = l (1-based: (2,3), (3,1), (1,2))
            const int l1 = (l + 1) % 3, l2 = (l + 2) % 3, l0 = l;
            const V3 slv = vsub(tri[l2], tri[l1]);
            const double ns = sqrt(vdot(slv, slv));
            const V3 sl = V3{slv.x / ns, slv.y / ns, slv.z / ns};
            const V3 ml = vcross(sl, n);
            const V3 pl1mr = vsub(tri[l1], r);
            const double tl0 = vdot(pl1mr, ml);
            const double ll = sqrt(vdot(slv, slv));
            const double sml = vdot(pl1mr, sl), spl = sml + ll;
            const V3 rmp2 = vsub(r, tri[l2]);
            const double Rpl = sqrt(vdot(rmp2, rmp2)), Rml = sqrt(vdot(pl1mr, pl1mr));
            const double R0l = sqrt(tl0 * tl0 + w0 * w0);
            if (nexp == -1) {
                mv[l] = ml;
                tl[l] = tl0;
                hhl[l] = vdot(vsub(tri[l1], tri[l0]), ml);
                double Km3;
                if (fabs(w0) > 1.0e-10) {
                    const double Bl = atan((tl0 * spl) / (R0l * R0l + fabs(w0) * Rpl)) -
                                      atan((tl0 * sml) / (R0l * R0l + fabs(w0) * Rml));
                    Km3 = 1.0 / fabs(w0) * Bl;
                } else {
                    Km3 = 0.0;
                }
                Il[l] = fabs(Rml + sml) > 0.0 ? log((Rpl + spl) / (Rml + sml)) : 0.0;
                Kl[m] = Kl[m] + 1.0 / ((double)nexp + 2.0) * ((double)nexp * w0 * w0 * Km3 + tl0 * Il[l]);
            } else {
                Il[l] = 1.0 / ((double)nexp + 1.0) *
                        (spl * pow(Rpl, (double)nexp) - sml * pow(Rml, (double)nexp) + (double)nexp * R0l * R0l * Il[l]);
            }
        }
        if (nexp != -1)
            Kl[m] = 1.0 / ((double)nexp + 2.0) * ((double)nexp * w0 * w0 * Kl[m - 1] + (tl[0] * Il[0] + tl[1] * Il[1] + tl[2] * Il[2]));
        Inl[m][0] = Il[0];
        Inl[m][1] = Il[1];
        Inl[m][2] = Il[2];
    }
    for (int nm = 1; nm <= NP; ++nm) {
        const V3 v1 = V3{Inl[nm][0] * mv[0].x + Inl[nm][1] * mv[1].x + Inl[nm][2] * mv[2].x,
                         Inl[nm][0] * mv[0].y + Inl[nm][1] * mv[1].y + Inl[nm][2] * mv[2].y,
                         Inl[nm][0] * mv[0].z + Inl[nm][1] * mv[1].z + Inl[nm][2] * mv[2].z};
        for (int l = 0; l < 3; ++l)
            out[nm - 1][l] = 1.0 / hhl[l] * (tl[l] * Kl[nm - 1] - 1.0 / (2.0 * (double)nm - 1.0) * vdot(mv[l], v1));
    }
}

// singularity_subtraction_int_V_GN: out[j] = int_B G(rf, r') N_j(r') dV'
template <class Q>
SCD_HD void int_V_GN_hd(V3 rf, double k, const V3 *B, double volB, const V3 *dNB, cd *out) {
    double sumw = 0.0;
    for (int i = 0; i < 24; ++i) sumw += Q::t5(i, 3) * 6.0 * volB;
    const double cut = 1.0e-10 * pow(sumw, F13_D);
    cd acc[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int i = 0; i < 24; ++i) {
        const double x = Q::t5(i, 0), y = Q::t5(i, 1), z = Q::t5(i, 2);
        const V3 rp = bary_point(B, x, y, z);
        const double wb = Q::t5(i, 3) * 6.0 * volB;
        const double RR = vdist(rp, rf);
        cd II;
        if (RR < cut) {
            II = cmk(0.0, k / (4.0 * PI));
        } else {
            II = green_hd(rf, rp, k);
            II.x -= 1.0 / (4 * PI) / RR;
        }
        const double sh[4] = {1 - x - y - z, x, y, z};
        for (int j = 0; j < 4; ++j) {
            acc[j].x += II.x * sh[j] * wb;
            acc[j].y += II.y * sh[j] * wb;
        }
    }
    double r5[4] = {0, 0, 0, 0}, r6[4] = {0, 0, 0, 0};
    for (int f = 0; f < 4; ++f) {
        V3 tri[3];
        face_tri(B, f, tri);
        const V3 tn = tri_normal(tri);
        double ai[2][3];
        analytic_tri_N<2>(tri, tn, rf, ai);
        const double a1 = vdot(tn, vsub(tri[0], rf));
        for (int l = 0; l < 3; ++l) r6[face_vertex(f, l)] += ai[0][l] * a1 * 0.5;
        const double s2 = ai[1][0] + ai[1][1] + ai[1][2];
        for (int j = 0; j < 4; ++j) r5[j] += vdot(tn, dNB[j]) * s2 * 0.5;
    }
    for (int j = 0; j < 4; ++j) out[j] = cmk(acc[j].x + 1.0 / (4 * PI) * (-r5[j] + r6[j]), acc[j].y);
}

// singularity_subtraction_int_S_GN: out[l] = int_tri G(rf, r') N_l(r') dS'
template <class Q>
SCD_HD void int_S_GN_hd(V3 rf, const V3 *tri, V3 tn, double k, cd *out) {
    V3 a, b;
    const double ww1 = tri_ww1(tri, a, b);
    double sumw = 0.0;
    for (int i = 0; i < 7; ++i) sumw += Q::r5(i, 2) * ww1;
    const double cut = 1.0e-10 * sqrt(sumw);
    cd acc[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
    for (int i = 0; i < 7; ++i) {
        const double x = Q::r5(i, 0), y = Q::r5(i, 1);
        const V3 rp = V3{tri[0].x + a.x * x + b.x * y, tri[0].y + a.y * x + b.y * y, tri[0].z + a.z * x + b.z * y};
        const double wb = Q::r5(i, 2) * ww1;
        const double R = vdist(rp, rf);
        cd II;
        if (R < cut) {
            II = cmk(0.0, k / (4 * PI));
        } else {
            II = green_hd(rf, rp, k);
            II.x -= 1.0 / (4 * PI) / R;
        }
        const double sh[3] = {1 - x - y, x, y};
        for (int l = 0; l < 3; ++l) {
            acc[l].x += II.x * wb * sh[l];
            acc[l].y += II.y * wb * sh[l];
        }
    }
    double ai[1][3];
    analytic_tri_N<1>(tri, tn, rf, ai);
    for (int l = 0; l < 3; ++l) out[l] = cmk(acc[l].x + 1.0 / (4 * PI) * ai[0][l], acc[l].y);
}

// geometry of one (test, basis) tet pair
struct LinPair {
    V3 T[4], B[4], dNT[4], dNB[4];
    double volT, volB, k;
    cd eps;      // permittivity of the test tet
    bool self;
};

SCD_HD void lin_pair_init(LinPair &p, const double *tT, const double *tB, double volT, double volB, double k, cd eps,
                          bool self) {
    for (int v = 0; v < 4; ++v) {
        p.T[v] = V3{tT[3 * v], tT[3 * v + 1], tT[3 * v + 2]};
        p.B[v] = V3{tB[3 * v], tB[3 * v + 1], tB[3 * v + 2]};
    }
    gradshape_hd(p.T, p.dNT);
    gradshape_hd(p.B, p.dNB);
    p.volT = volT;
    p.volB = volB;
    p.k = k;
    p.eps = eps;
    p.self = self;
}

constexpr int LIN_POINTS = 52;     // 24 tet points + 4 x 7 face points of the test tet
constexpr int LIN_ITEMS = 5 * LIN_POINTS;
constexpr int LIN_SCR = 16;        // scratch values per point
constexpr int LIN_SMALL = 40;      // GNN (16), II4 (12), II5 (12)

// test point pt (0..51) with its weight; for face points also face and rule index
template <class Q>
SCD_HD V3 lin_test_point(const LinPair &p, int pt, double &w, V3 *tn = nullptr) {
    if (pt < 24) {
        w = Q::t5(pt, 3) * 6.0 * p.volT;
        return bary_point(p.T, Q::t5(pt, 0), Q::t5(pt, 1), Q::t5(pt, 2));
    }
    const int ft = (pt - 24) / 7, i = (pt - 24) % 7;
    V3 tri[3], a, b;
    face_tri(p.T, ft, tri);
    w = Q::r5(i, 2) * tri_ww1(tri, a, b);
    if (tn) *tn = tri_normal(tri);
    const double x = Q::r5(i, 0), y = Q::r5(i, 1);
    return V3{tri[0].x + a.x * x + b.x * y, tri[0].y + a.y * x + b.y * y, tri[0].z + a.z * x + b.z * y};
}

// phase 1, item = 5 pt + part: part 0 -> int_V_GN at scr[16 pt + 0..3];
// part 1 + f -> int_S_GN over face f of B at scr[16 pt + 4 + 3 f + 0..2]
template <class Q>
SCD_HD void lin_point(const LinPair &p, int item, cd *scr) {
    const int pt = item / 5, part = item % 5;
    double w;
    const V3 rf = lin_test_point<Q>(p, pt, w);
    if (part == 0) {
        int_V_GN_hd<Q>(rf, p.k, p.B, p.volB, p.dNB, scr + LIN_SCR * pt);
    } else {
        V3 tri[3];
        face_tri(p.B, part - 1, tri);
        int_S_GN_hd<Q>(rf, tri, tri_normal(tri), p.k, scr + LIN_SCR * pt + 4 + 3 * (part - 1));
    }
}

// J_c(b) at test point pt: sum over the faces of B holding node b of n_c int N_b G dS'
SCD_HD cd lin_J(const LinPair &p, const cd *scr, int pt, int c, int b) {
    cd s = cmk(0, 0);
    for (int f = 0; f < 4; ++f) {
        for (int l = 0; l < 3; ++l)
            if (face_vertex(f, l) == b) {
                V3 tri[3];
                face_tri(p.B, f, tri);
                const V3 n = tri_normal(tri);
                const double nc = c == 0 ? n.x : c == 1 ? n.y : n.z;
                const cd v = scr[LIN_SCR * pt + 4 + 3 * f + l];
                s.x += v.x * nc;
                s.y += v.y * nc;
            }
    }
    return s;
}

SCD_HD double comp(V3 v, int c) { return c == 0 ? v.x : c == 1 ? v.y : v.z; }

template <class Q>
SCD_HD double tet_shape(int i, int a) {
    return a == 0 ? 1 - Q::t5(i, 0) - Q::t5(i, 1) - Q::t5(i, 2) : Q::t5(i, a - 1);
}
template <class Q>
SCD_HD double tri_shape(int i, int l) {
    return l == 0 ? 1 - Q::r5(i, 0) - Q::r5(i, 1) : Q::r5(i, l - 1);
}

// phase 2, idx 0..39: sm[a + 4 b] = GNN(a, b); sm[16 + 4 r + a] = II4; sm[28 + 4 c + b] = II5
template <class Q>
SCD_HD void lin_small(const LinPair &p, int idx, const cd *scr, cd *sm) {
    cd s = cmk(0, 0);
    if (idx < 16) {
        const int a = idx % 4, b = idx / 4;
        for (int i = 0; i < 24; ++i) {
            const double w = Q::t5(i, 3) * 6.0 * p.volT;
            const cd v = scr[LIN_SCR * i + b];
            const double f = tet_shape<Q>(i, a);
            s.x += v.x * f * w;
            s.y += v.y * f * w;
        }
    } else if (idx < 28) {
        const int q = idx - 16, r = q / 4, a = q % 4;
        for (int ft = 0; ft < 4; ++ft) {
            int l = -1;
            for (int m = 0; m < 3; ++m)
                if (face_vertex(ft, m) == a) l = m;
            cd in = cmk(0, 0);
            V3 tn = V3{0, 0, 0};
            if (l >= 0) {
                for (int i = 0; i < 7; ++i) {
                    double w;
                    lin_test_point<Q>(p, 24 + 7 * ft + i, w, &tn);
                    const cd *v = scr + LIN_SCR * (24 + 7 * ft + i);
                    const cd Is = cadd(cadd(cadd(v[0], v[1]), v[2]), v[3]);
                    const double f = tri_shape<Q>(i, l);
                    in.x += Is.x * f * w;
                    in.y += Is.y * f * w;
                }
            }
            const double nr = comp(tn, r);
            s.x += in.x * nr;
            s.y += in.y * nr;
        }
    } else {
        const int q = idx - 28, c = q / 4, b = q % 4;
        for (int i = 0; i < 24; ++i) {
            const double w = Q::t5(i, 3) * 6.0 * p.volT;
            const cd J = lin_J(p, scr, i, c, b);
            s.x += J.x * w;
            s.y += J.y * w;
        }
    }
    sm[idx] = s;
}

// phase 3, e = row + 12 col (row = 4 r + a, col = 4 c + b): entry of the
// block.  st[(a*4 + g)*27 + u]: projector g (S, Sx, Sy, Sz) of test node a;
// gp[(b*4 + g)*27 + u]: G times projector g of basis node b (box of the test
// tet's nodes x box of the basis tet's nodes, compute_pG).
template <class Q>
SCD_HD cd lin_entry(const LinPair &p, int e, const cd *scr, const cd *sm, const cd *st, const cd *gp) {
    const int row = e % 12, col = e / 12;
    const int r = row / 4, a = row % 4, c = col / 4, b = col % 4;
    // alok2: faces of T holding node a
    cd al2 = cmk(0, 0);
    for (int ft = 0; ft < 4; ++ft) {
        int l = -1;
        for (int m = 0; m < 3; ++m)
            if (face_vertex(ft, m) == a) l = m;
        cd ii = cmk(0, 0);
        V3 tn = V3{0, 0, 0};
        for (int i = 0; i < 7; ++i) {
            double w;
            lin_test_point<Q>(p, 24 + 7 * ft + i, w, &tn);
            if (l < 0) continue;
            const cd J = lin_J(p, scr, 24 + 7 * ft + i, c, b);
            const double f = tri_shape<Q>(i, l);
            ii.x += J.x * f * w;
            ii.y += J.y * f * w;
        }
        const double nr = comp(tn, r);
        al2.x += ii.x * nr;
        al2.y += ii.y * nr;
    }
    cd sG = cmk(0, 0);
    for (int q = 0; q < 16; ++q) sG = cadd(sG, sm[q]);
    const double dTa = comp(p.dNT[a], r), dBb = comp(p.dNB[b], c);
    const cd al1 = r == c ? sm[a + 4 * b] : cmk(0, 0);
    const cd al3 = cscale(sG, dTa * dBb);
    const cd al4 = cscale(sm[16 + row], dBb);
    const cd al5 = cscale(sm[28 + col], dTa);
    // precorrect_lin
    const double sv = sqrt(p.volT * p.volB);
    cd c1 = cmk(0, 0), c2 = cmk(0, 0);
    for (int u = 0; u < 27; ++u) {
        if (r == c) cfma(c1, gp[(b * 4 + 0) * 27 + u], st[(a * 4 + 0) * 27 + u]);
        cfma(c2, gp[(b * 4 + 1 + c) * 27 + u], st[(a * 4 + 1 + r) * 27 + u]);
    }
    c1 = cscale(c1, sv);
    c2 = cscale(c2, sv);
    cd v = csub(cadd(cscale(csub(al1, c1), -p.k * p.k), csub(csub(cadd(al2, al3), al4), al5)), c2);
    if (p.self && r == c) {
        double nn = 0.0;
        for (int i = 0; i < 24; ++i) nn += tet_shape<Q>(i, b) * tet_shape<Q>(i, a) * Q::t5(i, 3) * 6.0 * p.volT;
        v = cadd(v, cdiv(cmk(nn, 0.0), cmk(p.eps.x - 1.0, p.eps.y)));
    }
    return cscale(v, 1.0 / sqrt(p.volB * p.volT));
}

// projector columns of one tet (pfft_projection_lin, src/projection.f90:170-338):
// the Green integrals against sample point r of the four node functions,
// q[n] = int N_n G dV (order-5 tet rule) and q2[d][n] = sum over faces of
// n_d int N_n G dS (order-5 triangle rule)
template <class Q>
SCD_HD void lin_proj_sample(const V3 *t, double vol, V3 r, double k, cd *q, cd (*q2)[4]) {
    for (int n = 0; n < 4; ++n) {
        q[n] = cmk(0, 0);
        q2[0][n] = q2[1][n] = q2[2][n] = cmk(0, 0);
    }
    for (int i = 0; i < 24; ++i) {
        const double x = Q::t5(i, 0), y = Q::t5(i, 1), z = Q::t5(i, 2);
        const cd g = green_hd(r, bary_point(t, x, y, z), k);
        const double wb = Q::t5(i, 3) * 6.0 * vol;
        const double sh[4] = {1 - x - y - z, x, y, z};
        for (int n = 0; n < 4; ++n) {
            q[n].x += sh[n] * g.x * wb;
            q[n].y += sh[n] * g.y * wb;
        }
    }
    for (int f = 0; f < 4; ++f) {
        V3 tri[3], a, b;
        face_tri(t, f, tri);
        const double ww1 = tri_ww1(tri, a, b);
        const V3 n = tri_normal(tri);
        cd s[3] = {cmk(0, 0), cmk(0, 0), cmk(0, 0)};
        for (int i = 0; i < 7; ++i) {
            const double x = Q::r5(i, 0), y = Q::r5(i, 1);
            const V3 rp = V3{tri[0].x + a.x * x + b.x * y, tri[0].y + a.y * x + b.y * y, tri[0].z + a.z * x + b.z * y};
            const cd g = green_hd(r, rp, k);
            const double w = Q::r5(i, 2) * ww1;
            const double sh[3] = {1 - x - y, x, y};
            for (int l = 0; l < 3; ++l) {
                s[l].x += sh[l] * w * g.x;
                s[l].y += sh[l] * w * g.y;
            }
        }
        for (int l = 0; l < 3; ++l) {
            const int v = face_vertex(f, l);
            q2[0][v] = cadd(q2[0][v], cscale(s[l], n.x));
            q2[1][v] = cadd(q2[1][v], cscale(s[l], n.y));
            q2[2][v] = cadd(q2[2][v], cscale(s[l], n.z));
        }
    }
}

// Tile positions of block entry e = row + 12 col (row = 4 r + an, col = 4 c + bn)
// of the pair (test tet, basis tet), for a tile whose row group holds tet p and
// column group tet q (local tet indices).  A tile stores row pseudo-tet i x
// column pseudo-tet j as 3x3 blocks, element (r', c') at r' + 3 c'; an
// off-diagonal tile is also applied transposed, a diagonal tile holds both
// halves, and the 16 blocks inside one tet are stored once.  fwd: the test
// tet is tet p.  Writes (i, j, element) triples to pos and returns their number.
SCD_HD int lin_tile_positions(bool diag, bool fwd, int p, int q, int e, int *pos) {
    const int row = e % 12, col = e / 12;
    const int r = row / 4, an = row % 4, c = col / 4, bn = col % 4;
    if (diag) {
        const int lt = fwd ? p : q, lb = fwd ? q : p;
        pos[0] = 4 * lt + an; pos[1] = 4 * lb + bn; pos[2] = r + 3 * c;
        if (lt == lb) return 1;
        pos[3] = 4 * lb + bn; pos[4] = 4 * lt + an; pos[5] = c + 3 * r;
        return 2;
    }
    if (fwd) {
        pos[0] = 4 * p + an; pos[1] = 4 * q + bn; pos[2] = r + 3 * c;
    } else {
        pos[0] = 4 * p + bn; pos[1] = 4 * q + an; pos[2] = c + 3 * r;
    }
    return 1;
}
