// Per-wavelength operator construction from the mesh, on the device:
//   build_grid           src/geometry.f90:60-125        (host)
//   tetras_in_cubes      src/geometry.f90:330-377       (host binning)
//   pfft_projection_const src/projection.f90:17-166     (pinv on the host,
//                                                         per-tet kernel)
//   compute_near_zone_interactions_const
//                        src/precorrection.f90:131-264  (FP64 kernel that
//                                                         writes the tiles)
//   vswf2constant / calc_MN src/T_matrix.f90:280-305, src/mie.f90:408-496
// The quadrature rules are the published ones the reference tabulates
// (src/integration_points.f90): Keast's 24-point tetrahedron rule, the 7-point
// degree-5 triangle rule, the 1-point centroid rules and the 98 surface nodes
// of the 5x5x5 lattice on [-1,1]^3.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "geom.cuh"
#include "lin_setup.cuh"

namespace {

// ------------------------------------------------------------- quadrature
__constant__ double cQT5[24][4];   // (xi, eta, zeta, w)
__constant__ double cQR5[7][3];    // (xi, eta, w)
__constant__ double cPs[98][3];    // cube sample points (unscaled)

const HostQuad &hq() {
    static HostQuad q;
    return q;
}

int upload_quadrature(scd_ctx *c) {
    // per device: set once its tables are on the device (contexts of a
    // server build operators from several host threads)
    static std::atomic<bool> done[128];
    const bool tracked = c->dev >= 0 && c->dev < 128;
    if (tracked && done[c->dev].load(std::memory_order_acquire)) return SCD_OK;
    const HostQuad &q = hq();
    // copies on the context's stream, finished before any context of the
    // device may read the tables
    int rc = check_cuda(c, cudaMemcpyToSymbolAsync(cQT5, q.t5, sizeof q.t5, 0, cudaMemcpyHostToDevice, c->st), "quadrature");
    if (!rc) rc = check_cuda(c, cudaMemcpyToSymbolAsync(cQR5, q.r5, sizeof q.r5, 0, cudaMemcpyHostToDevice, c->st), "quadrature");
    if (!rc) rc = check_cuda(c, cudaMemcpyToSymbolAsync(cPs, q.ps, sizeof q.ps, 0, cudaMemcpyHostToDevice, c->st), "quadrature");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "quadrature");
    if (!rc && tracked) done[c->dev].store(true, std::memory_order_release);
    return rc;
}

// -------------------------------------------------------- geometry helpers
// faces opposite vertex 1..4 (src/common.f90:296-322)
__constant__ int cFACE[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
__device__ __forceinline__ void face_of(const V3 *t, int f, V3 *tri) {
    tri[0] = t[cFACE[f][0]]; tri[1] = t[cFACE[f][1]]; tri[2] = t[cFACE[f][2]];
}
// Gr (src/common.f90:271-279): exp(ikR) / (4 pi R)
__device__ __forceinline__ cd green(V3 rf, V3 rp, double k) { return green_hd(rf, rp, k); }

// analytical_integration, src/singularity_subtraction.f90:15-108: the
// integrals of 1/R and R over a triangle (Np = 2)
__device__ void analytic_tri(const V3 *tri, V3 n, V3 r, double &K1, double &K2) {
    const double w0 = vdot(vsub(r, tri[0]), n);
    double tl[3], Il[3];
    double Km1 = 0.0;
    // edges l = 1..3: (l2, l1) = (3,2), (1,3), (2,1) in 1-based vertex ids
    const int L2[3] = {2, 0, 1}, L1[3] = {1, 2, 0};
    double sp[3], sm[3], rp[3], rm[3], r0[3];
    for (int l = 0; l < 3; ++l) {
        const V3 p2 = tri[L2[l]], p1 = tri[L1[l]];
        const V3 slv = vsub(p2, p1);
        const double ns = sqrt(vdot(slv, slv));
        const V3 sl = V3{slv.x / ns, slv.y / ns, slv.z / ns};
        const V3 ml = vcross(sl, n);
        const V3 pl1mr = vsub(p1, r);
        const double tl0 = vdot(pl1mr, ml);
        const double ll = sqrt(vdot(slv, slv));
        const double sml = vdot(pl1mr, sl), spl = sml + ll;
        const V3 rmp2 = vsub(r, p2);
        const double Rpl = sqrt(vdot(rmp2, rmp2)), Rml = sqrt(vdot(pl1mr, pl1mr));
        const double R0l = sqrt(tl0 * tl0 + w0 * w0);
        tl[l] = tl0;
        double Km3;
        if (fabs(w0) > 1.0e-10) {
            const double Bl = atan((tl0 * spl) / (R0l * R0l + fabs(w0) * Rpl)) - atan((tl0 * sml) / (R0l * R0l + fabs(w0) * Rml));
            Km3 = 1.0 / fabs(w0) * Bl;
        } else {
            Km3 = 0.0;
        }
        if ((Rml + sml) > (Rpl - spl)) Il[l] = log(fabs((Rpl + spl) / (Rml + sml)));
        else Il[l] = log(fabs((Rml - sml) / (Rpl - spl)));
        Km1 = Km1 + 1.0 / (-1.0 + 2.0) * (-1.0 * w0 * w0 * Km3 + tl0 * Il[l]);
        sp[l] = spl; sm[l] = sml; rp[l] = Rpl; rm[l] = Rml; r0[l] = R0l;
    }
    // n = 1: I_l = 1/2 (s+ R+ - s- R- + R0^2 I_l); K1 = 1/3 (w0^2 K_-1 + sum t I)
    for (int l = 0; l < 3; ++l)
        Il[l] = 1.0 / (1.0 + 1.0) * (sp[l] * rp[l] - sm[l] * rm[l] + 1.0 * r0[l] * r0[l] * Il[l]);
    const double K1v = 1.0 / (1.0 + 2.0) * (1.0 * w0 * w0 * Km1 + (tl[0] * Il[0] + tl[1] * Il[1] + tl[2] * Il[2]));
    K1 = Km1;
    K2 = K1v;
}

// singularity_subtraction_int_V_G, src/singularity_subtraction.f90:112-189
__device__ cd int_V_G(V3 rf, double k, const V3 *Pb, const double *wb, double sumw, const V3 *B) {
    const double cut = 1.0e-10 * pow(sumw, F13_D);
    const double c4 = 1.0 / (4 * PI);
    cd intR = cmk(0, 0);
    for (int i = 0; i < 24; ++i) {
        const double RR = vdist(Pb[i], rf);
        cd II;
        if (RR < cut) II = cmk(0.0, k / (4.0 * PI));
        else {
            const double f = c4 * 1.0 * 1.0 / RR + c4 * (k * k) * (-0.5) * RR;
            II = green(rf, Pb[i], k);
            II.x -= f;
        }
        intR.x += II.x * wb[i];
        intR.y += II.y * wb[i];
    }
    double i4a = 0.0, i4b = 0.0;
    for (int f = 0; f < 4; ++f) {
        V3 tri[3];
        face_of(B, f, tri);
        const V3 n = tri_normal(tri);
        double K1, K2;
        analytic_tri(tri, n, rf, K1, K2);
        const double a1 = vdot(n, vsub(tri[0], rf));
        i4a = i4a + a1 * K1 * 0.5;
        i4b = i4b + a1 * K2 * 0.25;
    }
    const double f2 = c4 * 1.0 * i4a + c4 * (k * k) * (-0.5) * i4b;
    return cmk(intR.x + f2, intR.y);
}

// singularity_subtraction_int_S_G, src/singularity_subtraction.f90:193-243
__device__ cd int_S_G(V3 rf, const V3 *tri, V3 n, double k, const V3 *Pb, const double *wb, double sumw) {
    const double cut = 1.0e-10 * sqrt(sumw);
    const double c4 = 1.0 / (4 * PI);
    cd intR = cmk(0, 0);
    for (int i = 0; i < 7; ++i) {
        const double R = vdist(Pb[i], rf);
        cd II;
        if (R < cut) II = cmk(0.0, k / (4 * PI));
        else {
            const double f = c4 * 1.0 * 1.0 / R + c4 * (k * k) * (-0.5) * R;
            II = green(rf, Pb[i], k);
            II.x -= f;
        }
        intR.x += II.x * wb[i];
        intR.y += II.y * wb[i];
    }
    double K1, K2;
    analytic_tri(tri, n, rf, K1, K2);
    const double f2 = c4 * 1.0 * K1 + c4 * (k * k) * (-0.5) * K2;
    return cmk(intR.x + f2, intR.y);
}

}  // namespace

namespace {

// ---------------------------------------------------------------- blocks
// One near-zone block (src/precorrection.f90:183-254) for test tet t and
// basis tet b (original numbering t <= b):
//   blk = delta_tb I/(eps_t - 1) + (-k^2 (V_VG - corr) + (dV_dVG - corr2))/sqrt(vol_t vol_b)
// where corr = S_t^T G S_b I and corr2(r,c) = P_r,t^T G P_c,b with the 27x27
// grid Green matrix G of the two boxes (compute_pG, :21-46, precorrect_const,
// :50-82).  gs/gx/gy/gz = G S_b, G Sx_b, G Sy_b, G Sz_b (27 each).
struct TetGeo {
    V3 v[4];
    double vol;
};

__device__ void near_block(const TetGeo &T, const TetGeo &B, bool self, cd eps_t, double k,
                           const cd *St, const cd *Sxt, const cd *Syt, const cd *Szt, long long ps,
                           const cd *gs, const cd *gx, const cd *gy, const cd *gz, cd out[9]) {
    // precorrection (linear in S; computed from G times basis projectors)
    cd acorr = cmk(0, 0);
    cd corr2[9];
    for (int q = 0; q < 9; ++q) corr2[q] = cmk(0, 0);
    for (int a = 0; a < 27; ++a) {
        cfma(acorr, gs[a], St[a * ps]);
        const cd pt[3] = {Sxt[a * ps], Syt[a * ps], Szt[a * ps]};
        const cd gb[3] = {gx[a], gy[a], gz[a]};
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) cfma(corr2[r + 3 * c], gb[c], pt[r]);
    }
    const double sv = sqrt(T.vol * B.vol);
    acorr = cscale(acorr, sv);
    for (int q = 0; q < 9; ++q) corr2[q] = cscale(corr2[q], sv);

    // order-5 points of the basis tet (linmap_tet, src/common.f90:1354-1377)
    V3 Pb[24];
    double wb[24], sumw = 0.0;
    for (int i = 0; i < 24; ++i) {
        const double N2 = cQT5[i][0], N3 = cQT5[i][1], N4 = cQT5[i][2], N1 = 1 - N2 - N3 - N4;
        Pb[i] = V3{B.v[0].x * N1 + B.v[1].x * N2 + B.v[2].x * N3 + B.v[3].x * N4,
                   B.v[0].y * N1 + B.v[1].y * N2 + B.v[2].y * N3 + B.v[3].y * N4,
                   B.v[0].z * N1 + B.v[1].z * N2 + B.v[2].z * N3 + B.v[3].z * N4};
        wb[i] = cQT5[i][3] * 6.0 * B.vol;
        sumw += wb[i];
    }
    // integrate_V_V_G (src/precorrection.f90:729-760)
    cd vvg = cmk(0, 0);
    for (int i = 0; i < 24; ++i) {
        const double N2 = cQT5[i][0], N3 = cQT5[i][1], N4 = cQT5[i][2], N1 = 1 - N2 - N3 - N4;
        const V3 rf = V3{T.v[0].x * N1 + T.v[1].x * N2 + T.v[2].x * N3 + T.v[3].x * N4,
                         T.v[0].y * N1 + T.v[1].y * N2 + T.v[2].y * N3 + T.v[3].y * N4,
                         T.v[0].z * N1 + T.v[1].z * N2 + T.v[2].z * N3 + T.v[3].z * N4};
        const double wt = cQT5[i][3] * 6.0 * T.vol;
        const cd in = int_V_G(rf, k, Pb, wb, sumw, B.v);
        vvg.x += in.x * wt;
        vvg.y += in.y * wt;
    }
    // integrate_dV_dV_G (src/precorrection.f90:764-806)
    cd dvv[9];
    for (int q = 0; q < 9; ++q) dvv[q] = cmk(0, 0);
    for (int ft = 0; ft < 4; ++ft) {
        V3 ttri[3], ta, tb;
        face_of(T.v, ft, ttri);
        const V3 tn = tri_normal(ttri);
        const double tw1 = tri_ww1(ttri, ta, tb);
        for (int fb = 0; fb < 4; ++fb) {
            V3 btri[3], ba, bb;
            face_of(B.v, fb, btri);
            const V3 bn = tri_normal(btri);
            const double bw1 = tri_ww1(btri, ba, bb);
            V3 Pbt[7];
            double wbt[7], sw = 0.0;
            for (int j = 0; j < 7; ++j) {
                Pbt[j] = V3{btri[0].x + ba.x * cQR5[j][0] + bb.x * cQR5[j][1],
                            btri[0].y + ba.y * cQR5[j][0] + bb.y * cQR5[j][1],
                            btri[0].z + ba.z * cQR5[j][0] + bb.z * cQR5[j][1]};
                wbt[j] = cQR5[j][2] * bw1;
                sw += wbt[j];
            }
            cd acc = cmk(0, 0);
            for (int i = 0; i < 7; ++i) {
                const V3 rf = V3{ttri[0].x + ta.x * cQR5[i][0] + tb.x * cQR5[i][1],
                                 ttri[0].y + ta.y * cQR5[i][0] + tb.y * cQR5[i][1],
                                 ttri[0].z + ta.z * cQR5[i][0] + tb.z * cQR5[i][1]};
                const double wt = cQR5[i][2] * tw1;
                const cd in = int_S_G(rf, btri, bn, k, Pbt, wbt, sw);
                acc.x += in.x * wt;
                acc.y += in.y * wt;
            }
            const double tnv[3] = {tn.x, tn.y, tn.z}, bnv[3] = {bn.x, bn.y, bn.z};
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    const double m = tnv[r] * bnv[c];
                    dvv[r + 3 * c].x += m * acc.x;
                    dvv[r + 3 * c].y += m * acc.y;
                }
        }
    }
    const double k2 = k * k, inv = 1.0 / sqrt(B.vol * T.vol);
    const cd einv = cdiv(cmk(1.0, 0.0), cmk(eps_t.x - 1.0, eps_t.y));
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int q = r + 3 * c;
            cd v = cmk(0, 0);
            if (r == c) {
                const cd d1 = csub(vvg, acorr);
                v = cmk(-k2 * d1.x, -k2 * d1.y);
            }
            const cd d2 = csub(dvv[q], corr2[q]);
            v = cmk(inv * (v.x + d2.x), inv * (v.y + d2.y));
            if (self && r == c) v = cadd(v, einv);
            out[q] = v;
        }
}

// ------------------------------------------------------------- near kernel
// One CTA per tile (c1 <= c2).  Shared: box-node Green matrix G(c1,c2) and
// G (resp. G^T) times the basis projectors of every tet of the tile.
struct NearArgs {
    const NearTile *tiles;
    const double *tc;        // slot-ordered vertex coords, 12 per slot
    const double *vol;       // slot-ordered volumes
    const cd *eps;           // slot-ordered eps
    const cd *P;             // projectors [g][27*slot + j]
    const int *perm;         // slot -> original tet
    const int *cube_off;
    int T;
    int ncx, ncy, Nx, Ny;
    double delta, mx, my, mz, k;
    void *data;              // tile storage
    int c64;                 // 1: complex64 storage
};

__device__ __forceinline__ V3 box_node(const NearArgs &a, int cube, int j) {
    const int bx = cube % a.ncx, by = (cube / a.ncx) % a.ncy, bz = cube / (a.ncx * a.ncy);
    const int x = 2 * bx + j % 3, y = 2 * by + (j / 3) % 3, z = 2 * bz + j / 9;
    return V3{a.mx + a.delta * (double)x, a.my + a.delta * (double)y, a.mz + a.delta * (double)z};
}
__device__ __forceinline__ long long box_node_id(const NearArgs &a, int cube, int j) {
    const int bx = cube % a.ncx, by = (cube / a.ncx) % a.ncy, bz = cube / (a.ncx * a.ncy);
    const int x = 2 * bx + j % 3, y = 2 * by + (j / 3) % 3, z = 2 * bz + j / 9;
    return ((long long)z * a.Ny + y) * a.Nx + x;
}

__device__ __forceinline__ void load_tet(const NearArgs &a, int slot, TetGeo &t) {
    const double *p = a.tc + 12LL * slot;
    for (int v = 0; v < 4; ++v) t.v[v] = V3{p[3 * v], p[3 * v + 1], p[3 * v + 2]};
    t.vol = a.vol[slot];
}

// block (i, j) of tile tl, from column-major blk (transposed when tr)
__device__ __forceinline__ void store_block(const NearArgs &a, const NearTile &tl, int i, int j, const cd *blk, bool tr) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            const cd v = tr ? blk[c + 3 * r] : blk[r + 3 * c];
            const long long e = tl.data_off + tile_at(tl.n1, i, j, r + 3 * c);
            if (a.c64) ((cf *)a.data)[e] = make_float2((float)v.x, (float)v.y);
            else ((cd *)a.data)[e] = v;
        }
}

constexpr int NEAR_THREADS = 128;

// box-node Green matrix of a tile's two boxes and G (resp. G^T) times the
// projectors of every basis function of the tile, in shared memory
__device__ void tile_green(const NearArgs &a, const NearTile &tl, cd *G, cd *GP1, cd *GP2) {
    for (int e = threadIdx.x; e < 27 * 27; e += blockDim.x) {
        const int i = e / 27, j = e % 27;
        cd v = cmk(0, 0);
        if (box_node_id(a, tl.c1, i) != box_node_id(a, tl.c2, j))
            v = green(box_node(a, tl.c1, i), box_node(a, tl.c2, j), a.k);
        G[e] = v;
    }
    __syncthreads();
    const long long TT = 27LL * a.T;
    const int s1 = tl.s1, s2 = tl.s2;
    // GP2[j][g][row i of c1-box] = sum_q G[i][q] P_g(q, tet j of c2)   (test in c1, basis in c2)
    for (int e = threadIdx.x; e < tl.n2 * 108; e += blockDim.x) {
        const int j = e / 108, g = (e / 27) % 4, i = e % 27;
        const cd *p = a.P + (size_t)g * TT + (s2 + j);
        cd acc = cmk(0, 0);
        for (int q = 0; q < 27; ++q) cfma(acc, G[i * 27 + q], p[(size_t)q * a.T]);
        GP2[e] = acc;
    }
    // GP1[i][g][row q of c2-box] = sum_p G[p][q] P_g(p, tet i of c1)   (test in c2, basis in c1)
    if (tl.g1 != tl.g2) {
        for (int e = threadIdx.x; e < tl.n1 * 108; e += blockDim.x) {
            const int i = e / 108, g = (e / 27) % 4, q = e % 27;
            const cd *p = a.P + (size_t)g * TT + (s1 + i);
            cd acc = cmk(0, 0);
            for (int pp = 0; pp < 27; ++pp) cfma(acc, G[pp * 27 + q], p[(size_t)pp * a.T]);
            GP1[e] = acc;
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(NEAR_THREADS) k_near_build(NearArgs a) {
    extern __shared__ cd shm[];
    const NearTile tl = a.tiles[blockIdx.x];
    cd *G = shm;                                    // 27 x 27: G[i*27 + j] = Gr(node_c1(i), node_c2(j))
    cd *GP1 = G + 27 * 27;                          // per tet of c1: G^T P (4 x 27)
    cd *GP2 = GP1 + (size_t)tl.n1 * 108;            // per tet of c2: G P (4 x 27)
    tile_green(a, tl, G, GP1, GP2);
    const long long TT = 27LL * a.T;
    const int s1 = tl.s1, s2 = tl.s2;
    const bool diag = tl.g1 == tl.g2;
    const int npairs = tl.n1 * tl.n2;
    for (int e = threadIdx.x; e < npairs; e += blockDim.x) {
        const int i = e / tl.n2, j = e % tl.n2;
        if (diag && j < i) continue;                // diagonal tile: each pair once
        const int sa = s1 + i, sb = s2 + j;
        const bool fwd = a.perm[sa] <= a.perm[sb];  // test = lower original index
        const int st = fwd ? sa : sb, sbas = fwd ? sb : sa;
        const cd *gp = fwd ? GP2 + (size_t)j * 108 : GP1 + (size_t)i * 108;
        TetGeo Tt, Bt;
        load_tet(a, st, Tt);
        load_tet(a, sbas, Bt);
        cd blk[9];
        near_block(Tt, Bt, st == sbas, a.eps[st], a.k, a.P + st, a.P + TT + st, a.P + 2 * TT + st, a.P + 3 * TT + st,
                   a.T, gp, gp + 27, gp + 54, gp + 81, blk);
        store_block(a, tl, i, j, blk, !fwd);
        if (diag && i != j) store_block(a, tl, j, i, blk, true);
    }
}

// ------------------------------------------------------- linear basis
// quadrature accessor for the shared set-up arithmetic (lin_setup.cuh)
struct DevQ {
    SCD_HD static double t5(int i, int c) {
#ifdef __CUDA_ARCH__
        return cQT5[i][c];
#else
        return hq().t5[i][c];
#endif
    }
    SCD_HD static double r5(int i, int c) {
#ifdef __CUDA_ARCH__
        return cQR5[i][c];
#else
        return hq().r5[i][c];
#endif
    }
};

__device__ __forceinline__ void store_elem(const NearArgs &a, const NearTile &tl, int i, int j, int el, cd v) {
    const long long e = tl.data_off + tile_at(tl.n1, i, j, el);
    if (a.c64) ((cf *)a.data)[e] = make_float2((float)v.x, (float)v.y);
    else ((cd *)a.data)[e] = v;
}

constexpr int LIN_WARPS = 4;
constexpr int LIN_WARP_CD = LIN_POINTS * LIN_SCR + LIN_SMALL + 432;   // scratch, small sums, test projectors

// compute_near_zone_interactions_lin (src/precorrection.f90:268-371) on a
// tile of pseudo-tets (4 consecutive slots per tet, whole tets per group):
// one warp per tet pair computes the 12x12 block and writes its 16 3x3
// pseudo-tet blocks, mirrored between different tets, one-sided inside a tet.
__global__ void __launch_bounds__(32 * LIN_WARPS) k_near_build_lin(NearArgs a) {
    extern __shared__ cd shm[];
    const NearTile tl = a.tiles[blockIdx.x];
    cd *G = shm;
    cd *GP1 = G + 27 * 27;
    cd *GP2 = GP1 + (size_t)tl.n1 * 108;
    tile_green(a, tl, G, GP1, GP2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    cd *scr = GP2 + (size_t)tl.n2 * 108 + (size_t)warp * LIN_WARP_CD;
    cd *sm = scr + LIN_POINTS * LIN_SCR;
    cd *st = sm + LIN_SMALL;
    const bool diag = tl.g1 == tl.g2;
    const int nt1 = tl.n1 / 4, nt2 = tl.n2 / 4;
    for (int e = warp; e < nt1 * nt2; e += LIN_WARPS) {
        const int p = e / nt2, q = e % nt2;
        if (diag && q < p) continue;
        const int sa = tl.s1 + 4 * p, sb = tl.s2 + 4 * q;
        const bool fwd = a.perm[sa] <= a.perm[sb];      // test = lower original tet
        const int s_t = fwd ? sa : sb, s_b = fwd ? sb : sa;
        const cd *gp = diag ? GP2 + (size_t)4 * (fwd ? q : p) * 108 : fwd ? GP2 + (size_t)4 * q * 108 : GP1 + (size_t)4 * p * 108;
        LinPair pr;
        lin_pair_init(pr, a.tc + 12LL * s_t, a.tc + 12LL * s_b, a.vol[s_t], a.vol[s_b], a.k, a.eps[s_t], s_t == s_b);
        for (int i = lane; i < 432; i += 32) {
            const int an = i / 108, g = (i / 27) % 4, u = i % 27;
            st[i] = a.P[(size_t)(g * 27 + u) * a.T + s_t + an];
        }
        for (int it = lane; it < LIN_ITEMS; it += 32) lin_point<DevQ>(pr, it, scr);
        __syncwarp();
        for (int i = lane; i < LIN_SMALL; i += 32) lin_small<DevQ>(pr, i, scr, sm);
        __syncwarp();
        for (int i = lane; i < 144; i += 32) {
            const cd v = lin_entry<DevQ>(pr, i, scr, sm, st, gp);
            int pos[6];
            const int np = lin_tile_positions(diag, fwd, p, q, i, pos);
            for (int w = 0; w < np; ++w) store_elem(a, tl, pos[3 * w], pos[3 * w + 1], pos[3 * w + 2], v);
        }
        __syncwarp();
    }
}

// pfft_projection_lin (src/projection.f90:170-338) for one tet per warp: the
// node integrals against the 98 samples, then S = WW Q / sqrt(vol) and
// Sd = (WW Q2_d - WW (QdN dN_d)) / sqrt(vol) for its four pseudo-tet slots
__global__ void __launch_bounds__(32) k_projectors_lin(const double *tc, const double *vol, const int *cube_of_slot,
                                                       const int *slot0, int ntet, int T, const cd *WW, int ncx, int ncy,
                                                       double delta, double mx, double my, double mz, double box_delta,
                                                       double k, cd *P) {
    __shared__ cd Qs[17][98];   // Q[n] (4), Q2[d][n] (12), QdN
    const int q = blockIdx.x, lane = threadIdx.x;
    if (q >= ntet) return;
    const int s0 = slot0[q];
    const double *p = tc + 12LL * s0;
    V3 v[4];
    for (int i = 0; i < 4; ++i) v[i] = V3{p[3 * i], p[3 * i + 1], p[3 * i + 2]};
    const double vb = vol[s0];
    const int cube = cube_of_slot[s0];
    const int bx = cube % ncx, by = (cube / ncx) % ncy, bz = cube / (ncx * ncy);
    const V3 cpc = V3{mx + delta * (double)(2 * bx) + box_delta / 2.0, my + delta * (double)(2 * by) + box_delta / 2.0,
                      mz + delta * (double)(2 * bz) + box_delta / 2.0};
    const double sc = 2.0 * box_delta;
    for (int m = lane; m < 98; m += 32) {
        const V3 r = V3{sc * cPs[m][0] + cpc.x, sc * cPs[m][1] + cpc.y, sc * cPs[m][2] + cpc.z};
        cd qq[4], q2[3][4];
        lin_proj_sample<DevQ>(v, vb, r, k, qq, q2);
        for (int n = 0; n < 4; ++n) {
            Qs[n][m] = qq[n];
            for (int d = 0; d < 3; ++d) Qs[4 + 4 * d + n][m] = q2[d][n];
        }
        Qs[16][m] = cadd(cadd(cadd(qq[0], qq[1]), qq[2]), qq[3]);
    }
    __syncwarp();
    if (lane < 27) {
        V3 dN[4];
        gradshape_hd(v, dN);
        cd acc[17];
        for (int j = 0; j < 17; ++j) acc[j] = cmk(0, 0);
        for (int m = 0; m < 98; ++m) {
            const cd w = WW[lane * 98 + m];
            for (int j = 0; j < 17; ++j) cfma(acc[j], w, Qs[j][m]);
        }
        const double sv = sqrt(vb);
        for (int n = 0; n < 4; ++n) {
            P[(size_t)lane * T + s0 + n] = cmk(acc[n].x / sv, acc[n].y / sv);
            for (int d = 0; d < 3; ++d) {
                const cd x = csub(acc[4 + 4 * d + n], cscale(acc[16], comp(dN[n], d)));
                P[(size_t)((1 + d) * 27 + lane) * T + s0 + n] = cmk(x.x / sv, x.y / sv);
            }
        }
    }
}

// ------------------------------------------------------------ projectors
// pfft_projection_const per tet: Q(m) = Gr(sample m, centroid) vol and the
// face sums, then S = WW Q / sqrt(vol).  One warp per tet.
__global__ void k_projectors(const double *tc, const double *vol, const int *cube_of_slot, int T, const cd *WW,
                             int ncx, int ncy, double delta, double mx, double my, double mz, double box_delta,
                             double k, cd *P) {
    __shared__ cd Qs[4][4][98];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * 4 + warp;
    if (s >= T) return;
    const double *p = tc + 12LL * s;
    V3 v[4];
    for (int q = 0; q < 4; ++q) v[q] = V3{p[3 * q], p[3 * q + 1], p[3 * q + 2]};
    const double vb = vol[s];
    const int cube = cube_of_slot[s];
    const int bx = cube % ncx, by = (cube / ncx) % ncy, bz = cube / (ncx * ncy);
    const V3 node1 = V3{mx + delta * (double)(2 * bx), my + delta * (double)(2 * by), mz + delta * (double)(2 * bz)};
    const V3 cpc = V3{node1.x + box_delta / 2.0, node1.y + box_delta / 2.0, node1.z + box_delta / 2.0};
    // 1-point tet rule: barycentre, weight 1/6 * 6 vol
    const double N = 0.25, N1 = 1 - 0.25 - 0.25 - 0.25;
    const V3 pb = V3{v[0].x * N1 + v[1].x * N + v[2].x * N + v[3].x * N, v[0].y * N1 + v[1].y * N + v[2].y * N + v[3].y * N,
                     v[0].z * N1 + v[1].z * N + v[2].z * N + v[3].z * N};
    const double wb = 1.666666666666667e-01 * 6.0 * vb;
    V3 fp[4], fn[4];
    double fw[4];
    for (int f = 0; f < 4; ++f) {
        V3 tri[3], a, b;
        face_of(v, f, tri);
        const double ww1 = tri_ww1(tri, a, b);
        const double t0 = 3.333333333333330e-01;
        fp[f] = V3{tri[0].x + a.x * t0 + b.x * t0, tri[0].y + a.y * t0 + b.y * t0, tri[0].z + a.z * t0 + b.z * t0};
        fw[f] = 0.5 * ww1;
        fn[f] = tri_normal(tri);
    }
    const double sc = 2.0 * box_delta;
    for (int m = lane; m < 98; m += 32) {
        const V3 r = V3{sc * cPs[m][0] + cpc.x, sc * cPs[m][1] + cpc.y, sc * cPs[m][2] + cpc.z};
        const cd g0 = green(r, pb, k);
        cd q = cmk(g0.x * wb, g0.y * wb), qx = cmk(0, 0), qy = qx, qz = qx;
        for (int f = 0; f < 4; ++f) {
            const cd g = green(r, fp[f], k);
            const cd q2 = cmk(fw[f] * g.x, fw[f] * g.y);
            qx = cadd(qx, cscale(q2, fn[f].x));
            qy = cadd(qy, cscale(q2, fn[f].y));
            qz = cadd(qz, cscale(q2, fn[f].z));
        }
        Qs[warp][0][m] = q; Qs[warp][1][m] = qx; Qs[warp][2][m] = qy; Qs[warp][3][m] = qz;
    }
    __syncwarp();
    if (lane < 27) {
        cd acc[4] = {cmk(0, 0), cmk(0, 0), cmk(0, 0), cmk(0, 0)};
        for (int m = 0; m < 98; ++m) {
            const cd w = WW[lane * 98 + m];
            for (int g = 0; g < 4; ++g) cfma(acc[g], w, Qs[warp][g][m]);
        }
        const double sv = sqrt(vb);
        for (int g = 0; g < 4; ++g) P[(size_t)(g * 27 + lane) * T + s] = cmk(acc[g].x / sv, acc[g].y / sv);
    }
}

// ------------------------------------------------------------------ VSWF
// calc_MN with inou = 0 (src/mie.f90:408-496) at each tet centroid, times
// sqrt(vol) (vswf2constant, src/T_matrix.f90:280-305).  One thread per tet;
// mat is slot ordered, column stride n.
__device__ double envj(int n, double x) {
    n = n < 0 ? -n : n;
    if (n < 1) n = 1;
    return 0.5 * log10(6.28 * n) - (double)n * log10(1.36 * x / n);
}
__device__ int msta1(double x, int mp) {
    const double F11 = (double)1.1f;
    const double a0 = fabs(x);
    int n0 = (int)(F11 * a0) + 1;
    double f0 = envj(n0, a0) - mp;
    int n1 = n0 + 5;
    double f1 = envj(n1, a0) - mp;
    int nn = n1;
    for (int it = 1; it <= 20; ++it) {
        nn = n1 - (int)((n1 - n0) / (1.0 - f0 / f1));
        const double f = envj(nn, a0) - mp;
        if (abs(nn - n1) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn;
}
__device__ int msta2(double x, int n, int mp) {
    const double F11 = (double)1.1f;
    const double a0 = fabs(x), hmp = 0.5 * mp, ejn = envj(n, a0);
    double obj;
    int n0;
    if (ejn <= hmp) { obj = mp; n0 = (int)(F11 * a0); }
    else { obj = hmp + ejn; n0 = n; }
    double f0 = envj(n0, a0) - obj;
    int n1 = n0 + 5;
    double f1 = envj(n1, a0) - obj;
    int nn = n1;
    for (int it = 1; it <= 20; ++it) {
        nn = n1 - (int)((n1 - n0) / (1.0 - f0 / f1));
        const double f = envj(nn, a0) - obj;
        if (abs(nn - n1) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn + 10;
}
// spherical Bessel j_0..j_n of a real argument by Miller's backward
// recurrence normalised with j_0 or j_1 (Zhang & Jin CSPHJY, as
// cspherebessel in src/sfunctions.f90:20-69 with a real kr)
constexpr int VSWF_NMAX = 40;
__device__ void sph_bessel_j(int n, double z, double *csj) {
    const double a0 = fabs(z);
    for (int q = 0; q <= n; ++q) csj[q] = 0.0;
    if (a0 < 1.0e-60) { csj[0] = 1.0; return; }   // the reference zeroes j_0 here; unreachable for tet centroids
    csj[0] = sin(z) / z;
    csj[1] = (csj[0] - cos(z)) / z;
    if (n >= 2) {
        const double csa = csj[0], csb = csj[1];
        int nm = n;
        int m = msta1(a0, 200);
        if (m < n) nm = m; else m = msta2(a0, n, 15);
        double cf0 = 0.0, cf1 = 1.0 - 100, cf = 0.0;
        double keep[VSWF_NMAX + 2];
        for (int q = 0; q <= n; ++q) keep[q] = 0.0;
        for (int kk = m; kk >= 0; --kk) {
            cf = (2.0 * kk + 3.0) * cf1 / z - cf0;
            if (kk <= nm && kk <= n) keep[kk] = cf;
            cf0 = cf1;
            cf1 = cf;
        }
        const double cs = (fabs(csa) > fabs(csb)) ? csa / cf : csb / cf0;
        const int top = nm < n ? nm : n;
        for (int q = 0; q <= n; ++q) csj[q] = 0.0;
        for (int q = 0; q <= top; ++q) csj[q] = cs * keep[q];
    }
}
// associated Legendre P_N^m(x), m = 0..N, with the Condon-Shortley phase
// (legendre2, src/sfunctions.f90:615-686): column N of the recurrence table
__device__ void legendre_col(int N, double x, double *out, double *diag_scratch) {
    // PM(m, m) then upward in degree for each order m
    const double xq = sqrt(1.0 - x * x);
    double pmm = 1.0;
    for (int m = 0; m <= N; ++m) {
        if (m > 0) pmm = -(2.0 * m - 1.0) * xq * pmm;
        diag_scratch[m] = pmm;
    }
    for (int m = 0; m <= N; ++m) {
        double pm2 = diag_scratch[m];
        if (m == N) { out[m] = pm2; continue; }
        double pm1 = (2.0 * m + 1.0) * x * pm2;
        for (int l = m + 2; l <= N; ++l) {
            const double pl = ((2.0 * l - 1.0) * x * pm1 - (m + l - 1.0) * pm2) / (double)(l - m);
            pm2 = pm1;
            pm1 = pl;
        }
        out[m] = pm1;
    }
}

// columns c0 .. c0 + cw - 1 of the 2nm (M columns, then N columns) into
// mat[(col - c0) * ld + 3 s + d]
__global__ void k_vswf(const double *tc, const double *vol, int T, double k, int Nmax, cd *mat, long long ld, int c0,
                       int cw) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= T) return;
    const double *p = tc + 12LL * s;
    const double rx = (p[0] + p[3] + p[6] + p[9]) / 4.0, ry = (p[1] + p[4] + p[7] + p[10]) / 4.0,
                 rz = (p[2] + p[5] + p[8] + p[11]) / 4.0;
    const double r = sqrt(rx * rx + ry * ry + rz * rz);
    const double theta = r != 0.0 ? acos(rz / r) : 0.0, phi = atan2(ry, rx);
    const double kr = k * r;
    double sj[VSWF_NMAX + 2];
    sph_bessel_j(Nmax + 1, kr, sj);
    double L[VSWF_NMAX + 2], L1[VSWF_NMAX + 2], L2[VSWF_NMAX + 2], scr[VSWF_NMAX + 2];
    double st, ct, sp, cp;
    sincos(theta, &st, &ct);
    sincos(phi, &sp, &cp);
    const double H[3][3] = {{st * cp, ct * cp, -sp}, {st * sp, ct * sp, cp}, {ct, -st, 0.0}};
    const double sv = sqrt(vol[s]);
    const int nm = (Nmax + 1) * (Nmax + 1) - 1;
    int ind = 0;
    for (int n = 1; n <= Nmax; ++n) {
        const double alpha = sj[n];
        const double beta = sqrt((double)(n * (n + 1))) / kr * sj[n];
        const double gamma = (n + 1.0) / kr * sj[n] - sj[n + 1];
        legendre_col(n, ct, L, scr);
        legendre_col(n + 1, ct, L1, scr);
        legendre_col(n - 1, ct, L2, scr);
        const double q = sqrt(n * (n + 1.0)) / ((n * 2.0 + 1.0) * st);
        for (int m = -n; m <= n; ++m, ++ind) {
            const int mm = m < 0 ? -m : m;
            double fr = 1.0;
            for (int i = n - mm + 1; i <= n + mm; ++i) fr *= (double)i;   // (n+mm)!/(n-mm)!
            const double cc = sqrt((2.0 * n + 1.0) / fr / (4.0 * PI));
            double es, ec;
            sincos((double)m * phi, &es, &ec);
            const double Yr = L[mm];
            const double Y1 = L1[mm] * ((n - mm + 1.0) / (n + 1.0));
            const double Y2 = (mm == n) ? 0.0 : L2[mm] * ((double)(n + mm) / (double)n);
            // B = q (0, Y1 - Y2, i m (2n+1)/(n(n+1)) Y); C = (0, B3, -B2); P = (Y, 0, 0)
            const double b2 = q * (Y1 - Y2);                 // times e^{im phi}
            const double b3 = q * (m * (2 * n + 1.0) / (n * (n + 1.0))) * Yr;   // times i e^{im phi}
            const cd e = cmk(ec, es);
            const cd B2 = cscale(e, b2), B3 = cmul(cmk(0.0, b3), e);
            const cd Pv = cscale(e, Yr);
            const cd Mv[3] = {cmk(0, 0), cscale(B3, cc * alpha), cscale(B2, -cc * alpha)};
            const cd Nv[3] = {cscale(Pv, cc * beta), cscale(B2, cc * gamma), cscale(B3, cc * gamma)};
            const bool mcol = ind >= c0 && ind < c0 + cw, ncol = nm + ind >= c0 && nm + ind < c0 + cw;
            for (int d = 0; d < 3; ++d) {
                const cd Mc = cadd(cadd(cscale(Mv[0], H[d][0]), cscale(Mv[1], H[d][1])), cscale(Mv[2], H[d][2]));
                const cd Nc = cadd(cadd(cscale(Nv[0], H[d][0]), cscale(Nv[1], H[d][1])), cscale(Nv[2], H[d][2]));
                if (mcol) mat[(long long)(ind - c0) * ld + 3LL * s + d] = cscale(Mc, sv);
                if (ncol) mat[(long long)(nm + ind - c0) * ld + 3LL * s + d] = cscale(Nc, sv);
            }
        }
    }
}

// ----------------------------------------------------------------- pinv
// pinv (src/possu.f90:395-422) of the 98 x 27 sample matrix by one-sided
// Jacobi SVD: A V = U S, pinv = V S^-1 U^H keeping s > 1e-6.
typedef std::complex<double> zc;
std::vector<zc> pinv_jacobi(int M, int N, const std::vector<zc> &A) {
    std::vector<zc> U = A, V((size_t)N * N, 0.0);   // column j at [M*j]
    for (int j = 0; j < N; ++j) V[(size_t)N * j + j] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < N - 1; ++p)
            for (int q = p + 1; q < N; ++q) {
                double al = 0, be = 0;
                zc ga = 0;
                for (int i = 0; i < M; ++i) {
                    al += std::norm(U[(size_t)M * p + i]);
                    be += std::norm(U[(size_t)M * q + i]);
                    ga += std::conj(U[(size_t)M * p + i]) * U[(size_t)M * q + i];
                }
                const double ag = std::abs(ga);
                if (ag == 0.0 || ag <= 1e-16 * std::sqrt(al * be)) continue;
                off = std::max(off, ag / std::sqrt(al * be));
                const zc ph = ga / ag;
                const double zeta = (be - al) / (2.0 * ag);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = cs * t;
                for (int i = 0; i < M; ++i) {
                    const zc up = U[(size_t)M * p + i], uq = U[(size_t)M * q + i] * std::conj(ph);
                    U[(size_t)M * p + i] = cs * up - sn * uq;
                    U[(size_t)M * q + i] = (sn * up + cs * uq) * ph;
                }
                for (int i = 0; i < N; ++i) {
                    const zc vp = V[(size_t)N * p + i], vq = V[(size_t)N * q + i] * std::conj(ph);
                    V[(size_t)N * p + i] = cs * vp - sn * vq;
                    V[(size_t)N * q + i] = (sn * vp + cs * vq) * ph;
                }
            }
        if (off < 1e-15) break;
    }
    std::vector<zc> out((size_t)N * M, 0.0);   // (N, M) column-major: out[N*i + j]
    const double cut = (double)1e-6f;
    for (int l = 0; l < N; ++l) {
        double s = 0;
        for (int i = 0; i < M; ++i) s += std::norm(U[(size_t)M * l + i]);
        s = std::sqrt(s);
        if (!(s > cut)) continue;
        for (int i = 0; i < M; ++i) {
            const zc cu = std::conj(U[(size_t)M * l + i]) / (s * s);
            for (int j = 0; j < N; ++j) out[(size_t)N * i + j] += V[(size_t)N * l + j] * cu;
        }
    }
    return out;
}

zc host_green(const double *r, const double *p, double k) {
    const double a = r[0] - p[0], b = r[1] - p[1], c = r[2] - p[2];
    const double R = std::sqrt(a * a + b * b + c * c);
    const double d = 4.0 * PI * R;
    return zc(std::cos(k * R) / d, std::sin(k * R) / d);
}

// cube (0-based) of point p (point_in_cube, src/geometry.f90:13-55), -1 outside
int host_point_cube(const scd_ctx *c, const double *p) {
    const double bd = c->d.delta * 2;
    const int Mx = (int)std::floor((p[0] - c->d.min_coord[0]) / bd);
    const int My = (int)std::floor((p[1] - c->d.min_coord[1]) / bd);
    const int Mz = (int)std::floor((p[2] - c->d.min_coord[2]) / bd);
    if (Mx < 0 || My < 0 || Mz < 0 || Mx >= c->ncx || My >= c->ncy || Mz >= c->ncz) return -1;
    return Mx + c->ncx * My + c->ncx * c->ncy * Mz;
}

void tet_vertices(const scd_ctx *c, int t, double out[12]) {
    for (int v = 0; v < 4; ++v) {
        const int id = c->etopol[4LL * t + v] - 1;
        for (int d = 0; d < 3; ++d) out[3 * v + d] = c->coord[3LL * id + d];
    }
}

}  // namespace

// order set from an arbitrary binning (api.cu)
int set_order_from_cubes(scd_ctx *c, const std::vector<int> &cube_of_tet);

int setup_projectors_device(scd_ctx *c) {
    NvtxRange range("projectors build");
    if (!c->have_mesh) return set_error(c, SCD_NOT_READY, "scd_build_projectors needs scd_set_mesh");
    if (!c->have_k) return set_error(c, SCD_NOT_READY, "scd_build_projectors needs scd_set_wavenumber");
    int rc = upload_quadrature(c);
    if (rc) return rc;
    // W from the box of tet 1 (src/projection.f90:74-101)
    const HostQuad &q = hq();
    double tv[12], cp[3];
    tet_vertices(c, 0, tv);
    for (int d = 0; d < 3; ++d) cp[d] = (tv[d] + tv[3 + d] + tv[6 + d] + tv[9 + d]) / 4;
    const int cube = host_point_cube(c, cp);
    if (cube < 0) return set_error(c, SCD_BAD_ARG, "tet 1 lies outside the projection boxes");
    const int bx = cube % c->ncx, by = (cube / c->ncx) % c->ncy, bz = cube / (c->ncx * c->ncy);
    const double bd = c->d.delta * 2;
    double node1[3] = {c->d.min_coord[0] + c->d.delta * (double)(2 * bx), c->d.min_coord[1] + c->d.delta * (double)(2 * by),
                       c->d.min_coord[2] + c->d.delta * (double)(2 * bz)};
    double cpc[3];
    for (int d = 0; d < 3; ++d) cpc[d] = node1[d] + bd / 2.0;
    std::vector<zc> W(98 * 27);
    for (int m = 0; m < 98; ++m) {
        double r[3];
        for (int d = 0; d < 3; ++d) r[d] = 2.0 * bd * q.ps[m][d] + cpc[d];
        for (int u = 0; u < 27; ++u) {
            const double pnx[3] = {c->d.min_coord[0] + c->d.delta * (double)(2 * bx + u % 3),
                                   c->d.min_coord[1] + c->d.delta * (double)(2 * by + (u / 3) % 3),
                                   c->d.min_coord[2] + c->d.delta * (double)(2 * bz + u / 9)};
            W[98 * u + m] = host_green(r, pnx, c->k);
        }
    }
    std::vector<zc> WW = pinv_jacobi(98, 27, W);      // (27, 98): WW[27*m + u]
    std::vector<cd> WWh(27 * 98);
    for (int u = 0; u < 27; ++u)
        for (int m = 0; m < 98; ++m) WWh[u * 98 + m] = cmk(WW[27 * m + u].real(), WW[27 * m + u].imag());
    cd *dWW = nullptr;
    if (cudaMalloc(&dWW, sizeof(cd) * 27 * 98) != cudaSuccess) return set_error(c, SCD_OOM, "WW");
    cudaMemcpyAsync(dWW, WWh.data(), sizeof(cd) * 27 * 98, cudaMemcpyHostToDevice, c->st);
    if (!c->d_P && cudaMalloc(&c->d_P, sizeof(cd) * 4 * 27 * (size_t)c->T) != cudaSuccess) {
        cudaFree(dWW);
        return set_error(c, SCD_OOM, "projectors");
    }
    int *dcube = nullptr, *dslot0 = nullptr;
    const int ntet = c->T / c->nb;
    if (cudaMalloc(&dcube, sizeof(int) * c->T) != cudaSuccess ||
        (c->nb == 4 && cudaMalloc(&dslot0, sizeof(int) * ntet) != cudaSuccess)) {
        cudaFree(dWW);
        cudaFree(dcube);
        return set_error(c, SCD_OOM, "projector tables");
    }
    cudaMemcpyAsync(dcube, c->cube_of_slot.data(), sizeof(int) * c->T, cudaMemcpyHostToDevice, c->st);
    if (c->nb == 4) {
        // linear basis: one warp per tet over its four consecutive pseudo-tet slots
        std::vector<int> slot0(ntet);
        for (int q = 0; q < ntet; ++q) slot0[q] = c->slot_of[4 * q];
        cudaMemcpyAsync(dslot0, slot0.data(), sizeof(int) * ntet, cudaMemcpyHostToDevice, c->st);
        k_projectors_lin<<<ntet, 32, 0, c->st>>>(c->d_tc, c->d_tvol, dcube, dslot0, ntet, c->T, dWW, c->ncx, c->ncy,
                                                  c->d.delta, c->d.min_coord[0], c->d.min_coord[1], c->d.min_coord[2],
                                                  bd, c->k, c->d_P);
    } else {
        k_projectors<<<(c->T + 3) / 4, 128, 0, c->st>>>(c->d_tc, c->d_tvol, dcube, c->T, dWW, c->ncx, c->ncy, c->d.delta,
                                                        c->d.min_coord[0], c->d.min_coord[1], c->d.min_coord[2], bd, c->k,
                                                        c->d_P);
    }
    rc = check_cuda(c, cudaGetLastError(), "projectors launch");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "projectors");
    cudaFree(dWW);
    cudaFree(dcube);
    cudaFree(dslot0);
    if (!rc) c->have_proj = true;
    c->f_ready = false;
    return rc;
}

// tile list from geometry: (c1, c2) with c2 in the 27-neighbourhood of c1,
// c2 >= c1, both non-empty (find_near_cubes, src/geometry.f90:275-326)
int build_tile_layout(scd_ctx *c);

int setup_nearzone_device(scd_ctx *c, int prec) {
    NvtxRange range("near-zone build");
    if (!c->have_mesh) return set_error(c, SCD_NOT_READY, "scd_build_nearzone needs scd_set_mesh");
    if (!c->have_proj) return set_error(c, SCD_NOT_READY, "scd_build_nearzone needs the projectors");
    if (!c->have_k) return set_error(c, SCD_NOT_READY, "scd_build_nearzone needs scd_set_wavenumber");
    if (prec != SCD_STORE_C64 && prec != SCD_STORE_C128) return set_error(c, SCD_BAD_ARG, "storage_prec %d", prec);
    int rc = upload_quadrature(c);
    if (rc) return rc;
    c->have_near = false;
    c->nzm_ready = false;
    c->near_prec = prec;
    if ((rc = build_tile_layout(c))) return rc;
    const size_t esz = prec == SCD_STORE_C64 ? sizeof(cf) : sizeof(cd);
    if (c->d_tdata) { cudaFree(c->d_tdata); c->d_tdata = nullptr; }
    if (cudaMalloc(&c->d_tdata, esz * (size_t)std::max<long long>(c->tile_store, 1)) != cudaSuccess)
        return set_error(c, SCD_OOM, "near-zone tiles (%lld blocks)", c->tile_blocks);
    // padding between the planes of a tile is never written
    if ((rc = check_cuda(c, cudaMemsetAsync(c->d_tdata, 0, esz * (size_t)std::max<long long>(c->tile_store, 1), c->st),
                         "near-zone tiles")))
        return rc;
    int *dperm = c->d_perm;
    NearArgs a;
    a.tiles = c->d_tiles; a.tc = c->d_tc; a.vol = c->d_tvol; a.eps = c->d_eps; a.P = c->d_P; a.perm = dperm;
    a.cube_off = c->d_cube_off; a.T = c->T; a.ncx = c->ncx; a.ncy = c->ncy; a.Nx = c->Nx; a.Ny = c->Ny;
    a.delta = c->d.delta; a.mx = c->d.min_coord[0]; a.my = c->d.min_coord[1]; a.mz = c->d.min_coord[2];
    a.k = c->k; a.data = c->d_tdata; a.c64 = prec == SCD_STORE_C64;
    if (c->nb == 4) {
        // linear basis: 12x12 blocks per tet pair, written as pseudo-tet blocks
        const size_t sh = sizeof(cd) * (27 * 27 + (size_t)2 * c->max_per_group * 108 + (size_t)LIN_WARPS * LIN_WARP_CD);
        if ((rc = check_cuda(c, cudaFuncSetAttribute(k_near_build_lin, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh),
                             "near-zone shared memory")))
            return rc;
        k_near_build_lin<<<c->ntiles, 32 * LIN_WARPS, sh, c->st>>>(a);
    } else {
        const size_t sh = sizeof(cd) * (27 * 27 + (size_t)2 * c->max_per_group * 108);
        if (sh > 48 * 1024) cudaFuncSetAttribute(k_near_build, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
        k_near_build<<<c->ntiles, NEAR_THREADS, sh, c->st>>>(a);
    }
    rc = check_cuda(c, cudaGetLastError(), "near-zone launch");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "near-zone build");
    if (!rc) { c->have_near = true; c->nrhs_cap = 0; c->f_cap = 0; }
    return rc;
}

int setup_vswf(scd_ctx *c, int Nmax, cd *d_mat, int c0, int cw) {
    NvtxRange range("VSWF columns");
    if (!c->have_mesh) return set_error(c, SCD_NOT_READY, "VSWF right-hand sides need scd_set_mesh");
    if (!c->have_k) return set_error(c, SCD_NOT_READY, "VSWF right-hand sides need scd_set_wavenumber");
    if (Nmax < 1 || Nmax > VSWF_NMAX - 2) return set_error(c, SCD_BAD_ARG, "Nmax %d outside 1..%d", Nmax, VSWF_NMAX - 2);
    const int ntot = 2 * ((Nmax + 1) * (Nmax + 1) - 1);
    if (cw < 0) { c0 = 0; cw = ntot; }
    if (c0 < 0 || cw < 1 || c0 + cw > ntot) return set_error(c, SCD_BAD_ARG, "VSWF columns %d..%d outside 1..%d", c0 + 1, c0 + cw, ntot);
    k_vswf<<<(c->T + 127) / 128, 128, 0, c->st>>>(c->d_tc, c->d_tvol, c->T, c->k, Nmax, d_mat, c->n, c0, cw);
    return check_cuda(c, cudaGetLastError(), "vswf");
}

// 12x12 blocks V(4c + n, 4c' + n') of the linear basis, ordered by (tet_T,
// tet_B), from the pseudo-tet tiles: pseudo-block (n, n') of the tet pair is
// stored at (row slot, column slot) of its tile, or transposed at the mirrored
// position when the test tet's group is the tile's column group
static int export_linear_blocks(scd_ctx *c, int64_t B, const std::vector<cd> &data, scd_c128 *sp, int32_t *ind) {
    struct E { int t, b; const NearTile *tl; int pt, pb; bool swap; };
    std::vector<E> list;
    list.reserve((size_t)B);
    for (const NearTile &tl : c->tiles_h) {
        const int nt1 = tl.n1 / 4, nt2 = tl.n2 / 4;
        for (int p = 0; p < nt1; ++p)
            for (int q = 0; q < nt2; ++q) {
                if (tl.g1 == tl.g2 && q < p) continue;
                const int ta = c->perm[tl.s1 + 4 * p] / 4, tb = c->perm[tl.s2 + 4 * q] / 4;
                if (ta <= tb) list.push_back(E{ta, tb, &tl, p, q, false});
                else list.push_back(E{tb, ta, &tl, p, q, true});
            }
    }
    if ((int64_t)list.size() != B) return set_error(c, SCD_BAD_ARG, "B = %lld, the near zone has %zu tet pairs", (long long)B, list.size());
    std::sort(list.begin(), list.end(), [](const E &x, const E &y) { return x.t != y.t ? x.t < y.t : x.b < y.b; });
    for (size_t k = 0; k < list.size(); ++k) {
        const E &e = list[k];
        const NearTile &tl = *e.tl;
        for (int col = 0; col < 12; ++col)
            for (int row = 0; row < 12; ++row) {
                // the first position the kernel wrote the entry to
                int pp[6];
                lin_tile_positions(tl.g1 == tl.g2, !e.swap, e.pt, e.pb, row + 12 * col, pp);
                const cd v = data[(size_t)tl.data_off + (size_t)tile_at(tl.n1, pp[0], pp[1], pp[2])];
                sp[144 * k + row + 12 * col] = scd_c128{v.x, v.y};
            }
        ind[2 * k] = e.t + 1;
        ind[2 * k + 1] = e.b + 1;
    }
    return SCD_OK;
}

extern "C" {

int scd_grid_from_mesh(int32_t Nv, const double *coord, int32_t T, const int32_t *etopol, double grid_size,
                       int32_t M_ex, scd_grid_desc *d) {
    if (!coord || !etopol || !d || Nv < 4 || T < 1 || M_ex != 2 || !(grid_size > 0)) return SCD_BAD_ARG;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int v = 0; v < Nv; ++v)
        for (int q = 0; q < 3; ++q) {
            mn[q] = std::min(mn[q], coord[3LL * v + q]);
            mx[q] = std::max(mx[q], coord[3LL * v + q]);
        }
    double vol = 0.0;
    for (int t = 0; t < T; ++t) {
        double p[4][3];
        for (int v = 0; v < 4; ++v) {
            const int id = etopol[4LL * t + v] - 1;
            if (id < 0 || id >= Nv) return SCD_BAD_ARG;
            for (int q = 0; q < 3; ++q) p[v][q] = coord[3LL * id + q];
        }
        const V3 tv[4] = {V3{p[0][0], p[0][1], p[0][2]}, V3{p[1][0], p[1][1], p[1][2]}, V3{p[2][0], p[2][1], p[2][2]},
                          V3{p[3][0], p[3][1], p[3][2]}};
        vol += tet_vol(tv);
    }
    const double delta = grid_size * 1.0 / M_ex * std::pow(vol / (double)T, F13_D);
    int N[3];
    for (int q = 0; q < 3; ++q) {
        N[q] = (int)std::ceil(std::fabs(mx[q] - mn[q]) / delta) + 1;
        N[q] = N[q] + ((N[q] + 1) % 2) + 1;
    }
    std::memset(d, 0, sizeof *d);
    d->Nx = N[0]; d->Ny = N[1]; d->Nz = N[2];
    d->delta = delta;
    for (int q = 0; q < 3; ++q) d->min_coord[q] = mn[q];
    d->T = T; d->order = 0; d->M_ex = 2; d->near_zone = 1; d->device = 0;
    return SCD_OK;
}

int scd_set_mesh(scd_ctx *c, int32_t Nv, const double *coord, const int32_t *etopol, const scd_c128 *param) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (!coord || !etopol || !param || Nv < 4) return set_error(c, SCD_BAD_ARG, "bad mesh arrays");
    // with the linear basis every tet holds nb = 4 basis functions (pseudo-tets
    // 4t..4t+3, consecutive slots of the tet's box) that share its geometry
    const int ntet = c->T / c->nb;
    c->Nv = Nv;
    c->coord.assign(coord, coord + 3LL * Nv);
    c->etopol.assign(etopol, etopol + 4LL * ntet);
    c->param.resize(ntet);
    for (int t = 0; t < ntet; ++t) c->param[t] = cmk(param[t].re, param[t].im);
    std::vector<int> cube(c->T);
    for (int t = 0; t < ntet; ++t) {
        for (int v = 0; v < 4; ++v) {
            const int id = etopol[4LL * t + v];
            if (id < 1 || id > Nv) return set_error(c, SCD_BAD_ARG, "etopol(%d,%d) = %d outside 1..%d", v + 1, t + 1, id, Nv);
        }
        double tv[12], cp[3];
        tet_vertices(c, t, tv);
        for (int d = 0; d < 3; ++d) cp[d] = (tv[d] + tv[3 + d] + tv[6 + d] + tv[9 + d]) / 4;
        const int cb = host_point_cube(c, cp);
        if (cb < 0) return set_error(c, SCD_BAD_ARG, "tet %d lies outside the projection boxes", t + 1);
        for (int i = 0; i < c->nb; ++i) cube[c->nb * t + i] = cb;
    }
    int rc = set_order_from_cubes(c, cube);
    if (rc) return rc;
    std::vector<double> tc(12LL * c->T), vol(c->T);
    std::vector<cd> eps(c->T);
    for (int s = 0; s < c->T; ++s) {
        const int t = c->perm[s] / c->nb;
        tet_vertices(c, t, &tc[12LL * s]);
        const double *p = &tc[12LL * s];
        const V3 tv[4] = {V3{p[0], p[1], p[2]}, V3{p[3], p[4], p[5]}, V3{p[6], p[7], p[8]}, V3{p[9], p[10], p[11]}};
        vol[s] = tet_vol(tv);
        eps[s] = c->param[t];
    }
    cudaFree(c->d_tc); cudaFree(c->d_tvol); cudaFree(c->d_eps);
    c->d_tc = nullptr; c->d_tvol = nullptr; c->d_eps = nullptr;
    if (cudaMalloc(&c->d_tc, sizeof(double) * tc.size()) != cudaSuccess ||
        cudaMalloc(&c->d_tvol, sizeof(double) * vol.size()) != cudaSuccess ||
        cudaMalloc(&c->d_eps, sizeof(cd) * eps.size()) != cudaSuccess)
        return set_error(c, SCD_OOM, "mesh arrays");
    cudaMemcpyAsync(c->d_tc, tc.data(), sizeof(double) * tc.size(), cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->d_tvol, vol.data(), sizeof(double) * vol.size(), cudaMemcpyHostToDevice, c->st);
    cudaMemcpyAsync(c->d_eps, eps.data(), sizeof(cd) * eps.size(), cudaMemcpyHostToDevice, c->st);
    c->have_mesh = true;
    return check_cuda(c, cudaGetLastError(), "set_mesh");
}

int scd_build_projectors(scd_ctx *c) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    return setup_projectors_device(c);
}

int scd_build_nearzone(scd_ctx *c, int32_t prec) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    return setup_nearzone_device(c, prec);
}

int scd_get_projectors(scd_ctx *c, scd_c128 *S, scd_c128 *Sx, scd_c128 *Sy, scd_c128 *Sz, int32_t *indS) {
    if (!c) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (!c->have_proj) return set_error(c, SCD_NOT_READY, "projectors not set");
    const size_t TT = 27 * (size_t)c->T;
    std::vector<cd> h(4 * TT);
    int rc = check_cuda(c, cudaMemcpyAsync(h.data(), c->d_P, sizeof(cd) * h.size(), cudaMemcpyDeviceToHost, c->st), "get_projectors");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "get_projectors");
    if (rc) return rc;
    scd_c128 *dst[4] = {S, Sx, Sy, Sz};
    for (int s = 0; s < c->T; ++s) {
        const int t = c->perm[s];
        const int cube = c->cube_of_slot[s];
        const int bx = cube % c->ncx, by = (cube / c->ncx) % c->ncy, bz = cube / (c->ncx * c->ncy);
        for (int j = 0; j < 27; ++j) {
            for (int g = 0; g < 4; ++g)
                if (dst[g]) {
                    const cd v = h[(size_t)(g * 27 + j) * c->T + s];
                    dst[g][27LL * t + j] = scd_c128{v.x, v.y};
                }
            if (indS) {
                const long long node = ((long long)(2 * bz + j / 9) * c->Ny + (2 * by + (j / 3) % 3)) * c->Nx + (2 * bx + j % 3);
                indS[27LL * t + j] = (int32_t)(node + 1);
            }
        }
    }
    return SCD_OK;
}

int64_t scd_nearzone_count(scd_ctx *c) {
    if (!c || !c->have_near) return -1;
    // blocks between basis functions (nb = 1) or between tets (nb = 4: 12x12)
    long long B = 0;
    for (const NearTile &tl : c->tiles_h) {
        const long long n1 = tl.n1 / c->nb, n2 = tl.n2 / c->nb;
        if (tl.g1 == tl.g2) B += n1 * (n1 + 1) / 2;
        else B += n1 * n2;
    }
    return B;
}

// export in the reference layout, ordered by (tet_T, tet_B), widened to FP64
int scd_get_nearzone(scd_ctx *c, int64_t B, scd_c128 *sp, int32_t *ind) {
    if (!c || !sp || !ind) return SCD_BAD_ARG;
    cudaSetDevice(c->dev);
    if (!c->have_near) return set_error(c, SCD_NOT_READY, "near zone not set");
    if (B != scd_nearzone_count(c)) return set_error(c, SCD_BAD_ARG, "B = %lld, the near zone has %lld", (long long)B,
                                                   (long long)scd_nearzone_count(c));
    const size_t nb = (size_t)c->tile_store;
    std::vector<cd> data(nb);
    if (c->near_prec == SCD_STORE_C64) {
        std::vector<cf> f(nb);
        int rc = check_cuda(c, cudaMemcpyAsync(f.data(), c->d_tdata, sizeof(cf) * nb, cudaMemcpyDeviceToHost, c->st), "get_nearzone");
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "get_nearzone");
        if (rc) return rc;
        for (size_t i = 0; i < nb; ++i) data[i] = cmk(f[i].x, f[i].y);
    } else {
        int rc = check_cuda(c, cudaMemcpyAsync(data.data(), c->d_tdata, sizeof(cd) * nb, cudaMemcpyDeviceToHost, c->st), "get_nearzone");
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "get_nearzone");
        if (rc) return rc;
    }
    if (c->nb == 4) return export_linear_blocks(c, B, data, sp, ind);
    struct E { int t, b; size_t e; int ld; bool tr; };
    std::vector<E> list;
    list.reserve((size_t)B);
    for (const NearTile &tl : c->tiles_h) {
        for (int i = 0; i < tl.n1; ++i)
            for (int j = 0; j < tl.n2; ++j) {
                if (tl.g1 == tl.g2 && j < i) continue;
                const int ta = c->perm[tl.s1 + i], tb = c->perm[tl.s2 + j];
                const size_t e = (size_t)tl.data_off + (size_t)tile_at(tl.n1, i, j, 0);
                if (ta <= tb) list.push_back(E{ta, tb, e, tl.n1 | 1, false});
                else list.push_back(E{tb, ta, e, tl.n1 | 1, true});
            }
    }
    std::sort(list.begin(), list.end(), [](const E &x, const E &y) { return x.t != y.t ? x.t < y.t : x.b < y.b; });
    for (size_t q = 0; q < list.size(); ++q) {
        const cd *src = &data[list[q].e];
        const size_t ld = (size_t)list[q].ld;
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) {
                const cd v = list[q].tr ? src[(cc + 3 * r) * ld] : src[(r + 3 * cc) * ld];
                sp[9 * q + r + 3 * cc] = scd_c128{v.x, v.y};
            }
        ind[2 * q] = list[q].t + 1;
        ind[2 * q + 1] = list[q].b + 1;
    }
    return SCD_OK;
}

int scd_vswf_rhs(scd_ctx *c, int32_t Nmax, scd_c128 *mat) {
    if (!c || !mat) return SCD_BAD_ARG;
    if (c->nb != 1) return set_error(c, SCD_BAD_ARG, "scd_vswf_rhs: constant basis only");
    cudaSetDevice(c->dev);
    const int nm = (Nmax + 1) * (Nmax + 1) - 1;
    cd *d = nullptr;
    if (cudaMalloc(&d, sizeof(cd) * (size_t)c->n * 2 * nm) != cudaSuccess) return set_error(c, SCD_OOM, "vswf mat");
    int rc = setup_vswf(c, Nmax, d);
    if (!rc) {
        int r2 = ensure_work(c, 1);
        if (r2) { cudaFree(d); return r2; }
        for (int col = 0; col < 2 * nm && !rc; ++col) {
            launch_permute_out(c, d + (size_t)col * c->n, c->d_io, 1, c->n);
            rc = check_cuda(c, cudaMemcpyAsync(mat + (size_t)col * c->n, c->d_io, sizeof(cd) * c->n,
                                               cudaMemcpyDeviceToHost, c->st), "vswf copy");
        }
        if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "vswf");
    }
    cudaFree(d);
    return rc;
}

}  // extern "C"
