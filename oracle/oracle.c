/* CPU oracle for the scadyn T-matrix solve path — TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of jherrane/scadyn's Fortran algorithm for the
 * T-matrix solve (pFFT JVIE matvec inside restarted GMRES, plus the
 * per-wavelength setup that produces its operator data).  Each function cites
 * the reference file:line it restates.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load this library, to check results.
 *
 * Parity: UNPINNED by reference golden vectors (the reference ships none and
 * cannot be compiled here).  Cross-checked against an independent numpy/scipy
 * restatement, the Mie series (and convergence to it under mesh
 * refinement), T-matrix reciprocity and the energy balance (see tests/).
 *
 * Floating-point notes that follow the reference's source literally:
 *  - single-precision literals promoted to double: `(x)**(1.0/3.0)` uses the
 *    float value of 1/3 (src/geometry.f90:88, src/singularity_subtraction.f90:140),
 *    `0.001` in the GMRES re-orthogonalisation test (src/gmres_module.f90:251),
 *    `1e-6` in pinv (src/possu.f90:413), `1.1` in msta1/msta2
 *    (src/sfunctions.f90:95,119);
 *  - `cf1 = dcmplx(1.0d0 - 100)` = -99 in cspherebessel (src/sfunctions.f90:45);
 *  - the near-zone blocks are narrowed to complex64 on store
 *    (src/precorrection.f90:251) and widened on use (src/sparse_mat.f90:113,116).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI 3.141592653589793   /* src/common.f90:20 */
static const double F13 = (double)(1.0f / 3.0f);   /* Fortran `1.0/3.0` (default real) */

/* ------------------------------------------------------------------ helpers */
static inline double dot3(const double *a, const double *b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
static inline void sub3(const double *a, const double *b, double *c) { c[0]=a[0]-b[0]; c[1]=a[1]-b[1]; c[2]=a[2]-b[2]; }
/* crossRR, src/common.f90:185-192 */
static inline void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1]*b[2] - a[2]*b[1];
    c[1] = -a[0]*b[2] + a[2]*b[0];
    c[2] = a[0]*b[1] - a[1]*b[0];
}
/* norm(r, rp), src/common.f90:219-225 */
static inline double norm2pt(const double *r, const double *rp) {
    double a = r[0]-rp[0], b = r[1]-rp[1], c = r[2]-rp[2];
    return sqrt(a*a + b*b + c*c);
}
/* Gr, src/common.f90:271-279: exp(ikR)/(4 pi R) */
static inline zc Gr(const double *rf, const double *rp, double k) {
    double R = norm2pt(rf, rp);
    double d = 4.0*PI*R;
    return CMPLX(cos(k*R)/d, sin(k*R)/d);
}
/* tetra_volume, src/common.f90:255-267 */
static double tetra_volume(const double tc[4][3]) {
    double p41[3], p21[3], p31[3], cr[3];
    sub3(tc[3], tc[0], p41); sub3(tc[1], tc[0], p21); sub3(tc[2], tc[0], p31);
    cross3(p21, p31, cr);
    double dt = dot3(p41, cr);
    return sqrt(dt*dt)/6.0;
}
static void tet_coord(const double *coord, const int32_t *etopol, int t, double tc[4][3]) {
    for (int c = 0; c < 4; ++c) {
        int v = etopol[4*t + c] - 1;
        for (int d = 0; d < 3; ++d) tc[c][d] = coord[3*v + d];
    }
}
/* tetra_face, src/common.f90:296-322 (faces opposite vertex 1..4) */
static const int FACE[4][3] = {{1,2,3},{0,3,2},{0,1,3},{0,2,1}};
static void tetra_face(const double tc[4][3], int f, double tri[3][3]) {
    for (int i = 0; i < 3; ++i) for (int d = 0; d < 3; ++d) tri[i][d] = tc[FACE[f][i]][d];
}
/* tri_n_vectors, src/common.f90:326-339 */
static void tri_n_vector(const double tri[3][3], double n[3]) {
    double a1[3], a2[3], c[3];
    sub3(tri[1], tri[0], a1); sub3(tri[2], tri[0], a2);
    cross3(a1, a2, c);
    double len = sqrt(c[0]*c[0] + c[1]*c[1] + c[2]*c[2]);
    for (int d = 0; d < 3; ++d) n[d] = c[d]/len;
}

/* ---------------------------------------------------------- quadrature
 * Published rules at the values the reference tabulates
 * (src/integration_points.f90:126-467):
 *  - tetrahedron, order 1: centroid, weight 1/6;
 *  - tetrahedron, order 5: Keast's 24-point degree-6 rule (three 4-point
 *    orbits [a,b,b,b] and one 12-point orbit [c,c,d,e]);
 *  - triangle, order 1: centroid, weight 1/2;
 *  - triangle, order 5: the 7-point degree-5 rule (Strang-Fix / Dunavant).
 * Points are barycentric (xi, eta, zeta) of the reference element; the order
 * of the points is the reference's.
 */
static double QT5P[24][3], QT5W[24];
static double QR5P[7][2], QR5W[7];
static const double QT1P[1][3] = {{0.25, 0.25, 0.25}};
static const double QT1W[1] = {1.666666666666667e-01};
static const double QR1P[1][2] = {{3.333333333333330e-01, 3.333333333333330e-01}};
static const double QR1W[1] = {0.5};
static int quad_ready = 0;
static void quad_init(void) {
    if (quad_ready) return;
    const double A[3][2] = {{3.561913862225449e-01, 2.146028712591517e-01},
                            {8.779781243961660e-01, 4.067395853461134e-02},
                            {3.298632957317306e-02, 3.223378901422757e-01}};
    const double W4[3] = {6.653791709694644e-03, 1.679535175886776e-03, 9.226196923942397e-03};
    int p = 0;
    for (int o = 0; o < 3; ++o) {
        double a = A[o][0], b = A[o][1];
        const double pts[4][3] = {{a,b,b},{b,b,b},{b,b,a},{b,a,b}};
        for (int i = 0; i < 4; ++i, ++p) { memcpy(QT5P[p], pts[i], sizeof pts[i]); QT5W[p] = W4[o]; }
    }
    const double c = 6.366100187501753e-02, d = 2.696723314583159e-01, e = 6.030056647916491e-01;
    const double p12[12][3] = {{d,c,c},{c,d,c},{c,c,d},{e,c,c},{c,e,c},{c,c,e},
                               {c,d,e},{d,e,c},{e,c,d},{c,e,d},{d,c,e},{e,d,c}};
    for (int i = 0; i < 12; ++i, ++p) { memcpy(QT5P[p], p12[i], sizeof p12[i]); QT5W[p] = 8.035714285714281e-03; }
    const double t0 = 3.333333333333330e-01;
    const double a1 = 5.971587178977000e-02, b1 = 4.701420641051150e-01;
    const double a2 = 7.974269853530870e-01, b2 = 1.012865073234560e-01;
    const double tp[7][2] = {{t0,t0},{a1,b1},{b1,b1},{b1,a1},{a2,b2},{b2,b2},{b2,a2}};
    const double tw[7] = {1.125000000000000e-01, 6.619707639425300e-02, 6.619707639425300e-02,
                          6.619707639425300e-02, 6.296959027241350e-02, 6.296959027241350e-02,
                          6.296959027241350e-02};
    memcpy(QR5P, tp, sizeof tp); memcpy(QR5W, tw, sizeof tw);
    quad_ready = 1;
}
/* linmap_tet, src/common.f90:1354-1377 */
static void linmap_tet(const double tc[4][3], int n, const double (*P0)[3], const double *W0,
                       double (*P)[3], double *W) {
    double vol = tetra_volume(tc);
    for (int i = 0; i < n; ++i) {
        double N1 = 1 - P0[i][0] - P0[i][1] - P0[i][2], N2 = P0[i][0], N3 = P0[i][1], N4 = P0[i][2];
        for (int d = 0; d < 3; ++d)
            P[i][d] = tc[0][d]*N1 + tc[1][d]*N2 + tc[2][d]*N3 + tc[3][d]*N4;
        W[i] = W0[i]*6.0*vol;
    }
}
/* linmap_tri, src/common.f90:1381-1408 */
static void linmap_tri(const double tri[3][3], int n, const double (*P0)[2], const double *W0,
                       double (*P)[3], double *W) {
    double a[3], b[3], ww[3];
    sub3(tri[1], tri[0], a); sub3(tri[2], tri[0], b);
    double aa = a[0]*a[0] + a[1]*a[1] + a[2]*a[2];
    ww[0] = aa*b[0]; ww[1] = aa*b[1]; ww[2] = aa*b[2];
    double ab = a[0]*b[0] + a[1]*b[1] + a[2]*b[2];
    double ww1 = sqrt((ww[0]*b[0] + ww[1]*b[1] + ww[2]*b[2]) - ab*ab);
    for (int i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) P[i][d] = tri[0][d] + a[d]*P0[i][0] + b[d]*P0[i][1];
        W[i] = W0[i]*ww1;
    }
}
/* sample_points_cube, src/integration_points.f90:503-805: the 98 surface
 * nodes of the 5x5x5 lattice {-1,-1/2,0,1/2,1}^3, in the reference's order
 * (face z=-1, face z=+1, the y=-1 and y=+1 bands, the x=-1 and x=+1 bands). */
static void sample_points_cube(double P[98][3]) {
    static const double v[5] = {-1.0, -0.5, 0.0, 0.5, 1.0};
    int n = 0;
    for (int iy = 4; iy >= 0; --iy) for (int ix = 0; ix < 5; ++ix) { P[n][0]=v[ix]; P[n][1]=v[iy]; P[n][2]=-1.0; ++n; }
    for (int iy = 0; iy < 5; ++iy) for (int ix = 0; ix < 5; ++ix) { P[n][0]=v[ix]; P[n][1]=v[iy]; P[n][2]= 1.0; ++n; }
    for (int iz = 1; iz <= 3; ++iz) for (int ix = 0; ix < 5; ++ix) { P[n][0]=v[ix]; P[n][1]=-1.0; P[n][2]=v[iz]; ++n; }
    for (int iz = 3; iz >= 1; --iz) for (int ix = 0; ix < 5; ++ix) { P[n][0]=v[ix]; P[n][1]= 1.0; P[n][2]=v[iz]; ++n; }
    for (int iz = 1; iz <= 3; ++iz) for (int iy = 3; iy >= 1; --iy) { P[n][0]=-1.0; P[n][1]=v[iy]; P[n][2]=v[iz]; ++n; }
    for (int iz = 1; iz <= 3; ++iz) for (int iy = 1; iy <= 3; ++iy) { P[n][0]= 1.0; P[n][1]=v[iy]; P[n][2]=v[iz]; ++n; }
}

/* ------------------------------------------------------------- geometry */
void orc_node_coord(const orc_geom *g, int node1, double out[3]) {
    int i = node1 - 1;
    int kx = i % g->Nx, ly = (i / g->Nx) % g->Ny, mz = i / (g->Nx*g->Ny);
    out[0] = g->min_coord[0] + g->delta*(double)kx;   /* src/geometry.f90:112-114 */
    out[1] = g->min_coord[1] + g->delta*(double)ly;
    out[2] = g->min_coord[2] + g->delta*(double)mz;
}

/* point_in_cube, src/geometry.f90:13-55 */
int orc_point_in_cube(const orc_geom *g, const double p[3]) {
    int Mx = (int)floor((p[0] - g->min_coord[0])/g->box_delta);
    int My = (int)floor((p[1] - g->min_coord[1])/g->box_delta);
    int Mz = (int)floor((p[2] - g->min_coord[2])/g->box_delta);
    if (Mx < 0 || My < 0 || Mz < 0 || Mx >= g->Nx_cube || My >= g->Ny_cube || Mz >= g->Nz_cube) return 0;
    return Mx + g->Nx_cube*My + g->Nx_cube*g->Ny_cube*Mz + 1;
}

/* build_grid (src/geometry.f90:60-125), build_box for M_ex = 2
 * (src/geometry.f90:185-219) and tetras_in_cubes (src/geometry.f90:330-377). */
int orc_geom_build(orc_geom *g) {
    if (g->M_ex != 2) return -1;
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int v = 0; v < g->Nv; ++v) for (int d = 0; d < 3; ++d) {
        double c = g->coord[3*v + d];
        if (c < mn[d]) mn[d] = c;
        if (c > mx[d]) mx[d] = c;
    }
    memcpy(g->min_coord, mn, sizeof mn);
    double vol = 0.0, tc[4][3];
    for (int t = 0; t < g->T; ++t) { tet_coord(g->coord, g->etopol, t, tc); vol += tetra_volume(tc); }
    double delta = g->grid_size*1.0/g->M_ex*pow(vol/(double)g->T, F13);
    int N[3];
    for (int d = 0; d < 3; ++d) {
        N[d] = (int)ceil(fabs(mx[d] - mn[d])/delta) + 1;
        N[d] = N[d] + ((N[d] + 1) % 2) + 1;           /* M_ex = 1 or 2: make even */
    }
    g->Nx = N[0]; g->Ny = N[1]; g->Nz = N[2];
    g->delta = delta;
    const int M = 2, Nx = g->Nx, Ny = g->Ny;
    g->Nx_cube = (g->Nx - 2)/M; g->Ny_cube = (g->Ny - 2)/M; g->Nz_cube = (g->Nz - 2)/M;
    g->N_cubes = g->Nx_cube*g->Ny_cube*g->Nz_cube;
    g->box_delta = delta*M;
    g->etopol_box = (int32_t *)malloc(sizeof(int32_t)*27*(size_t)g->N_cubes);
    for (int z = 0; z < g->Nz_cube; ++z) for (int y = 0; y < g->Ny_cube; ++y) for (int x = 0; x < g->Nx_cube; ++x) {
        int c = x + g->Nx_cube*(y + g->Ny_cube*z);
        int first = 1 + 2*x + 2*y*Nx + 2*z*Nx*Ny;
        for (int cz = 0; cz < 3; ++cz) for (int by = 0; by < 3; ++by) for (int ax = 0; ax < 3; ++ax)
            g->etopol_box[27*c + ax + 3*by + 9*cz] = first + ax + by*Nx + cz*Nx*Ny;
    }
    /* tetras_in_cubes */
    int *cube_of = (int *)malloc(sizeof(int)*(size_t)g->T);
    int *cnt = (int *)calloc((size_t)g->N_cubes, sizeof(int));
    for (int t = 0; t < g->T; ++t) {
        tet_coord(g->coord, g->etopol, t, tc);
        double cp[3];
        for (int d = 0; d < 3; ++d) cp[d] = (tc[0][d] + tc[1][d] + tc[2][d] + tc[3][d])/4;
        int c = orc_point_in_cube(g, cp);
        if (c == 0) { free(cube_of); free(cnt); return -2; }
        cube_of[t] = c - 1;
        cnt[c - 1]++;
    }
    int mxc = 0;
    for (int c = 0; c < g->N_cubes; ++c) if (cnt[c] > mxc) mxc = cnt[c];
    g->N_tet_cube = mxc;
    g->tetras = (int32_t *)calloc((size_t)mxc*(size_t)g->N_cubes, sizeof(int32_t));
    memset(cnt, 0, sizeof(int)*(size_t)g->N_cubes);
    for (int t = 0; t < g->T; ++t) {
        int c = cube_of[t];
        g->tetras[(size_t)mxc*c + cnt[c]] = t + 1;
        cnt[c]++;
    }
    free(cube_of); free(cnt);
    return 0;
}

void orc_geom_free(orc_geom *g) {
    free(g->etopol_box); g->etopol_box = NULL;
    free(g->tetras); g->tetras = NULL;
}

/* find_near_cubes, src/geometry.f90:275-326 */
int orc_find_near_cubes(const orc_geom *g, int cube, int32_t *out) {
    int M = 2*g->near_zone + 1, pM = g->near_zone + 1;
    int Mx = g->Nx_cube, My = g->Ny_cube, Mz = g->Nz_cube;
    for (int i = 0; i < M*M*M; ++i) out[i] = 0;
    int z = (cube - 1)/(Mx*My) + 1;
    int y = (cube - (z - 1)*Mx*My - 1)/Mx + 1;
    int x = (cube - (z - 1)*Mx*My - (y - 1)*Mx - 1) + 1;
    int las = 0;
    for (int i1 = 1; i1 <= M; ++i1) {
        int zz = z - pM + i1;
        if (zz > 0 && zz < Mz + 1)
            for (int i2 = 1; i2 <= M; ++i2) {
                int yy = y - pM + i2;
                if (yy > 0 && yy < My + 1)
                    for (int i3 = 1; i3 <= M; ++i3) {
                        int xx = x - pM + i3;
                        if (xx > 0 && xx < Mx + 1) out[las++] = xx + Mx*(yy - 1) + Mx*My*(zz - 1);
                    }
            }
    }
    return las;
}

/* ---------------------------------------------------------------- pinv */
/* One-sided (Hestenes) Jacobi SVD of a complex M x N matrix (M >= N), then
 * pinv = V diag(1/s) U^H keeping s > 1e-6 (src/possu.f90:395-422; the
 * reference calls LAPACK ZGESVD, whose exact rounding is not reproduced). */
int orc_pinv(int M, int N, const zc *A, zc *Ainv) {
    if (M < N) return -1;
    zc *U = (zc *)malloc(sizeof(zc)*(size_t)M*N);
    zc *V = (zc *)calloc((size_t)N*N, sizeof(zc));
    memcpy(U, A, sizeof(zc)*(size_t)M*N);              /* column j at U[M*j] */
    for (int j = 0; j < N; ++j) V[N*j + j] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < N - 1; ++p) for (int q = p + 1; q < N; ++q) {
            double al = 0, be = 0; zc ga = 0;
            for (int i = 0; i < M; ++i) {
                zc up = U[M*p + i], uq = U[M*q + i];
                al += creal(up)*creal(up) + cimag(up)*cimag(up);
                be += creal(uq)*creal(uq) + cimag(uq)*cimag(uq);
                ga += conj(up)*uq;
            }
            double ag = cabs(ga);
            if (ag == 0.0 || ag <= 1e-16*sqrt(al*be)) continue;
            double r = ag/sqrt(al*be); if (r > off) off = r;
            zc ph = ga/ag;                                  /* e^{i phi} */
            double zeta = (be - al)/(2.0*ag);
            double t = (zeta >= 0 ? 1.0 : -1.0)/(fabs(zeta) + sqrt(1.0 + zeta*zeta));
            double c = 1.0/sqrt(1.0 + t*t), s = c*t;
            for (int i = 0; i < M; ++i) {
                zc up = U[M*p + i], uq = U[M*q + i]*conj(ph);
                U[M*p + i] = c*up - s*uq;
                U[M*q + i] = (s*up + c*uq)*ph;
            }
            for (int i = 0; i < N; ++i) {
                zc vp = V[N*p + i], vq = V[N*q + i]*conj(ph);
                V[N*p + i] = c*vp - s*vq;
                V[N*q + i] = (s*vp + c*vq)*ph;
            }
        }
        if (off < 1e-15) break;
    }
    const double cut = (double)1e-6f;
    for (int i = 0; i < N*M; ++i) Ainv[i] = 0;
    for (int l = 0; l < N; ++l) {
        double s = 0; for (int i = 0; i < M; ++i) s += creal(U[M*l+i])*creal(U[M*l+i]) + cimag(U[M*l+i])*cimag(U[M*l+i]);
        s = sqrt(s);
        if (!(s > cut)) continue;
        /* u_l = U[:,l]/s;  Ainv(j,i) += V(j,l) * conj(u_l(i)) / s */
        for (int i = 0; i < M; ++i) {
            zc cu = conj(U[M*l + i])/(s*s);
            for (int j = 0; j < N; ++j) Ainv[(size_t)N*i + j] += V[N*l + j]*cu;
        }
    }
    free(U); free(V);
    return 0;
}

/* ----------------------------------------------------------- projection */
/* pfft_projection_const, src/projection.f90:17-166 (M_ex = 2: 27 box nodes,
 * 98 sample points, 1-point tet and triangle rules). */
int orc_pfft_projection_const(const orc_geom *g, zc *S, zc *Sx, zc *Sy, zc *Sz, int32_t *indS) {
    quad_init();
    double P0[98][3], Ps[98][3];
    sample_points_cube(P0);
    for (int m = 0; m < 98; ++m) for (int d = 0; d < 3; ++d) Ps[m][d] = 2.0*g->box_delta*P0[m][d];
    const double k = g->k;
    double tc[4][3], Pb[1][3], wb[1], cp[3], node1[3], cpc[3];
    /* W from the cube of tet 1 (src/projection.f90:74-101) */
    tet_coord(g->coord, g->etopol, 0, tc);
    for (int d = 0; d < 3; ++d) cp[d] = (tc[0][d] + tc[1][d] + tc[2][d] + tc[3][d])/4;
    int cube = orc_point_in_cube(g, cp);
    if (cube == 0) return -2;
    const int32_t *bn = g->etopol_box + 27*(cube - 1);
    orc_node_coord(g, bn[0], node1);
    for (int d = 0; d < 3; ++d) cpc[d] = node1[d] + g->box_delta/2.0;
    zc *W = (zc *)malloc(sizeof(zc)*98*27), *WW = (zc *)malloc(sizeof(zc)*27*98);
    for (int m = 0; m < 98; ++m) {
        double r[3] = {Ps[m][0] + cpc[0], Ps[m][1] + cpc[1], Ps[m][2] + cpc[2]};
        for (int u = 0; u < 27; ++u) { double pn[3]; orc_node_coord(g, bn[u], pn); W[98*u + m] = Gr(r, pn, k); }
    }
    orc_pinv(98, 27, W, WW);
    zc Q[98], Qx[98], Qy[98], Qz[98];
    for (int t = 0; t < g->T; ++t) {
        tet_coord(g->coord, g->etopol, t, tc);
        double volB = tetra_volume(tc);
        linmap_tet(tc, 1, QT1P, QT1W, Pb, wb);
        for (int d = 0; d < 3; ++d) cp[d] = (tc[0][d] + tc[1][d] + tc[2][d] + tc[3][d])/4;
        cube = orc_point_in_cube(g, cp);
        if (cube == 0) { free(W); free(WW); return -2; }
        bn = g->etopol_box + 27*(cube - 1);
        orc_node_coord(g, bn[0], node1);
        for (int d = 0; d < 3; ++d) cpc[d] = node1[d] + g->box_delta/2.0;
        for (int m = 0; m < 98; ++m) {
            double r[3] = {Ps[m][0] + cpc[0], Ps[m][1] + cpc[1], Ps[m][2] + cpc[2]};
            Q[m] = Gr(r, Pb[0], k)*wb[0];
            Qx[m] = Qy[m] = Qz[m] = 0;
            for (int f = 0; f < 4; ++f) {
                double tri[3][3], n[3], Pt[1][3], wt[1];
                tetra_face(tc, f, tri);
                linmap_tri(tri, 1, QR1P, QR1W, Pt, wt);
                tri_n_vector(tri, n);
                zc Q2 = wt[0]*Gr(r, Pt[0], k);
                Qx[m] += n[0]*Q2; Qy[m] += n[1]*Q2; Qz[m] += n[2]*Q2;
            }
        }
        double sv = sqrt(volB);
        for (int u = 0; u < 27; ++u) {
            zc s0 = 0, s1 = 0, s2 = 0, s3 = 0;
            for (int m = 0; m < 98; ++m) {
                zc w = WW[27*m + u];
                s0 += w*Q[m]; s1 += w*Qx[m]; s2 += w*Qy[m]; s3 += w*Qz[m];
            }
            S[27*t + u] = s0/sv; Sx[27*t + u] = s1/sv; Sy[27*t + u] = s2/sv; Sz[27*t + u] = s3/sv;
            indS[27*t + u] = bn[u];
        }
    }
    free(W); free(WW);
    return 0;
}

/* ------------------------------------------------- singularity subtraction */
#define NP 2
/* analytical_integration, src/singularity_subtraction.f90:15-108 */
static void analytical_integration(const double tri[3][3], const double n[3], const double r[3], double out[NP]) {
    static const int ind[7] = {3, 1, 2, 3, 1, 2, 3};
    double Kl[NP + 1] = {0}, tl[3] = {0}, Il[3] = {0};
    double rmp1[3]; sub3(r, tri[0], rmp1);
    double w0 = dot3(rmp1, n);
    int nn = 0;
    for (int m = 0; m <= NP; ++m) {
        int nexp = 2*m - 1;
        for (int l = 1; l <= 3; ++l) {
            int l2 = ind[l + 2] - 1, l1 = ind[l + 1] - 1, lm1 = ind[l - 1] - 1;
            double slv[3], sl[3], ml[3], pl1mr[3], pl2mpl1[3], rmplm1[3];
            sub3(tri[l2], tri[l1], slv);
            double normslv = sqrt(dot3(slv, slv));
            for (int d = 0; d < 3; ++d) sl[d] = slv[d]/normslv;
            cross3(sl, n, ml);
            sub3(tri[l1], r, pl1mr);
            double tl0 = dot3(pl1mr, ml);
            sub3(tri[l2], tri[l1], pl2mpl1);
            double ll = sqrt(dot3(pl2mpl1, pl2mpl1));
            double sml = dot3(pl1mr, sl), spl = sml + ll;
            sub3(r, tri[lm1], rmplm1);
            double Rpl = sqrt(dot3(rmplm1, rmplm1)), Rml = sqrt(dot3(pl1mr, pl1mr));
            double R0l = sqrt(tl0*tl0 + w0*w0);
            if (nexp == -1) {
                double Km3;
                tl[l - 1] = tl0;
                if (fabs(w0) > 1.0e-10) {
                    double Bl = atan((tl0*spl)/(R0l*R0l + fabs(w0)*Rpl)) - atan((tl0*sml)/(R0l*R0l + fabs(w0)*Rml));
                    Km3 = 1.0/fabs(w0)*Bl;
                } else {
                    Km3 = 0; Il[l - 1] = 0;
                }
                if ((Rml + sml) > (Rpl - spl)) Il[l - 1] = log(fabs((Rpl + spl)/(Rml + sml)));
                else Il[l - 1] = log(fabs((Rml - sml)/(Rpl - spl)));
                Kl[nn] = Kl[nn] + 1/((double)nexp + 2.0)*((double)nexp*w0*w0*Km3 + tl0*Il[l - 1]);
            } else {
                Il[l - 1] = 1/((double)nexp + 1.0)*(spl*pow(Rpl, (double)nexp) - sml*pow(Rml, (double)nexp)
                                                   + (double)nexp*R0l*R0l*Il[l - 1]);
            }
        }
        if (nexp != -1)
            Kl[nn] = 1/((double)nexp + 2.0)*((double)nexp*w0*w0*Kl[nn - 1] + (tl[0]*Il[0] + tl[1]*Il[1] + tl[2]*Il[2]));
        nn++;
    }
    for (int j = 0; j < NP; ++j) out[j] = Kl[j];
}

/* singularity_subtraction_int_V_G, src/singularity_subtraction.f90:112-189 */
static zc int_V_G(const double rf[3], double k, int nb, const double (*Pb)[3], const double *wb, const double B[4][3]) {
    static const double fact[2] = {1.0, -0.5}, ak[2] = {0.5, 0.25};
    zc intR = 0;
    double sw = 0; for (int i = 0; i < nb; ++i) sw += wb[i];
    double cut = 1.0e-10*pow(sw, F13);
    for (int i = 0; i < nb; ++i) {
        double RR = norm2pt(Pb[i], rf);
        zc II;
        if (RR < cut) II = CMPLX(0.0, k/(4.0*PI));
        else {
            double f = 0;
            for (int l = 1; l <= NP; ++l)
                f = f + 1.0/(4*PI)*pow(k, 2.0*(l - 1.0))*fact[l - 1]*pow(RR, 2.0*(l - 1.0) - 1.0);
            II = Gr(rf, Pb[i], k) - f;
        }
        intR = intR + II*wb[i];
    }
    double intR4[NP] = {0};
    for (int f1 = 0; f1 < 4; ++f1) {
        double tri[3][3], tn[3], i2[NP], rr2[3];
        tetra_face(B, f1, tri);
        tri_n_vector(tri, tn);
        analytical_integration(tri, tn, rf, i2);
        sub3(tri[0], rf, rr2);
        double a1 = dot3(tn, rr2);
        for (int j = 0; j < NP; ++j) intR4[j] = intR4[j] + a1*i2[j]*ak[j];
    }
    double f2 = 0;
    for (int l2 = 1; l2 <= NP; ++l2) f2 = f2 + 1.0/(4*PI)*pow(k, 2.0*(l2 - 1))*fact[l2 - 1]*intR4[l2 - 1];
    return intR + f2;
}

/* singularity_subtraction_int_S_G, src/singularity_subtraction.f90:193-243 */
static zc int_S_G(const double rf[3], const double tri[3][3], const double tn[3], double k,
                  int nb, const double (*Pb)[3], const double *wb) {
    static const double fact[2] = {1.0, -0.5};
    zc intR = 0;
    double sw = 0; for (int i = 0; i < nb; ++i) sw += wb[i];
    double cut = 1.0e-10*pow(sw, 0.5);
    for (int i = 0; i < nb; ++i) {
        double R = norm2pt(Pb[i], rf);
        zc II;
        if (R < cut) II = CMPLX(0.0, k/(4*PI));
        else {
            double f = 0;
            for (int l = 1; l <= NP; ++l)
                f = f + 1/(4*PI)*pow(k, 2.0*((double)l - 1.0))*fact[l - 1]*pow(R, 2.0*((double)l - 1) - 1);
            II = Gr(rf, Pb[i], k) - f;
        }
        intR = intR + II*wb[i];
    }
    double i2[NP];
    analytical_integration(tri, tn, rf, i2);
    double f2 = 0.0;
    for (int l2 = 1; l2 <= NP; ++l2) f2 = f2 + 1/(4*PI)*pow(k, 2.0*((double)l2 - 1.0))*fact[l2 - 1]*i2[l2 - 1];
    return intR + f2;
}

/* ------------------------------------------------------------ near zone */
/* block count in the assembly loop order (src/sparse_mat.f90:13-60 counts the
 * same set of pairs) */
static int64_t count_cube(const orc_geom *g, int tc1, const int32_t *near, int nnear) {
    const int32_t *tests = g->tetras + (size_t)g->N_tet_cube*(tc1 - 1);
    if (tests[0] == 0) return 0;
    int64_t c = 0;
    for (int i1 = 0; i1 < nnear; ++i1) {
        const int32_t *bases = g->tetras + (size_t)g->N_tet_cube*(near[i1] - 1);
        for (int t1 = 0; t1 < g->N_tet_cube && tests[t1]; ++t1)
            for (int b1 = 0; b1 < g->N_tet_cube && bases[b1]; ++b1)
                if (bases[b1] >= tests[t1]) c++;
    }
    return c;
}

int64_t orc_nearzone_count(const orc_geom *g) {
    int32_t near[125];
    int64_t total = 0;
    for (int c = 1; c <= g->N_cubes; ++c) {
        int nn = orc_find_near_cubes(g, c, near);
        total += count_cube(g, c, near, nn);
    }
    return total;
}

/* compute_near_zone_interactions_const, src/precorrection.f90:131-264, with
 * compute_pG (:21-46), precorrect_const (:50-82), integrate_V_V_G (:729-760)
 * and integrate_dV_dV_G (:764-806).  Blocks are written in the reference's
 * loop order; cubes are distributed over threads with precomputed offsets. */
int orc_nearzone_const(const orc_geom *g, const zc *S, const zc *Sx, const zc *Sy, const zc *Sz,
                       int64_t B, fc *sp32, zc *sp64, int32_t *sp_ind, int nthreads) {
    quad_init();
    const int NC = g->N_cubes;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t)*(size_t)(NC + 1));
    off[0] = 0;
    {
        int32_t near[125];
        for (int c = 1; c <= NC; ++c) {
            int nn = orc_find_near_cubes(g, c, near);
            off[c] = off[c - 1] + count_cube(g, c, near, nn);
        }
    }
    if (off[NC] != B) { free(off); return -3; }
    const double k = g->k;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int tcube = 1; tcube <= NC; ++tcube) {
        const int32_t *tests = g->tetras + (size_t)g->N_tet_cube*(tcube - 1);
        if (tests[0] == 0) continue;
        int32_t near[125];
        int nn = orc_find_near_cubes(g, tcube, near);
        int64_t blok = off[tcube - 1];
        zc G[27*27];
        for (int i1 = 0; i1 < nn; ++i1) {
            int bcube = near[i1];
            const int32_t *bases = g->tetras + (size_t)g->N_tet_cube*(bcube - 1);
            const int32_t *tb = g->etopol_box + 27*(tcube - 1), *bb = g->etopol_box + 27*(bcube - 1);
            /* compute_pG: G(i1,i2) at G[i1 + 27*i2] */
            for (int a = 0; a < 27; ++a) {
                double r[3]; orc_node_coord(g, tb[a], r);
                for (int b = 0; b < 27; ++b) {
                    if (tb[a] != bb[b]) { double rp[3]; orc_node_coord(g, bb[b], rp); G[a + 27*b] = Gr(r, rp, k); }
                    else G[a + 27*b] = 0;
                }
            }
            for (int t1 = 0; t1 < g->N_tet_cube && tests[t1]; ++t1) {
                int tT = tests[t1];
                double Tc[4][3]; tet_coord(g->coord, g->etopol, tT - 1, Tc);
                double volT = tetra_volume(Tc);
                zc ep = g->param[tT - 1];
                for (int b1 = 0; b1 < g->N_tet_cube && bases[b1]; ++b1) {
                    int tB = bases[b1];
                    if (tB < tT) continue;
                    double Bc[4][3]; tet_coord(g->coord, g->etopol, tB - 1, Bc);
                    double volB = tetra_volume(Bc);
                    /* precorrect_const */
                    const zc *ST = S + 27*(size_t)(tT - 1), *SB = S + 27*(size_t)(tB - 1);
                    const zc *PT[3] = {Sx + 27*(size_t)(tT - 1), Sy + 27*(size_t)(tT - 1), Sz + 27*(size_t)(tT - 1)};
                    const zc *PB[3] = {Sx + 27*(size_t)(tB - 1), Sy + 27*(size_t)(tB - 1), Sz + 27*(size_t)(tB - 1)};
                    zc gs[27], gv[3][27];
                    for (int a = 0; a < 27; ++a) {
                        zc s0 = 0, s1 = 0, s2 = 0, s3 = 0;
                        for (int b = 0; b < 27; ++b) {
                            zc gg = G[a + 27*b];
                            s0 += gg*SB[b]; s1 += gg*PB[0][b]; s2 += gg*PB[1][b]; s3 += gg*PB[2][b];
                        }
                        gs[a] = s0; gv[0][a] = s1; gv[1][a] = s2; gv[2][a] = s3;
                    }
                    zc acorr = 0;
                    for (int a = 0; a < 27; ++a) acorr += gs[a]*ST[a];
                    zc corr2[3][3];
                    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) {
                        zc s = 0;
                        for (int a = 0; a < 27; ++a) s += gv[c][a]*PT[r][a];
                        corr2[r][c] = s;
                    }
                    double sv = sqrt(volT*volB);
                    acorr = acorr*sv;
                    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) corr2[r][c] = corr2[r][c]*sv;
                    /* integrate_V_V_G (order-5 tet rules on both) */
                    double Pt[24][3], wt[24], Pb[24][3], wbb[24];
                    linmap_tet(Tc, 24, (const double (*)[3])QT5P, QT5W, Pt, wt);
                    linmap_tet(Bc, 24, (const double (*)[3])QT5P, QT5W, Pb, wbb);
                    zc intVV = 0;
                    for (int i = 0; i < 24; ++i) intVV = intVV + int_V_G(Pt[i], k, 24, (const double (*)[3])Pb, wbb, (const double (*)[3])Bc)*wt[i];
                    /* integrate_dV_dV_G (order-5 triangle rules) */
                    zc alok2[3][3] = {{0}};
                    for (int ft = 0; ft < 4; ++ft) {
                        double Ttri[3][3], Tn[3], Ptt[7][3], wtt[7];
                        tetra_face(Tc, ft, Ttri); tri_n_vector(Ttri, Tn);
                        linmap_tri(Ttri, 7, (const double (*)[2])QR5P, QR5W, Ptt, wtt);
                        for (int fb = 0; fb < 4; ++fb) {
                            double Btri[3][3], Bn[3], Pbt[7][3], wbt[7];
                            tetra_face(Bc, fb, Btri); tri_n_vector(Btri, Bn);
                            linmap_tri(Btri, 7, (const double (*)[2])QR5P, QR5W, Pbt, wbt);
                            for (int i = 0; i < 7; ++i) {
                                zc in = int_S_G(Ptt[i], (const double (*)[3])Btri, Bn, k, 7, (const double (*)[3])Pbt, wbt);
                                for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c)
                                    alok2[r][c] = alok2[r][c] + (Tn[r]*Bn[c])*in*wtt[i];
                            }
                        }
                    }
                    zc blk[3][3];
                    double k2 = k*k, inv = 1.0/sqrt(volB*volT);
                    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) {
                        zc alok = (tT == tB && r == c) ? 1.0/(ep - 1.0) : 0.0;
                        zc alok1 = (r == c) ? intVV : 0.0;
                        zc corr = (r == c) ? acorr : 0.0;
                        blk[r][c] = alok + inv*(-k2*(alok1 - corr) + (alok2[r][c] - corr2[r][c]));
                    }
                    for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) {
                        if (sp32) sp32[9*blok + r + 3*c] = (fc)blk[r][c];
                        if (sp64) sp64[9*blok + r + 3*c] = blk[r][c];
                    }
                    sp_ind[2*blok] = tT; sp_ind[2*blok + 1] = tB;
                    blok++;
                }
            }
        }
        if (blok != off[tcube]) err = -4;
    }
    free(off);
    return err;
}

/* ---------------------------------------------- linear basis (order 1) set-up */
/* gradshape, src/common.f90:454-492: gradients of the four barycentric shape
 * functions, dN[n][d] = dN_n/dx_d (the rot output is not needed here) */
static void gradshape(const double tc[4][3], double dN[4][3]) {
    double J[3][3];   /* J[row d][col e] = tc[e+1][d] - tc[0][d] */
    for (int d = 0; d < 3; ++d) for (int e = 0; e < 3; ++e) J[d][e] = tc[e + 1][d] - tc[0][d];
    const double detJ = J[0][0]*(J[1][1]*J[2][2] - J[1][2]*J[2][1]) - J[0][1]*(J[1][0]*J[2][2] - J[1][2]*J[2][0])
                      + J[0][2]*(J[1][0]*J[2][1] - J[1][1]*J[2][0]);
    double J0[3][3];
    J0[0][0] = J[1][1]*J[2][2] - J[1][2]*J[2][1];
    J0[1][0] = -(J[0][1]*J[2][2] - J[0][2]*J[2][1]);
    J0[2][0] = (J[0][1]*J[1][2] - J[0][2]*J[1][1]);
    J0[0][1] = -(J[1][0]*J[2][2] - J[1][2]*J[2][0]);
    J0[1][1] = (J[0][0]*J[2][2] - J[0][2]*J[2][0]);
    J0[2][1] = -(J[0][0]*J[1][2] - J[0][2]*J[1][0]);
    J0[0][2] = J[1][0]*J[2][1] - J[1][1]*J[2][0];
    J0[1][2] = -(J[0][0]*J[2][1] - J[0][1]*J[2][0]);
    J0[2][2] = (J[0][0]*J[1][1] - J[0][1]*J[1][0]);
    for (int d = 0; d < 3; ++d) {
        dN[1][d] = J0[d][0]/detJ;
        dN[2][d] = J0[d][1]/detJ;
        dN[3][d] = J0[d][2]/detJ;
        dN[0][d] = -dN[1][d] - dN[2][d] - dN[3][d];
    }
}

/* analytical_integration_N, src/singularity_subtraction_N.f90:15-136: for the
 * three shape functions of a triangle (vertex l <-> the edge opposite it) the
 * integrals of N_l R^(2 nm - 3) over the triangle, out[nm-1][l], nm = 1..Np */
#define NPMAX 2
static void analytical_integration_N(const double tri[3][3], const double n[3], const double r[3], int Np,
                                     double out[NPMAX][3]) {
    static const int ind[7] = {3, 1, 2, 3, 1, 2, 3};
    double Kl[NPMAX + 1] = {0}, Il[3] = {0}, tl[3] = {0}, hhl[3] = {0}, mvek[3][3] = {{0}};
    double Inl[NPMAX + 1][3];
    double rmp1[3]; sub3(r, tri[0], rmp1);
    const double w0 = dot3(rmp1, n);
    int nn = 0;
    for (int m = 0; m <= Np; ++m) {
        const int nexp = 2*m - 1;
        for (int l = 1; l <= 3; ++l) {
            const int l2 = ind[l + 2] - 1, l1 = ind[l + 1] - 1, l0 = ind[l] - 1, lm1 = ind[l - 1] - 1;
            double slv[3], sl[3], ml[3], pl1mr[3], pl2mpl1[3], rmplm1[3], pl1mpl0[3];
            sub3(tri[l2], tri[l1], slv);
            const double normslv = sqrt(dot3(slv, slv));
            for (int d = 0; d < 3; ++d) sl[d] = slv[d]/normslv;
            cross3(sl, n, ml);
            sub3(tri[l1], r, pl1mr);
            const double tl0 = dot3(pl1mr, ml);
            sub3(tri[l2], tri[l1], pl2mpl1);
            const double ll = sqrt(dot3(pl2mpl1, pl2mpl1));
            const double sml = dot3(pl1mr, sl), spl = sml + ll;
            sub3(r, tri[lm1], rmplm1);
            const double Rpl = sqrt(dot3(rmplm1, rmplm1)), Rml = sqrt(dot3(pl1mr, pl1mr));
            const double R0l = sqrt(tl0*tl0 + w0*w0);
            sub3(tri[l1], tri[l0], pl1mpl0);
            const double hl = dot3(pl1mpl0, ml);
            if (nexp == -1) {
                for (int d = 0; d < 3; ++d) mvek[l - 1][d] = ml[d];
                tl[l - 1] = tl0;
                hhl[l - 1] = hl;
                double Km3;
                if (fabs(w0) > 1.0e-10) {
                    const double Bl = atan((tl0*spl)/(R0l*R0l + fabs(w0)*Rpl)) - atan((tl0*sml)/(R0l*R0l + fabs(w0)*Rml));
                    Km3 = 1.0/fabs(w0)*Bl;
                } else {
                    Km3 = 0.0;
                    Il[l - 1] = 0.0;
                }
                if (fabs(Rml + sml) > 0.0) Il[l - 1] = log((Rpl + spl)/(Rml + sml));
                else Il[l - 1] = 0.0;
                Kl[nn] = Kl[nn] + 1.0/((double)nexp + 2.0)*((double)nexp*w0*w0*Km3 + tl0*Il[l - 1]);
            } else {
                Il[l - 1] = 1.0/((double)nexp + 1.0)*(spl*pow(Rpl, (double)nexp) - sml*pow(Rml, (double)nexp)
                                                     + (double)nexp*R0l*R0l*Il[l - 1]);
            }
        }
        if (nexp != -1)
            Kl[nn] = 1.0/((double)nexp + 2.0)*((double)nexp*w0*w0*Kl[nn - 1] + (tl[0]*Il[0] + tl[1]*Il[1] + tl[2]*Il[2]));
        for (int l = 0; l < 3; ++l) Inl[nn][l] = Il[l];
        nn++;
    }
    double v1[NPMAX + 1][3];
    for (int i1 = 0; i1 <= Np; ++i1)
        for (int d = 0; d < 3; ++d) v1[i1][d] = Inl[i1][0]*mvek[0][d] + Inl[i1][1]*mvek[1][d] + Inl[i1][2]*mvek[2][d];
    for (int nm = 1; nm <= Np; ++nm)
        for (int l = 0; l < 3; ++l) {
            const double dl = dot3(mvek[l], v1[nm]);
            out[nm - 1][l] = 1.0/hhl[l]*(tl[l]*Kl[nm - 1] - 1.0/(2.0*(double)nm - 1.0)*dl);
        }
}

/* singularity_subtraction_int_V_GN, src/singularity_subtraction_N.f90:140-238:
 * I_j(rf) = int_B G(rf, r') N_j(r') dV' (j = 1..4), 1/R subtracted and
 * integrated analytically (Np = 1); shape[i][j] at the 24 points Pb */
static void int_V_GN(const double rf[3], double k, const double (*Pb)[3], const double *wb, const double B[4][3],
                     const double (*shape)[4], zc out[4]) {
    zc intR[4] = {0, 0, 0, 0};
    double sw = 0; for (int i = 0; i < 24; ++i) sw += wb[i];
    const double cut = 1.0e-10*pow(sw, F13);
    for (int i = 0; i < 24; ++i) {
        const double RR = norm2pt(Pb[i], rf);
        zc II;
        if (RR < cut) II = CMPLX(0.0, k/(4.0*PI));
        else {
            const double f = 1.0/(4*PI)*pow(k, 0.0)*1.0*pow(RR, -1.0);
            II = Gr(rf, Pb[i], k) - f;
        }
        for (int j = 0; j < 4; ++j) intR[j] = intR[j] + II*shape[i][j]*wb[i];
    }
    double intR5[4] = {0}, intR6[4] = {0}, dN[4][3];
    gradshape(B, dN);
    for (int f1 = 0; f1 < 4; ++f1) {
        double tri[3][3], tn[3], i2[NPMAX][3], rr2[3];
        tetra_face(B, f1, tri);
        tri_n_vector(tri, tn);
        analytical_integration_N(tri, tn, rf, 2, i2);
        sub3(tri[0], rf, rr2);
        const double a1 = dot3(tn, rr2);
        for (int l = 0; l < 3; ++l) intR6[FACE[f1][l]] += i2[0][l]*a1*0.5;
        const double s2 = i2[1][0] + i2[1][1] + i2[1][2];
        for (int j = 0; j < 4; ++j) intR5[j] += dot3(tn, dN[j])*s2*0.5*1.0;
    }
    for (int j = 0; j < 4; ++j) out[j] = intR[j] + 1.0/(4*PI)*1.0*1.0*(-intR5[j] + intR6[j]);
}

/* singularity_subtraction_int_S_GN, src/singularity_subtraction_N.f90:242-294:
 * int_tri G(rf, r') N_l(r') dS' for the triangle's three shape functions */
static void int_S_GN(const double rf[3], const double tri[3][3], const double tn[3], double k,
                     const double (*Pb)[3], const double *wb, zc out[3]) {
    zc intR[3] = {0, 0, 0};
    double sw = 0; for (int i = 0; i < 7; ++i) sw += wb[i];
    const double cut = 1.0e-10*pow(sw, 0.5);
    for (int i = 0; i < 7; ++i) {
        const double R = norm2pt(Pb[i], rf);
        zc II;
        if (R < cut) II = CMPLX(0.0, k/(4*PI));
        else II = Gr(rf, Pb[i], k) - 1.0/(4*PI)*pow(k, 0.0)*1.0*pow(R, -1.0);
        const double s[3] = {1.0 - QR5P[i][0] - QR5P[i][1], QR5P[i][0], QR5P[i][1]};
        for (int l = 0; l < 3; ++l) intR[l] = intR[l] + II*wb[i]*s[l];
    }
    double i2[NPMAX][3];
    analytical_integration_N(tri, tn, rf, 1, i2);
    for (int l = 0; l < 3; ++l) out[l] = intR[l] + 1.0/(4*PI)*1.0*1.0*i2[0][l];
}

/* tet shape functions at the 24 order-5 points: shape[i][j] */
static void tet5_shape(double shape[24][4]) {
    for (int i = 0; i < 24; ++i) {
        shape[i][0] = 1 - QT5P[i][0] - QT5P[i][1] - QT5P[i][2];
        shape[i][1] = QT5P[i][0]; shape[i][2] = QT5P[i][1]; shape[i][3] = QT5P[i][2];
    }
}

/* single-point forms of the constant-basis integrals for tests: B (4,3)
 * vertices, tri (3,3); out[0] = int 1/R dS, out[1] = int R dS */
void orc_analytical_integration(const double tri[9], const double r[3], double out[2]) {
    double t[3][3], n[3];
    memcpy(t, tri, sizeof t);
    tri_n_vector(t, n);
    analytical_integration(t, n, r, out);
}
zc orc_int_V_G(const double rf[3], double k, const double B[12]) {
    quad_init();
    double Bc[4][3], Pb[24][3], wb[24];
    memcpy(Bc, B, sizeof Bc);
    linmap_tet(Bc, 24, (const double (*)[3])QT5P, QT5W, Pb, wb);
    return int_V_G(rf, k, 24, (const double (*)[3])Pb, wb, (const double (*)[3])Bc);
}
zc orc_int_S_G(const double rf[3], double k, const double tri[9]) {
    quad_init();
    double t[3][3], n[3], Pb[7][3], wb[7];
    memcpy(t, tri, sizeof t);
    tri_n_vector(t, n);
    linmap_tri(t, 7, (const double (*)[2])QR5P, QR5W, Pb, wb);
    return int_S_G(rf, (const double (*)[3])t, n, k, 7, (const double (*)[3])Pb, wb);
}

/* single-point forms of the above for tests: B (4,3) vertices, tri (3,3) */
void orc_int_V_GN(const double rf[3], double k, const double B[12], zc out[4]) {
    quad_init();
    double Bc[4][3], Pb[24][3], wb[24], shape[24][4];
    memcpy(Bc, B, sizeof Bc);
    linmap_tet(Bc, 24, (const double (*)[3])QT5P, QT5W, Pb, wb);
    tet5_shape(shape);
    int_V_GN(rf, k, (const double (*)[3])Pb, wb, (const double (*)[3])Bc, (const double (*)[4])shape, out);
}
void orc_int_S_GN(const double rf[3], const double tri[9], double k, zc out[3]) {
    quad_init();
    double t[3][3], n[3], Pb[7][3], wb[7];
    memcpy(t, tri, sizeof t);
    tri_n_vector(t, n);
    linmap_tri(t, 7, (const double (*)[2])QR5P, QR5W, Pb, wb);
    int_S_GN(rf, (const double (*)[3])t, n, k, (const double (*)[3])Pb, wb, out);
}
void orc_gradshape(const double tc[12], double dN[12]) {
    double t[4][3], d[4][3];
    memcpy(t, tc, sizeof t);
    gradshape(t, d);
    memcpy(dN, d, sizeof d);
}

/* pfft_projection_lin, src/projection.f90:170-338: four projector columns per
 * tet (node n of tet t in column 4(t-1)+n), order-5 tet and triangle rules.
 * Outputs (27, 4T). */
int orc_pfft_projection_lin(const orc_geom *g, zc *S, zc *Sx, zc *Sy, zc *Sz, int32_t *indS) {
    quad_init();
    double P0[98][3], Ps[98][3], shape[24][4];
    sample_points_cube(P0);
    tet5_shape(shape);
    for (int m = 0; m < 98; ++m) for (int d = 0; d < 3; ++d) Ps[m][d] = 2.0*g->box_delta*P0[m][d];
    const double k = g->k;
    double tc[4][3], cp[3], node1[3], cpc[3];
    tet_coord(g->coord, g->etopol, 0, tc);
    for (int d = 0; d < 3; ++d) cp[d] = (tc[0][d] + tc[1][d] + tc[2][d] + tc[3][d])/4;
    int cube = orc_point_in_cube(g, cp);
    if (cube == 0) return -2;
    const int32_t *bn = g->etopol_box + 27*(cube - 1);
    orc_node_coord(g, bn[0], node1);
    for (int d = 0; d < 3; ++d) cpc[d] = node1[d] + g->box_delta/2.0;
    zc *W = (zc *)malloc(sizeof(zc)*98*27), *WW = (zc *)malloc(sizeof(zc)*27*98);
    for (int m = 0; m < 98; ++m) {
        double r[3] = {Ps[m][0] + cpc[0], Ps[m][1] + cpc[1], Ps[m][2] + cpc[2]};
        for (int u = 0; u < 27; ++u) { double pn[3]; orc_node_coord(g, bn[u], pn); W[98*u + m] = Gr(r, pn, k); }
    }
    orc_pinv(98, 27, W, WW);
    int err = 0;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16)
#endif
    for (int t = 0; t < g->T; ++t) {
        double Bc[4][3], c3[3], n1c[3], cc[3], Pb[24][3], wb[24], dN[4][3];
        tet_coord(g->coord, g->etopol, t, Bc);
        const double volB = tetra_volume(Bc);
        linmap_tet(Bc, 24, (const double (*)[3])QT5P, QT5W, Pb, wb);
        gradshape(Bc, dN);
        for (int d = 0; d < 3; ++d) c3[d] = (Bc[0][d] + Bc[1][d] + Bc[2][d] + Bc[3][d])/4;
        const int cb = orc_point_in_cube(g, c3);
        if (cb == 0) { err = -2; continue; }
        const int32_t *bt = g->etopol_box + 27*(cb - 1);
        orc_node_coord(g, bt[0], n1c);
        for (int d = 0; d < 3; ++d) cc[d] = n1c[d] + g->box_delta/2.0;
        zc Q[98][4], Q2[3][98][4];
        double ftri[4][3][3], fn[4][3], Pt[4][7][3], wt[4][7];
        for (int f = 0; f < 4; ++f) {
            tetra_face(Bc, f, ftri[f]);
            linmap_tri(ftri[f], 7, (const double (*)[2])QR5P, QR5W, Pt[f], wt[f]);
            tri_n_vector(ftri[f], fn[f]);
        }
        for (int m = 0; m < 98; ++m) {
            const double r[3] = {Ps[m][0] + cc[0], Ps[m][1] + cc[1], Ps[m][2] + cc[2]};
            for (int n = 0; n < 4; ++n) { Q[m][n] = 0; Q2[0][m][n] = Q2[1][m][n] = Q2[2][m][n] = 0; }
            for (int i = 0; i < 24; ++i) {
                const zc gg = Gr(r, Pb[i], k);
                for (int n = 0; n < 4; ++n) Q[m][n] = Q[m][n] + shape[i][n]*gg*wb[i];
            }
            for (int f = 0; f < 4; ++f) {
                zc q2[3] = {0, 0, 0};
                for (int i = 0; i < 7; ++i) {
                    const double s[3] = {1.0 - QR5P[i][0] - QR5P[i][1], QR5P[i][0], QR5P[i][1]};
                    const zc gg = Gr(r, Pt[f][i], k);
                    for (int l = 0; l < 3; ++l) q2[l] = q2[l] + s[l]*wt[f][i]*gg;
                }
                for (int l = 0; l < 3; ++l)
                    for (int d = 0; d < 3; ++d) Q2[d][m][FACE[f][l]] += fn[f][d]*q2[l];
            }
        }
        const double sv = sqrt(volB);
        for (int n = 0; n < 4; ++n) {
            const size_t col = 27*(size_t)(4*t + n);
            for (int u = 0; u < 27; ++u) {
                zc s0 = 0, sd[3] = {0, 0, 0}, qd[3] = {0, 0, 0};
                for (int m = 0; m < 98; ++m) {
                    const zc w = WW[27*m + u];
                    const zc qdn = Q[m][0] + Q[m][1] + Q[m][2] + Q[m][3];
                    s0 += w*Q[m][n];
                    for (int d = 0; d < 3; ++d) { sd[d] += w*Q2[d][m][n]; qd[d] += w*(qdn*dN[n][d]); }
                }
                S[col + u] = s0/sv;
                Sx[col + u] = (sd[0] - qd[0])/sv;
                Sy[col + u] = (sd[1] - qd[1])/sv;
                Sz[col + u] = (sd[2] - qd[2])/sv;
                indS[col + u] = bt[u];
            }
        }
    }
    free(W); free(WW);
    return err;
}

/* One 12x12 block of compute_near_zone_interactions_lin
 * (src/precorrection.f90:268-371) for test tet tT <= basis tet tB (1-based),
 * V(4c + n, 4c' + n') column-major in blk[r + 12 q]; G is compute_pG of their
 * boxes (G(i1, i2) at G[i1 + 27 i2]).  Pieces: integrate_NN (:375-405),
 * integrate_V_V_GNN (:409-445), integrate_dV_V_GNN (:449-524),
 * integrate_dV_dV_GNN (:528-617), integrate_V_dV_GNN (:621-685), aloks
 * (:689-717), precorrect_lin (:86-127). */
static void near_block_lin(const orc_geom *g, const zc *S, const zc *Sx, const zc *Sy, const zc *Sz, const zc *G,
                           int tT, int tB, zc blk[144]) {
    const double k = g->k;
    double Tc[4][3], Bc[4][3], dNT[4][3], dNB[4][3], shape[24][4];
    tet_coord(g->coord, g->etopol, tT - 1, Tc);
    tet_coord(g->coord, g->etopol, tB - 1, Bc);
    const double volT = tetra_volume(Tc), volB = tetra_volume(Bc);
    gradshape(Tc, dNT);
    gradshape(Bc, dNB);
    tet5_shape(shape);
    /* precorrect_lin: corr(n_T, n_B) and corr2(4r + n_T, 4c + n_B) */
    zc corr[144], corr2[144];
    for (int q = 0; q < 144; ++q) corr[q] = corr2[q] = 0;
    const zc *PS[4] = {S, Sx, Sy, Sz};
    for (int i1 = 0; i1 < 4; ++i1) {
        zc gv[4][27];
        for (int s = 0; s < 4; ++s) {
            const zc *pb = PS[s] + 27*(size_t)(4*(tB - 1) + i1);
            for (int a = 0; a < 27; ++a) {
                zc acc = 0;
                for (int b = 0; b < 27; ++b) acc += G[a + 27*b]*pb[b];
                gv[s][a] = acc;
            }
        }
        for (int i2 = 0; i2 < 4; ++i2) {
            const size_t colT = 27*(size_t)(4*(tT - 1) + i2);
            zc a0 = 0;
            for (int a = 0; a < 27; ++a) a0 += gv[0][a]*S[colT + a];
            for (int c = 0; c < 3; ++c) corr[(4*c + i2) + 12*(4*c + i1)] = a0;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    zc s = 0;
                    for (int a = 0; a < 27; ++a) s += gv[1 + c][a]*PS[1 + r][colT + a];
                    corr2[(4*r + i2) + 12*(4*c + i1)] = s;
                }
        }
    }
    const double sv = sqrt(volT*volB);
    for (int q = 0; q < 144; ++q) { corr[q] = corr[q]*sv; corr2[q] = corr2[q]*sv; }
    double Pt[24][3], wt[24], Pb[24][3], wb[24];
    linmap_tet(Tc, 24, (const double (*)[3])QT5P, QT5W, Pt, wt);
    linmap_tet(Bc, 24, (const double (*)[3])QT5P, QT5W, Pb, wb);
    /* integrate_NN */
    zc alok[144];
    for (int q = 0; q < 144; ++q) alok[q] = 0;
    if (tT == tB) {
        double intN[4][4] = {{0}};
        for (int i = 0; i < 24; ++i)
            for (int b = 0; b < 4; ++b)
                for (int a = 0; a < 4; ++a) intN[a][b] += shape[i][b]*shape[i][a]*wt[i];
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) alok[(4*c + a) + 12*(4*c + b)] = intN[a][b];
    }
    /* integrate_V_V_GNN: GNN(a, b) */
    zc GNN[4][4] = {{0}};
    for (int i = 0; i < 24; ++i) {
        zc Iv[4];
        int_V_GN(Pt[i], k, (const double (*)[3])Pb, wb, (const double (*)[3])Bc, (const double (*)[4])shape, Iv);
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) GNN[a][b] = GNN[a][b] + Iv[b]*shape[i][a]*wt[i];
    }
    /* faces of both tets with their order-5 points */
    double Ttri[4][3][3], Tn[4][3], Ptt[4][7][3], wtt[4][7];
    double Btri[4][3][3], Bn[4][3], Pbt[4][7][3], wbt[4][7];
    for (int f = 0; f < 4; ++f) {
        tetra_face(Tc, f, Ttri[f]); tri_n_vector(Ttri[f], Tn[f]);
        linmap_tri(Ttri[f], 7, (const double (*)[2])QR5P, QR5W, Ptt[f], wtt[f]);
        tetra_face(Bc, f, Btri[f]); tri_n_vector(Btri[f], Bn[f]);
        linmap_tri(Btri[f], 7, (const double (*)[2])QR5P, QR5W, Pbt[f], wbt[f]);
    }
    /* integrate_dV_V_GNN: alok4(row, 4c + b) = II4(row) dN_B[b][c] */
    zc II4[12];
    for (int q = 0; q < 12; ++q) II4[q] = 0;
    for (int ft = 0; ft < 4; ++ft) {
        zc intN[4] = {0, 0, 0, 0};
        for (int i = 0; i < 7; ++i) {
            zc Iv[4];
            int_V_GN(Ptt[ft][i], k, (const double (*)[3])Pb, wb, (const double (*)[3])Bc, (const double (*)[4])shape, Iv);
            const zc Is = Iv[0] + Iv[1] + Iv[2] + Iv[3];
            const double s[3] = {1.0 - QR5P[i][0] - QR5P[i][1], QR5P[i][0], QR5P[i][1]};
            for (int l = 0; l < 3; ++l) intN[FACE[ft][l]] = intN[FACE[ft][l]] + Is*s[l]*wtt[ft][i];
        }
        for (int r = 0; r < 3; ++r)
            for (int a = 0; a < 4; ++a) II4[4*r + a] = II4[4*r + a] + intN[a]*Tn[ft][r];
    }
    /* J_c(b; rf) = sum over the faces of B of n_c int_face G N_b dS' */
#define JSUM(rf, J)                                                                                   \
    do {                                                                                              \
        for (int q_ = 0; q_ < 12; ++q_) (J)[q_] = 0;                                                  \
        for (int fb_ = 0; fb_ < 4; ++fb_) {                                                           \
            zc in_[3];                                                                                \
            int_S_GN((rf), (const double (*)[3])Btri[fb_], Bn[fb_], k, (const double (*)[3])Pbt[fb_], \
                     wbt[fb_], in_);                                                                  \
            for (int l_ = 0; l_ < 3; ++l_)                                                            \
                for (int c_ = 0; c_ < 3; ++c_)                                                        \
                    (J)[4*c_ + FACE[fb_][l_]] = (J)[4*c_ + FACE[fb_][l_]] + in_[l_]*Bn[fb_][c_];      \
        }                                                                                             \
    } while (0)
    /* integrate_dV_dV_GNN */
    zc alok2[144];
    for (int q = 0; q < 144; ++q) alok2[q] = 0;
    for (int ft = 0; ft < 4; ++ft) {
        zc II[3][4][4];   /* II[c][a][b] */
        memset(II, 0, sizeof II);
        for (int i = 0; i < 7; ++i) {
            zc J[12];
            JSUM(Ptt[ft][i], J);
            const double s[3] = {1.0 - QR5P[i][0] - QR5P[i][1], QR5P[i][0], QR5P[i][1]};
            for (int l = 0; l < 3; ++l)
                for (int c = 0; c < 3; ++c)
                    for (int b = 0; b < 4; ++b)
                        II[c][FACE[ft][l]][b] = II[c][FACE[ft][l]][b] + J[4*c + b]*s[l]*wtt[ft][i];
        }
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c)
                for (int a = 0; a < 4; ++a)
                    for (int b = 0; b < 4; ++b)
                        alok2[(4*r + a) + 12*(4*c + b)] = alok2[(4*r + a) + 12*(4*c + b)] + II[c][a][b]*Tn[ft][r];
    }
    /* integrate_V_dV_GNN: alok5(4r + a, col) = dN_T[a][r] II5(col) */
    zc II5[12];
    for (int q = 0; q < 12; ++q) II5[q] = 0;
    for (int i = 0; i < 24; ++i) {
        zc J[12];
        JSUM(Pt[i], J);
        for (int q = 0; q < 12; ++q) II5[q] = II5[q] + J[q]*wt[i];
    }
#undef JSUM
    /* aloks and the block */
    zc sG = 0;
    for (int b = 0; b < 4; ++b) for (int a = 0; a < 4; ++a) sG += GNN[a][b];
    const zc ep = g->param[tT - 1];
    const double k2 = k*k, inv = 1.0/sqrt(volB*volT);
    for (int c = 0; c < 3; ++c)
        for (int b = 0; b < 4; ++b)
            for (int r = 0; r < 3; ++r)
                for (int a = 0; a < 4; ++a) {
                    const int row = 4*r + a, col = 4*c + b, q = row + 12*col;
                    const zc alok1 = r == c ? GNN[a][b] : 0;
                    const zc alok3 = (dNT[a][r]*dNB[b][c])*sG;
                    const zc alok4 = II4[row]*dNB[b][c];
                    const zc alok5 = dNT[a][r]*II5[col];
                    blk[q] = inv*(alok[q]/(ep - 1.0) + (-k2*(alok1 - corr[q]) + (alok2[q] + alok3 - alok4 - alok5) - corr2[q]));
                }
}

/* compute_near_zone_interactions_lin, src/precorrection.f90:268-371: 12x12
 * blocks sp(12,12,B) for the same tet pairs, in the same order, as the
 * constant-basis assembly. */
int orc_nearzone_lin(const orc_geom *g, const zc *S, const zc *Sx, const zc *Sy, const zc *Sz,
                     int64_t B, fc *sp32, zc *sp64, int32_t *sp_ind, int nthreads) {
    quad_init();
    const int NC = g->N_cubes;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t)*(size_t)(NC + 1));
    off[0] = 0;
    {
        int32_t near[125];
        for (int c = 1; c <= NC; ++c) {
            int nn = orc_find_near_cubes(g, c, near);
            off[c] = off[c - 1] + count_cube(g, c, near, nn);
        }
    }
    if (off[NC] != B) { free(off); return -3; }
    const double k = g->k;
    int err = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int tcube = 1; tcube <= NC; ++tcube) {
        const int32_t *tests = g->tetras + (size_t)g->N_tet_cube*(tcube - 1);
        if (tests[0] == 0) continue;
        int32_t near[125];
        int nn = orc_find_near_cubes(g, tcube, near);
        int64_t blok = off[tcube - 1];
        zc G[27*27];
        for (int i1 = 0; i1 < nn; ++i1) {
            const int bcube = near[i1];
            const int32_t *bases = g->tetras + (size_t)g->N_tet_cube*(bcube - 1);
            const int32_t *tb = g->etopol_box + 27*(tcube - 1), *bb = g->etopol_box + 27*(bcube - 1);
            for (int a = 0; a < 27; ++a) {
                double r[3]; orc_node_coord(g, tb[a], r);
                for (int b = 0; b < 27; ++b) {
                    if (tb[a] != bb[b]) { double rp[3]; orc_node_coord(g, bb[b], rp); G[a + 27*b] = Gr(r, rp, k); }
                    else G[a + 27*b] = 0;
                }
            }
            for (int t1 = 0; t1 < g->N_tet_cube && tests[t1]; ++t1)
                for (int b1 = 0; b1 < g->N_tet_cube && bases[b1]; ++b1) {
                    const int tT = tests[t1], tB = bases[b1];
                    if (tB < tT) continue;
                    zc blk[144];
                    near_block_lin(g, S, Sx, Sy, Sz, G, tT, tB, blk);
                    for (int q = 0; q < 144; ++q) {
                        if (sp32) sp32[144*blok + q] = (fc)blk[q];
                        if (sp64) sp64[144*blok + q] = blk[q];
                    }
                    sp_ind[2*blok] = tT; sp_ind[2*blok + 1] = tB;
                    blok++;
                }
        }
        if (blok != off[tcube]) err = -4;
    }
    free(off);
    return err;
}

/* -------------------------------------------------------------------- FFT */
/* Recursive mixed-radix DFT with FFTW's sign convention (forward exp(-i),
 * unnormalised).  Any length; small prime factors. */
static void fft_rec(const zc *in, int is, zc *out, int L, const zc *w, int wstep, int L0, zc *tmp) {
    if (L == 1) { out[0] = in[0]; return; }
    int p = 2; while (L % p) ++p;
    int m = L/p;
    for (int q = 0; q < p; ++q) fft_rec(in + (size_t)q*is, is*p, out + (size_t)q*m, m, w, wstep*p, L0, tmp);
    for (int k = 0; k < m; ++k) {
        for (int r = 0; r < p; ++r) {
            zc s = 0;
            for (int q = 0; q < p; ++q) {
                long e = ((long)q*(k + (long)r*m)) % L;
                s += w[(e*wstep) % L0]*out[(size_t)q*m + k];
            }
            tmp[r] = s;
        }
        for (int r = 0; r < p; ++r) out[(size_t)k + (size_t)r*m] = tmp[r];
    }
}

int orc_fft1d(int L, zc *x, int sign) {
    zc *w = (zc *)malloc(sizeof(zc)*(size_t)L), *o = (zc *)malloc(sizeof(zc)*(size_t)L), *t = (zc *)malloc(sizeof(zc)*(size_t)L);
    for (int j = 0; j < L; ++j) { double a = 2.0*PI*(double)j/(double)L; w[j] = CMPLX(cos(a), sign*sin(a)); }
    fft_rec(x, 1, o, L, w, 1, L, t);
    memcpy(x, o, sizeof(zc)*(size_t)L);
    free(w); free(o); free(t);
    return 0;
}

/* Line transforms: iterative radix-2 for power-of-two lengths (bit-reversal
 * then butterflies with a precomputed root table), the recursive mixed-radix
 * routine otherwise.  3D passes run their line loops with OpenMP, like the
 * reference's `!$OMP` regions in FFT3d_2/IFFT3d_2. */
typedef struct { int L, pow2; zc *w, *o, *t, *line; int *rev; } fft_plan;
static void plan_init(fft_plan *p, int L, int sign) {
    p->L = L;
    p->pow2 = (L & (L - 1)) == 0;
    p->w = (zc *)malloc(sizeof(zc)*(size_t)L); p->o = (zc *)malloc(sizeof(zc)*(size_t)L);
    p->t = (zc *)malloc(sizeof(zc)*(size_t)L); p->line = (zc *)malloc(sizeof(zc)*(size_t)L);
    p->rev = (int *)malloc(sizeof(int)*(size_t)L);
    for (int j = 0; j < L; ++j) { double a = 2.0*PI*(double)j/(double)L; p->w[j] = CMPLX(cos(a), sign*sin(a)); }
    if (p->pow2) {
        int lg = 0; while ((1 << lg) < L) ++lg;
        for (int i = 0; i < L; ++i) { int r = 0; for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b); p->rev[i] = r; }
    }
}
static void plan_free(fft_plan *p) { free(p->w); free(p->o); free(p->t); free(p->line); free(p->rev); }
static void fft_pow2(fft_plan *p, zc *x) {
    const int L = p->L;
    for (int i = 0; i < L; ++i) p->o[p->rev[i]] = x[i];
    for (int len = 2; len <= L; len <<= 1) {
        const int half = len >> 1, step = L/len;
        for (int b = 0; b < L; b += len)
            for (int j = 0; j < half; ++j) {
                zc u = p->o[b + j], v = p->o[b + j + half]*p->w[j*step];
                p->o[b + j] = u + v;
                p->o[b + j + half] = u - v;
            }
    }
    memcpy(x, p->o, sizeof(zc)*(size_t)L);
}
/* transform the line A[base + i*stride], i < L, in place */
static void plan_line(fft_plan *p, zc *A, size_t base, size_t stride) {
    for (int i = 0; i < p->L; ++i) p->line[i] = A[base + i*stride];
    if (p->pow2) fft_pow2(p, p->line);
    else { fft_rec(p->line, 1, p->o, p->L, p->w, 1, p->L, p->t); memcpy(p->line, p->o, sizeof(zc)*(size_t)p->L); }
    for (int i = 0; i < p->L; ++i) A[base + i*stride] = p->line[i];
}

/* Batched mixed-radix Stockham transforms for 5-smooth lengths: FB lines at
 * a time, held as separate real and imaginary arrays [L][FB] so that the
 * butterflies run over the batch with plain double arithmetic (the C
 * `_Complex` multiply of -O2 goes through a library call).  Stage with radix
 * R and sub-transform size Ns: element j < L/R takes x[j + q L/R] (q < R),
 * multiplies by exp(sign 2 pi i k q / (Ns R)), k = j mod Ns, forms the R-point
 * DFT and stores it at (j / Ns) Ns R + k + s Ns -- natural order out, no bit
 * reversal.  Other lengths keep the line routines above. */
#define FB 16
typedef struct {
    int L, nst, ok;
    int R[40];
    double *twr[40], *twi[40];        /* per stage: [k*R + q], k < Ns */
    double *ar, *ai, *br, *bi;        /* [L][FB] */
    fft_plan slow;
} bfft_plan;

static void bplan_init(bfft_plan *p, int L, int sign) {
    memset(p, 0, sizeof *p);
    p->L = L;
    int n = L;
    const int rs[4] = {4, 2, 3, 5};
    for (int i = 0; i < 4; ++i) while (n % rs[i] == 0 && p->nst < 40) { p->R[p->nst++] = rs[i]; n /= rs[i]; }
    p->ok = n == 1;
    if (!p->ok) { plan_init(&p->slow, L, sign); return; }
    int Ns = 1;
    for (int st = 0; st < p->nst; ++st) {
        const int R = p->R[st];
        p->twr[st] = (double *)malloc(sizeof(double)*(size_t)Ns*R);
        p->twi[st] = (double *)malloc(sizeof(double)*(size_t)Ns*R);
        for (int k = 0; k < Ns; ++k)
            for (int q = 0; q < R; ++q) {
                const double a = sign*2.0*PI*(double)(k*q)/(double)(Ns*R);
                p->twr[st][k*R + q] = cos(a);
                p->twi[st][k*R + q] = sin(a);
            }
        Ns *= R;
    }
    p->ar = (double *)malloc(sizeof(double)*(size_t)L*FB); p->ai = (double *)malloc(sizeof(double)*(size_t)L*FB);
    p->br = (double *)malloc(sizeof(double)*(size_t)L*FB); p->bi = (double *)malloc(sizeof(double)*(size_t)L*FB);
}

static void bplan_free(bfft_plan *p) {
    if (!p->ok) { plan_free(&p->slow); return; }
    for (int st = 0; st < p->nst; ++st) { free(p->twr[st]); free(p->twi[st]); }
    free(p->ar); free(p->ai); free(p->br); free(p->bi);
}

/* one Stockham stage over the batch: x -> y */
static void bstage(const bfft_plan *p, int st, int Ns, int sign, const double *xr, const double *xi, double *yr, double *yi) {
    const int L = p->L, R = p->R[st], NR = L/R;
    const double *twr = p->twr[st], *twi = p->twi[st];
    double cr[5], ci[5];                                   /* roots exp(sign 2 pi i t / R) */
    for (int t = 0; t < R; ++t) { const double a = sign*2.0*PI*(double)t/(double)R; cr[t] = cos(a); ci[t] = sin(a); }
    for (int j = 0; j < NR; ++j) {
        const int k = j % Ns, idx = (j/Ns)*Ns*R + k;
        double vr[5][FB], vi[5][FB];
        for (int q = 0; q < R; ++q) {
            const double *sr = xr + (size_t)(j + q*NR)*FB, *si = xi + (size_t)(j + q*NR)*FB;
            const double wr = twr[k*R + q], wi = twi[k*R + q];
            for (int b = 0; b < FB; ++b) { vr[q][b] = sr[b]*wr - si[b]*wi; vi[q][b] = sr[b]*wi + si[b]*wr; }
        }
        double *o[5][2];
        for (int t = 0; t < R; ++t) { o[t][0] = yr + (size_t)(idx + t*Ns)*FB; o[t][1] = yi + (size_t)(idx + t*Ns)*FB; }
        if (R == 2) {
            for (int b = 0; b < FB; ++b) {
                o[0][0][b] = vr[0][b] + vr[1][b]; o[0][1][b] = vi[0][b] + vi[1][b];
                o[1][0][b] = vr[0][b] - vr[1][b]; o[1][1][b] = vi[0][b] - vi[1][b];
            }
        } else if (R == 4) {
            /* X1 = (v0 - v2) + w (v1 - v3), X3 = (v0 - v2) - w (v1 - v3), w = sign * i */
            for (int b = 0; b < FB; ++b) {
                const double a0r = vr[0][b] + vr[2][b], a0i = vi[0][b] + vi[2][b];
                const double a1r = vr[0][b] - vr[2][b], a1i = vi[0][b] - vi[2][b];
                const double a2r = vr[1][b] + vr[3][b], a2i = vi[1][b] + vi[3][b];
                const double a3r = vr[1][b] - vr[3][b], a3i = vi[1][b] - vi[3][b];
                const double w3r = -sign*a3i, w3i = sign*a3r;   /* w * a3 */
                o[0][0][b] = a0r + a2r; o[0][1][b] = a0i + a2i;
                o[2][0][b] = a0r - a2r; o[2][1][b] = a0i - a2i;
                o[1][0][b] = a1r + w3r; o[1][1][b] = a1i + w3i;
                o[3][0][b] = a1r - w3r; o[3][1][b] = a1i - w3i;
            }
        } else {
            for (int t = 0; t < R; ++t)
                for (int b = 0; b < FB; ++b) {
                    double sr = vr[0][b], si = vi[0][b];
                    for (int q = 1; q < R; ++q) {
                        const int e = (q*t) % R;
                        sr += vr[q][b]*cr[e] - vi[q][b]*ci[e];
                        si += vr[q][b]*ci[e] + vi[q][b]*cr[e];
                    }
                    o[t][0][b] = sr; o[t][1][b] = si;
                }
        }
    }
}

/* transform lines base_b + i*stride (b < nb <= FB, i < L) in place */
static void bplan_lines(bfft_plan *p, int sign, zc *A, const size_t *base, int nb, size_t stride) {
    const int L = p->L;
    if (!p->ok) { for (int b = 0; b < nb; ++b) plan_line(&p->slow, A, base[b], stride); return; }
    for (int i = 0; i < L; ++i)
        for (int b = 0; b < FB; ++b) {
            const zc v = b < nb ? A[base[b] + i*stride] : 0;
            p->ar[(size_t)i*FB + b] = creal(v);
            p->ai[(size_t)i*FB + b] = cimag(v);
        }
    double *xr = p->ar, *xi = p->ai, *yr = p->br, *yi = p->bi;
    int Ns = 1;
    for (int st = 0; st < p->nst; ++st) {
        bstage(p, st, Ns, sign, xr, xi, yr, yi);
        double *t = xr; xr = yr; yr = t;
        t = xi; xi = yi; yi = t;
        Ns *= p->R[st];
    }
    for (int i = 0; i < L; ++i)
        for (int b = 0; b < nb; ++b) A[base[b] + i*stride] = CMPLX(xr[(size_t)i*FB + b], xi[(size_t)i*FB + b]);
}

static int smooth5(int L) {
    for (int r = 2; r <= 5; ++r) while (L % r == 0) L /= r;
    return L == 1;
}

/* pass over lines (i1 < n1, i2 < n2) with base = i1*s1 + i2*s2: FB
 * consecutive i2 per batch for 5-smooth lengths, one line per work item
 * otherwise (finer load balance for the slower generic routine) */
static void pass_lines(int L, int sign, zc *A, int n1, size_t s1, int n2, size_t s2, size_t stride) {
    if (!smooth5(L)) {
#pragma omp parallel
        {
            fft_plan p; plan_init(&p, L, sign);
#pragma omp for collapse(2) schedule(static)
            for (int i1 = 0; i1 < n1; ++i1) for (int i2 = 0; i2 < n2; ++i2) plan_line(&p, A, i1*s1 + i2*s2, stride);
            plan_free(&p);
        }
        return;
    }
    const int nc = (n2 + FB - 1)/FB;
#pragma omp parallel
    {
        bfft_plan p; bplan_init(&p, L, sign);
        size_t base[FB];
#pragma omp for collapse(2) schedule(static)
        for (int i1 = 0; i1 < n1; ++i1)
            for (int c = 0; c < nc; ++c) {
                const int i2a = c*FB, nb = n2 - i2a < FB ? n2 - i2a : FB;
                for (int b = 0; b < nb; ++b) base[b] = i1*s1 + (size_t)(i2a + b)*s2;
                bplan_lines(&p, sign, A, base, nb, stride);
            }
        bplan_free(&p);
    }
}

/* FFT3d / IFFT3d: full unnormalised 3D transform (src/possu.f90:124-136,209-221) */
int orc_fft3d(int Px, int Py, int Pz, zc *A, int sign) {
    size_t sy = (size_t)Px, sz = (size_t)Px*Py;
    pass_lines(Px, sign, A, Pz, sz, Py, sy, 1);
    pass_lines(Py, sign, A, Pz, sz, Px, 1, sy);
    pass_lines(Pz, sign, A, Py, sy, Px, 1, sz);
    return 0;
}

/* FFT3d_2 / IFFT3d_2: the zero-padding-pruned passes (src/possu.f90:140-204,225-289) */
int orc_fft3d_pruned(int Px, int Py, int Pz, zc *A, int inverse) {
    int sign = inverse ? 1 : -1;
    size_t sy = (size_t)Px, sz = (size_t)Px*Py;
    if (!inverse) {
        pass_lines(Px, sign, A, Pz/2, sz, Py/2, sy, 1);
        pass_lines(Py, sign, A, Pz/2, sz, Px, 1, sy);
        pass_lines(Pz, sign, A, Py, sy, Px, 1, sz);
    } else {
        pass_lines(Pz, sign, A, Py, sy, Px, 1, sz);
        pass_lines(Py, sign, A, Pz/2, sz, Px, 1, sy);
        pass_lines(Px, sign, A, Pz/2, sz, Py/2, sy, 1);
    }
    return 0;
}

/* build_G, src/build_G.f90:1-66 */
int orc_build_G(const orc_geom *g, zc *Fg) {
    const int Nx = g->Nx, Ny = g->Ny, Nz = g->Nz, Px = 2*Nx, Py = 2*Ny, Pz = 2*Nz;
    size_t tot = (size_t)Px*Py*Pz;
    for (size_t i = 0; i < tot; ++i) Fg[i] = 0;
    double n1[3]; orc_node_coord(g, 1, n1);
#define AIX(a, b, c) ((size_t)((a) - 1) + (size_t)Px*((size_t)((b) - 1) + (size_t)Py*(size_t)((c) - 1)))
    int las = 1;
    for (int m1 = 1; m1 <= Nz; ++m1) for (int l1 = 1; l1 <= Ny; ++l1) for (int k1 = 1; k1 <= Nx; ++k1) {
        double nl[3]; orc_node_coord(g, las, nl);
        double R = norm2pt(n1, nl);
        zc cmp = 0;
        if (R > 0.0) { double d = 4*PI*R; cmp = CMPLX(cos(g->k*R)/d, sin(g->k*R)/d); }
        Fg[AIX(k1, l1, m1)] = cmp;
        if (k1 != 1) Fg[AIX(Px - k1 + 2, l1, m1)] = cmp;
        if (k1 != 1 && m1 != 1) Fg[AIX(Px - k1 + 2, l1, Pz - m1 + 2)] = cmp;
        if (k1 != 1 && l1 != 1) Fg[AIX(Px - k1 + 2, Py - l1 + 2, m1)] = cmp;
        if (k1 != 1 && l1 != 1 && m1 != 1) Fg[AIX(Px - k1 + 2, Py - l1 + 2, Pz - m1 + 2)] = cmp;
        if (m1 != 1) Fg[AIX(k1, l1, Pz - m1 + 2)] = cmp;
        if (l1 != 1) Fg[AIX(k1, Py - l1 + 2, m1)] = cmp;
        if (l1 != 1 && m1 != 1) Fg[AIX(k1, Py - l1 + 2, Pz - m1 + 2)] = cmp;
        las++;
    }
#undef AIX
    Fg[0] = 0;
    return orc_fft3d(Px, Py, Pz, Fg, -1);
}

/* ------------------------------------------------------------- matvec */
/* sparse_T_matmul, src/sparse.f90:13-43 (serial, as the reference) */
void orc_sparse_T_matmul(int T, const zc *val, const int32_t *ind, const zc *x, int Ngrid, zc *out) {
    for (int i = 0; i < Ngrid; ++i) out[i] = 0;
    for (int i = 0; i < T; ++i) for (int j = 0; j < 27; ++j) {
        int row = ind[27*(size_t)i + j] - 1;
        out[row] = out[row] + val[27*(size_t)i + j]*x[i];
    }
}
/* sparse_eps_matmul, src/sparse.f90:47-77 (eps not applied, as :68,70) */
void orc_sparse_eps_matmul(int T, const zc *val, const int32_t *ind, const zc *x, zc *out) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < T; ++i) {
        zc s = 0;
        for (int j = 0; j < 27; ++j) s = s + val[27*(size_t)i + j]*x[ind[27*(size_t)i + j] - 1];
        out[i] = s;
    }
}
/* matmul_Acorr_const, src/sparse_mat.f90:96-123: Ax[a] += V x[b]; if a != b,
 * Ax[b] += V^T x[a] (transpose, not conjugate).  With several threads each
 * thread accumulates privately, as the reference's `reduction(+:Ax)`. */
void orc_matmul_Acorr_const(int T, int64_t B, const fc *sp32, const zc *sp64, const int32_t *sp_ind,
                            const zc *x, zc *Ax, int nthreads) {
    size_t n = 3*(size_t)T;
    for (size_t i = 0; i < n; ++i) Ax[i] = 0;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#else
    nthreads = 1;
#endif
    if (nthreads == 1) {
        for (int64_t i1 = 0; i1 < B; ++i1) {
            size_t a = 3*(size_t)(sp_ind[2*i1] - 1), b = 3*(size_t)(sp_ind[2*i1 + 1] - 1);
            zc v[9];
            for (int q = 0; q < 9; ++q) v[q] = sp32 ? (zc)sp32[9*i1 + q] : sp64[9*i1 + q];
            zc y0 = v[0]*x[b] + v[3]*x[b + 1] + v[6]*x[b + 2];
            zc y1 = v[1]*x[b] + v[4]*x[b + 1] + v[7]*x[b + 2];
            zc y2 = v[2]*x[b] + v[5]*x[b + 1] + v[8]*x[b + 2];
            Ax[a] += y0; Ax[a + 1] += y1; Ax[a + 2] += y2;
            if (a != b) {
                zc z0 = v[0]*x[a] + v[1]*x[a + 1] + v[2]*x[a + 2];
                zc z1 = v[3]*x[a] + v[4]*x[a + 1] + v[5]*x[a + 2];
                zc z2 = v[6]*x[a] + v[7]*x[a + 1] + v[8]*x[a + 2];
                Ax[b] += z0; Ax[b + 1] += z1; Ax[b + 2] += z2;
            }
        }
        return;
    }
    zc *priv = (zc *)calloc(n*(size_t)nthreads, sizeof(zc));
#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads)
#endif
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        zc *y = priv + n*(size_t)tid;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t i1 = 0; i1 < B; ++i1) {
            size_t a = 3*(size_t)(sp_ind[2*i1] - 1), b = 3*(size_t)(sp_ind[2*i1 + 1] - 1);
            zc v[9];
            for (int q = 0; q < 9; ++q) v[q] = sp32 ? (zc)sp32[9*i1 + q] : sp64[9*i1 + q];
            y[a]     += v[0]*x[b] + v[3]*x[b + 1] + v[6]*x[b + 2];
            y[a + 1] += v[1]*x[b] + v[4]*x[b + 1] + v[7]*x[b + 2];
            y[a + 2] += v[2]*x[b] + v[5]*x[b + 1] + v[8]*x[b + 2];
            if (a != b) {
                y[b]     += v[0]*x[a] + v[1]*x[a + 1] + v[2]*x[a + 2];
                y[b + 1] += v[3]*x[a] + v[4]*x[a + 1] + v[5]*x[a + 2];
                y[b + 2] += v[6]*x[a] + v[7]*x[a + 1] + v[8]*x[a + 2];
            }
        }
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (size_t i = 0; i < n; ++i) {
            zc s = 0;
            for (int t = 0; t < nthreads; ++t) s += priv[n*(size_t)t + i];
            Ax[i] = s;
        }
    }
    free(priv);
}

/* matmul_Acorr, src/sparse_mat.f90:64-92 (linear basis): 12 unknowns per tet
 * ordered (component, node) as x(12(t-1) + 4c + i); Ax[a] += V x[b] and, if
 * a != b, Ax[b] += V^T x[a].  V(r, c) is stored column-major per block. */
void orc_matmul_Acorr(int T, int64_t B, const fc *sp32, const zc *sp64, const int32_t *sp_ind,
                      const zc *x, zc *Ax) {
    size_t n = 12*(size_t)T;
    for (size_t i = 0; i < n; ++i) Ax[i] = 0;
    for (int64_t i1 = 0; i1 < B; ++i1) {
        size_t a = 12*(size_t)(sp_ind[2*i1] - 1), b = 12*(size_t)(sp_ind[2*i1 + 1] - 1);
        const size_t v0 = 144*(size_t)i1;
        for (int r = 0; r < 12; ++r) {
            zc s = 0;
            for (int c = 0; c < 12; ++c) s += (sp32 ? (zc)sp32[v0 + r + 12*c] : sp64[v0 + r + 12*c])*x[b + c];
            Ax[a + r] += s;
        }
        if (a != b)
            for (int c = 0; c < 12; ++c) {
                zc s = 0;
                for (int r = 0; r < 12; ++r) s += (sp32 ? (zc)sp32[v0 + r + 12*c] : sp64[v0 + r + 12*c])*x[a + r];
                Ax[b + c] += s;
            }
    }
}

/* one convolution: grid source -> pruned FFT -> x Fg -> pruned IFFT -> octant/(8N^3) */
static void convolve(const orc_op *op, zc *grid_src /* N^3 */, zc *SS, zc *out /* N^3 */) {
    const orc_geom *g = op->g;
    const int Nx = g->Nx, Ny = g->Ny, Nz = g->Nz, Px = 2*Nx, Py = 2*Ny, Pz = 2*Nz;
    size_t tot = (size_t)Px*Py*Pz;
    /* vec2arr2, src/common.f90:1412-1458 */
    for (size_t i = 0; i < tot; ++i) SS[i] = 0;
    for (int m = 0; m < Nz; ++m) for (int l = 0; l < Ny; ++l) for (int k = 0; k < Nx; ++k)
        SS[k + (size_t)Px*(l + (size_t)Py*m)] = grid_src[k + (size_t)Nx*(l + (size_t)Ny*m)];
    orc_fft3d_pruned(Px, Py, Pz, SS, 0);
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < tot; ++i) SS[i] = op->Fg[i]*SS[i];
    orc_fft3d_pruned(Px, Py, Pz, SS, 1);
    /* arr2vec, src/common.f90:417-438 */
    double sc = 8.0*Nx*Ny*Nz;
    for (int m = 0; m < Nz; ++m) for (int l = 0; l < Ny; ++l) for (int k = 0; k < Nx; ++k)
        out[k + (size_t)Nx*(l + (size_t)Ny*m)] = SS[k + (size_t)Px*(l + (size_t)Py*m)]/sc;
}

/* compute_Ax2, src/gmres_module.f90:57-176, constant (order 0) or linear
 * (order 1) basis.  The linear basis has 4 projector columns per tet (one per
 * node, S(27, 4T)) and 12 unknowns per tet, x(12(t-1) + 4c + i) for component
 * c and node i (:88-95, :156-165).  merged = 1 folds convolutions 4-6
 * (:122-144) into one by linearity. */
int orc_compute_Ax2(const orc_op *op, const zc *x, zc *Ax) {
    const orc_geom *g = op->g;
    const int Nb = op->order == 1 ? 4 : 1;
    const int T = Nb*op->T;   /* projector columns */
    const size_t mm = (size_t)g->Nx*g->Ny*g->Nz, tot = 8*mm;
    zc *X = (zc *)malloc(sizeof(zc)*3*(size_t)T);
    zc *src = (zc *)malloc(sizeof(zc)*mm), *res = (zc *)malloc(sizeof(zc)*mm), *SS = (zc *)malloc(sizeof(zc)*tot);
    zc *Y[3], *Y2[3], *tmp = (zc *)malloc(sizeof(zc)*(size_t)T);
    for (int d = 0; d < 3; ++d) { Y[d] = (zc *)malloc(sizeof(zc)*(size_t)T); Y2[d] = (zc *)calloc((size_t)T, sizeof(zc)); }
    if (Nb == 1)
        for (int t = 0; t < T; ++t) for (int d = 0; d < 3; ++d) X[(size_t)d*T + t] = x[3*(size_t)t + d];
    else
        for (int t = 0; t < op->T; ++t) for (int i = 0; i < 4; ++i) for (int d = 0; d < 3; ++d)
            X[(size_t)d*T + 4*(size_t)t + i] = x[12*(size_t)t + 4*d + i];
    const zc *P[3] = {op->Sx, op->Sy, op->Sz};
    for (int d = 0; d < 3; ++d) {
        orc_sparse_T_matmul(T, op->S, op->indS, X + (size_t)d*T, (int)mm, src);
        convolve(op, src, SS, res);
        orc_sparse_eps_matmul(T, op->S, op->indS, res, Y[d]);
    }
    if (!op->merged) {
        for (int d = 0; d < 3; ++d) {
            orc_sparse_T_matmul(T, P[d], op->indS, X + (size_t)d*T, (int)mm, src);
            convolve(op, src, SS, res);
            for (int e = 0; e < 3; ++e) {
                orc_sparse_eps_matmul(T, P[e], op->indS, res, tmp);
                for (int t = 0; t < T; ++t) Y2[e][t] = Y2[e][t] + tmp[t];
            }
        }
    } else {
        zc *acc = (zc *)calloc(mm, sizeof(zc));
        for (int d = 0; d < 3; ++d) {
            orc_sparse_T_matmul(T, P[d], op->indS, X + (size_t)d*T, (int)mm, src);
            for (size_t i = 0; i < mm; ++i) acc[i] += src[i];
        }
        convolve(op, acc, SS, res);
        for (int e = 0; e < 3; ++e) orc_sparse_eps_matmul(T, P[e], op->indS, res, Y2[e]);
        free(acc);
    }
    const double k2 = op->k*op->k;
    if (Nb == 1) {
        orc_matmul_Acorr_const(T, op->B, op->sp32, op->sp64, op->sp_ind, x, Ax, op->nthreads);
        for (int t = 0; t < T; ++t) for (int d = 0; d < 3; ++d)
            Ax[3*(size_t)t + d] = Ax[3*(size_t)t + d] + (Y2[d][t] - k2*Y[d][t]);
    } else {
        orc_matmul_Acorr(op->T, op->B, op->sp32, op->sp64, op->sp_ind, x, Ax);
        for (int t = 0; t < op->T; ++t) for (int i = 0; i < 4; ++i) for (int d = 0; d < 3; ++d) {
            const size_t b = 4*(size_t)t + i;
            Ax[12*(size_t)t + 4*d + i] = Ax[12*(size_t)t + 4*d + i] + (Y2[d][b] - k2*Y[d][b]);
        }
    }
    free(X); free(src); free(res); free(SS); free(tmp);
    for (int d = 0; d < 3; ++d) { free(Y[d]); free(Y2[d]); }
    return 0;
}

/* ---------------------------------------------------------------- GMRES */
static zc zdot(size_t n, const zc *a, const zc *b) {   /* Fortran dot_product: sum conj(a) b */
    double re = 0, im = 0;
#pragma omp parallel for reduction(+:re,im) schedule(static)
    for (size_t i = 0; i < n; ++i) { zc p = conj(a[i])*b[i]; re += creal(p); im += cimag(p); }
    return CMPLX(re, im);
}
static void zaxpy(size_t n, zc a, const zc *x, zc *y) {   /* y -= a x */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; ++i) y[i] = y[i] - a*x[i];
}

/* y = inv(H(1:i,1:i)) g(1:i) for the upper-triangular H left by the Givens
 * rotations; the reference forms the inverse with ZGETRF/ZGETRI
 * (src/possu.f90:331-365), which needs no row swaps on a triangular matrix,
 * so back substitution gives the same solution up to rounding. */
static void tri_solve(int i, int ld, const zc *H, const zc *g, zc *y) {
    for (int r = i - 1; r >= 0; --r) {
        zc s = g[r];
        for (int c = r + 1; c < i; ++c) s -= H[r + (size_t)ld*c]*y[c];
        y[r] = s/H[r + (size_t)ld*r];
    }
}

/* gmres, src/gmres_module.f90:180-325.  The matvec the reference repeats at
 * the end of each cycle (:309) is not repeated: the next cycle recomputes it
 * (:224) and nothing reads the first one. */
int orc_gmres(const orc_op *op, const zc *rhs, zc *xout, double tol, int m, int cycles, orc_gmres_info *info) {
    const size_t n = (op->order == 1 ? 12 : 3)*(size_t)op->T;
    zc *x = (zc *)malloc(sizeof(zc)*n), *r = (zc *)malloc(sizeof(zc)*n), *w = (zc *)malloc(sizeof(zc)*n);
    zc *V = (zc *)calloc(n*(size_t)(m + 1), sizeof(zc));
    zc *H = (zc *)calloc((size_t)(m + 1)*m, sizeof(zc));
    zc *cs = (zc *)calloc((size_t)m + 1, sizeof(zc)), *sn = (zc *)calloc((size_t)m + 1, sizeof(zc));
    zc *g = (zc *)calloc((size_t)m + 1, sizeof(zc)), *y = (zc *)calloc((size_t)m, sizeof(zc));
    const int ld = m + 1;
    memcpy(x, rhs, sizeof(zc)*n);
    double b_norm = creal(csqrt(zdot(n, rhs, rhs)));
    double error = 1e300;
    const double reorth = (double)0.001f;
    int iters = 0, matvecs = 0, cyc = 0, hlen = 0;
    for (int it = 1; it <= cycles; ++it) {
        cyc = it;
        orc_compute_Ax2(op, x, w); matvecs++;
        for (size_t i = 0; i < n; ++i) r[i] = rhs[i] - w[i];
        zc rn = csqrt(zdot(n, r, r));
        for (size_t i = 0; i < n; ++i) V[i] = r[i]/rn;
        for (int i = 0; i <= m; ++i) g[i] = 0;
        g[0] = csqrt(zdot(n, r, r));
        int conv_i = 0;
        for (int i = 1; i <= m; ++i) {
            zc *vi = V + n*(size_t)(i - 1), *vn = V + n*(size_t)i;
            orc_compute_Ax2(op, vi, w); matvecs++;
            iters++;
            double normav = creal(csqrt(zdot(n, w, w)));
            for (int k = 1; k <= i; ++k) {
                zc h = zdot(n, V + n*(size_t)(k - 1), w);
                H[(k - 1) + (size_t)ld*(i - 1)] = h;
                zaxpy(n, h, V + n*(size_t)(k - 1), w);
            }
            zc hn = csqrt(zdot(n, w, w));
            H[i + (size_t)ld*(i - 1)] = hn;
            double normav2 = creal(hn);
            memcpy(vn, w, sizeof(zc)*n);
            if (normav + reorth*normav2 == normav) {
                for (int j = 1; j <= i; ++j) {
                    zc hr = zdot(n, V + n*(size_t)(j - 1), vn);
                    H[(j - 1) + (size_t)ld*(i - 1)] += hr;
                    zaxpy(n, hr, V + n*(size_t)(j - 1), vn);
                }
                H[i + (size_t)ld*(i - 1)] = csqrt(zdot(n, vn, vn));
            }
            zc hh = H[i + (size_t)ld*(i - 1)];
            if (hh != 0.0) for (size_t q = 0; q < n; ++q) vn[q] = vn[q]/hh;
            zc *Hc = H + (size_t)ld*(i - 1);
            for (int k = 1; k <= i - 1; ++k) {
                zc tmp = cs[k - 1]*Hc[k - 1] - sn[k - 1]*Hc[k];
                Hc[k] = sn[k - 1]*Hc[k - 1] + conj(cs[k - 1])*Hc[k];
                Hc[k - 1] = tmp;
            }
            double nu = creal(csqrt(conj(Hc[i - 1])*Hc[i - 1] + conj(Hc[i])*Hc[i]));
            if (nu != 0.0) {
                cs[i - 1] = conj(Hc[i - 1]/nu);
                sn[i - 1] = -Hc[i]/nu;
                Hc[i - 1] = cs[i - 1]*Hc[i - 1] - sn[i - 1]*Hc[i];
                Hc[i] = 0.0;
                zc t1 = g[i - 1], t2 = g[i];
                g[i - 1] = cs[i - 1]*t1 - sn[i - 1]*t2;
                g[i] = sn[i - 1]*t1 + conj(cs[i - 1])*t2;
            }
            error = cabs(g[i])/b_norm;
            if (info && info->history && hlen < info->history_len) info->history[hlen++] = error;
            if (error < tol) { conv_i = i; break; }
        }
        int kdim = conv_i ? conv_i : m;
        tri_solve(kdim, ld, H, g, y);
        /* x = x + matmul(V(:,1:i), y) */
#pragma omp parallel for schedule(static)
        for (size_t q = 0; q < n; ++q) {
            zc s = 0;
            for (int c = 0; c < kdim; ++c) s += V[n*(size_t)c + q]*y[c];
            x[q] = x[q] + s;
        }
        if (error < tol) break;
    }
    memcpy(xout, x, sizeof(zc)*n);
    if (info) {
        info->iters = iters; info->matvecs = matvecs; info->cycles = cyc;
        info->converged = error < tol; info->relres = error; info->history_len = hlen;
    }
    free(x); free(r); free(w); free(V); free(H); free(cs); free(sn); free(g); free(y);
    return (error < tol) ? 0 : 1;
}

/* The orthogonalisation of one Arnoldi step of orc_gmres against i Krylov
 * vectors (src/gmres_module.f90:241-244): h_k = <v_k, w>, w -= h_k v_k for
 * k = 1..i, with the same zdot/zaxpy; timed alone by the CPU baseline. */
void orc_mgs_terms(size_t n, int i, const zc *V, zc *w, zc *h) {
    for (int k = 0; k < i; ++k) {
        h[k] = zdot(n, V + n*(size_t)k, w);
        zaxpy(n, h[k], V + n*(size_t)k, w);
    }
}

/* ------------------------------------------------- special functions */
/* envj / msta1 / msta2, src/sfunctions.f90:81-145 (Zhang & Jin) */
static double envj(int n, double x) {
    n = n < 0 ? -n : n; if (n < 1) n = 1;
    return 0.5*log10(6.28*n) - (double)n*log10(1.36*x/n);
}
static const double F11 = (double)1.1f;
static int msta1(double x, int mp) {
    double a0 = fabs(x);
    int n0 = (int)(F11*a0) + 1;
    double f0 = envj(n0, a0) - mp;
    int n1 = n0 + 5;
    double f1 = envj(n1, a0) - mp;
    int nn = n1;
    for (int it = 1; it <= 20; ++it) {
        nn = n1 - (int)((n1 - n0)/(1.0 - f0/f1));
        double f = envj(nn, a0) - mp;
        if (abs(nn - n1) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn;
}
static int msta2(double x, int n, int mp) {
    double a0 = fabs(x), hmp = 0.5*mp, ejn = envj(n, a0), obj;
    int n0;
    if (ejn <= hmp) { obj = mp; n0 = (int)(F11*a0); }
    else { obj = hmp + ejn; n0 = n; }
    double f0 = envj(n0, a0) - obj;
    int n1 = n0 + 5;
    double f1 = envj(n1, a0) - obj;
    int nn = n1;
    for (int it = 1; it <= 20; ++it) {
        nn = n1 - (int)((n1 - n0)/(1.0 - f0/f1));
        double f = envj(nn, a0) - obj;
        if (abs(nn - n1) < 1) break;
        n0 = n1; f0 = f1; n1 = nn; f1 = f;
    }
    return nn + 10;
}
/* cspherebessel, src/sfunctions.f90:20-69 (Zhang & Jin CSPHJY, values only) */
void orc_cspherebessel(int n, zc z, zc *csj, zc *csy) {
    double a0 = cabs(z);
    int nm = n;
    if (a0 < 1.0e-60) {
        for (int k = 0; k <= n; ++k) { csj[k] = 0; csy[k] = -1.0e300; }
        csy[0] = 1.0;
        return;
    }
    for (int k = 0; k <= n; ++k) csj[k] = 0;
    csj[0] = csin(z)/z;
    csj[1] = (csj[0] - ccos(z))/z;
    if (n >= 2) {
        zc csa = csj[0], csb = csj[1], cs = 0, cf = 0;
        int m = msta1(a0, 200);
        if (m < n) nm = m; else m = msta2(a0, n, 15);
        zc cf0 = 0, cf1 = 1.0 - 100;
        for (int k = m; k >= 0; --k) {
            cf = (2.0*k + 3.0)*cf1/z - cf0;
            if (k <= nm) csj[k] = cf;
            cf0 = cf1; cf1 = cf;
        }
        if (cabs(csa) > cabs(csb)) cs = csa/cf;
        if (cabs(csa) <= cabs(csb)) cs = csb/cf0;
        int top = nm < n ? nm : n;
        for (int k = 0; k <= top; ++k) csj[k] = cs*csj[k];
    }
    for (int k = 0; k <= n; ++k) csy[k] = 1.0e200;
    csy[0] = -ccos(z)/z;
    csy[1] = (csy[0] - csin(z))/z;
    int top = nm < n ? nm : n;
    for (int k = 2; k <= top; ++k) {
        if (cabs(csj[k - 1]) > cabs(csj[k - 2])) csy[k] = (csj[k]*csy[k - 1] - 1.0/(z*z))/csj[k - 1];
        else csy[k] = (csj[k]*csy[k - 2] - (2.0*k - 1.0)/(z*z*z))/csj[k - 2];
    }
}
/* legendre2, src/sfunctions.f90:615-686: associated Legendre P_N^m(x),
 * m = 0..N (the derivative table PD does not feed the result) */
void orc_legendre2(int N, double x, double *P) {
    int D = N + 2;
    double *PM = (double *)calloc((size_t)D*D, sizeof(double));
#define PMi(a, b) PM[(a) - 1 + (size_t)D*((b) - 1)]
    PMi(1, 1) = 1.0;
    if (fabs(x) == 1.0) for (int i1 = 1; i1 <= N; ++i1) PMi(1, i1 + 1) = pow(x, i1);
    int LS = 1; if (fabs(x) > 1.0) LS = -1;
    double xq = sqrt(LS*(1.0 - x*x));
    for (int i1 = 1; i1 <= N; ++i1) PMi(i1 + 1, i1 + 1) = -LS*(2.0*i1 - 1.0)*xq*PMi(i1, i1);
    for (int i1 = 0; i1 <= N; ++i1) PMi(i1 + 1, i1 + 2) = (2.0*i1 + 1.0)*x*PMi(i1 + 1, i1 + 1);
    for (int i1 = 0; i1 <= N; ++i1) for (int i2 = i1 + 2; i2 <= N; ++i2)
        PMi(i1 + 1, i2 + 1) = ((2.0*i2 - 1.0)*x*PMi(i1 + 1, i2) - (i1 + i2 - 1.0)*PMi(i1 + 1, i2 - 1))/(double)(i2 - i1);
    for (int m = 0; m <= N; ++m) P[m] = PMi(m + 1, N + 1);
#undef PMi
    free(PM);
}
static double factorial(int a) { double b = 1.0; for (int i = 1; i <= a; ++i) b = b*i; return b; }

/* calc_MN with inou = 0, src/mie.f90:408-496: regular VSWFs at Po, in
 * Cartesian components; MM, NN are (3, nm) column-major */
int orc_calc_MN(int Nmax, zc k, const double Po[3], zc *MM, zc *NN) {
    double r = sqrt(Po[0]*Po[0] + Po[1]*Po[1] + Po[2]*Po[2]);
    double theta = r != 0.0 ? acos(Po[2]/r) : 0.0, phi = atan2(Po[1], Po[0]);
    zc kr = k*r;
    zc *sphj = (zc *)malloc(sizeof(zc)*(size_t)(Nmax + 2)), *sphy = (zc *)malloc(sizeof(zc)*(size_t)(Nmax + 2));
    orc_cspherebessel(Nmax + 1, kr, sphj, sphy);
    double *L = (double *)malloc(sizeof(double)*(size_t)(Nmax + 3)), *L1 = (double *)malloc(sizeof(double)*(size_t)(Nmax + 3)),
           *L2 = (double *)malloc(sizeof(double)*(size_t)(Nmax + 3));
    double st = sin(theta), ct = cos(theta), sp = sin(phi), cp = cos(phi);
    double Hm[3][3] = {{st*cp, ct*cp, -sp}, {st*sp, ct*sp, cp}, {ct, -st, 0.0}};
    int ind = 0;
    for (int n = 1; n <= Nmax; ++n) {
        zc alpha = sphj[n];
        zc beta = csqrt((zc)(double)(n*(n + 1)))/kr*sphj[n];
        zc gamma = (n + 1.0)/kr*sphj[n] - sphj[n + 1];
        orc_legendre2(n, ct, L); orc_legendre2(n + 1, ct, L1); orc_legendre2(n - 1, ct, L2);
        double q = sqrt(n*(n + 1.0))/((n*2.0 + 1.0)*st);
        for (int m = -n; m <= n; ++m, ++ind) {
            int mm = abs(m);
            double cc = sqrt((2.0*n + 1.0)*factorial(n - mm)/factorial(n + mm)/(4.0*PI));
            zc e = cexp(CMPLX(0.0, m*phi));
            zc Y = L[mm]*e, Y1 = L1[mm]*e, Y2 = (mm == n) ? 0.0 : L2[mm]*e;
            Y1 = Y1*((n - mm + 1.0)/(n + 1.0));
            Y2 = Y2*((double)(n + mm)/(double)n);
            zc Bv[3] = {0, Y1 - Y2, (CMPLX(0.0, (double)(float)(m*(2*n + 1.0f)))/(double)(float)(n*(n + 1.0f)))*Y};
            for (int d = 0; d < 3; ++d) Bv[d] = Bv[d]*q;
            zc Cv[3] = {0, Bv[2], -Bv[1]};
            zc Pv[3] = {Y, 0, 0};
            zc Mn[3], Nn[3];
            for (int d = 0; d < 3; ++d) { Mn[d] = cc*alpha*Cv[d]; Nn[d] = cc*(beta*Pv[d] + gamma*Bv[d]); }
            for (int d = 0; d < 3; ++d) {
                MM[3*ind + d] = Hm[d][0]*Mn[0] + Hm[d][1]*Mn[1] + Hm[d][2]*Mn[2];
                NN[3*ind + d] = Hm[d][0]*Nn[0] + Hm[d][1]*Nn[1] + Hm[d][2]*Nn[2];
            }
        }
    }
    free(sphj); free(sphy); free(L); free(L1); free(L2);
    return 0;
}

/* vswf2constant, src/T_matrix.f90:280-305: mat(3T, 2nm) column-major */
int orc_vswf2constant(const double *coord, const int32_t *etopol, int T, zc k, int Nmax, zc *mat) {
    int nm = (Nmax + 1)*(Nmax + 1) - 1;
    size_t n = 3*(size_t)T;
    zc *MM = (zc *)malloc(sizeof(zc)*3*(size_t)nm), *NN = (zc *)malloc(sizeof(zc)*3*(size_t)nm);
    for (int t = 0; t < T; ++t) {
        double tc[4][3], r[3];
        tet_coord(coord, etopol, t, tc);
        for (int d = 0; d < 3; ++d) r[d] = (tc[0][d] + tc[1][d] + tc[2][d] + tc[3][d])/4.0;
        orc_calc_MN(Nmax, k, r, MM, NN);
        double sv = sqrt(tetra_volume(tc));
        for (int c = 0; c < nm; ++c) for (int d = 0; d < 3; ++d) {
            mat[3*(size_t)t + d + n*(size_t)c] = MM[3*c + d]*sv;
            mat[3*(size_t)t + d + n*(size_t)(nm + c)] = NN[3*c + d]*sv;
        }
    }
    free(MM); free(NN);
    return 0;
}

/* T_mat(:, c) = matmul(transpose(conjg(mat)), x_c), src/T_matrix.f90:260 */
void orc_T_assemble(int n, int ncol, const zc *mat, const zc *X, zc *Tc) {
#pragma omp parallel for schedule(static)
    for (int c = 0; c < ncol; ++c) for (int r = 0; r < ncol; ++r) {
        zc s = 0;
        for (int i = 0; i < n; ++i) s += conj(mat[i + (size_t)n*r])*X[i + (size_t)n*c];
        Tc[r + (size_t)ncol*c] = s;
    }
}

/* Mie coefficients in the convention of mie_T_matrix (src/T_matrix.f90:131-168)
 * with a complex refractive index m (BHMIE-style lossy sphere,
 * src/mie.f90:99-172); j_n via csphjy and h_n via sphankel
 * (src/sfunctions.f90:342-512). */
static void sbesseljd(int n, zc z, zc *j, zc *dj) {
    zc *csj = (zc *)malloc(sizeof(zc)*(size_t)(n + 1)), *csy = (zc *)malloc(sizeof(zc)*(size_t)(n + 1));
    orc_cspherebessel(n, z, csj, csy);
    for (int i = 1; i <= n; ++i) { j[i - 1] = csj[i]; dj[i - 1] = csj[i - 1] - i*csj[i]/z; }
    free(csj); free(csy);
}
static void shankeljd(int n, zc x, zc *h, zc *dh) {
    zc *H = (zc *)malloc(sizeof(zc)*(size_t)(n + 2));
    H[0] = -CMPLX(0.0, 1.0)*cexp(CMPLX(0.0, 1.0)*x)/x;
    H[1] = (1.0/x - CMPLX(0.0, 1.0))*H[0];
    for (int nn = 2; nn <= n + 1; ++nn) H[nn] = (2.0*nn - 1.0)/x*H[nn - 1] - H[nn - 2];
    for (int i = 1; i <= n; ++i) { h[i - 1] = H[i]; dh[i - 1] = H[i - 1] - i*H[i]/x; }
    free(H);
}
int orc_mie_T(int Nmax, double ka, zc m, zc *a_n, zc *b_n) {
    zc *j0 = (zc *)malloc(sizeof(zc)*(size_t)Nmax), *j0d = (zc *)malloc(sizeof(zc)*(size_t)Nmax);
    zc *j1 = (zc *)malloc(sizeof(zc)*(size_t)Nmax), *j1d = (zc *)malloc(sizeof(zc)*(size_t)Nmax);
    zc *h0 = (zc *)malloc(sizeof(zc)*(size_t)Nmax), *h0d = (zc *)malloc(sizeof(zc)*(size_t)Nmax);
    sbesseljd(Nmax, ka, j0, j0d);
    sbesseljd(Nmax, ka*m, j1, j1d);
    shankeljd(Nmax, ka, h0, h0d);
    for (int j = 0; j < Nmax; ++j) {
        b_n[j] = -(j1d[j]*j0[j] - m*j0d[j]*j1[j])/(j1d[j]*h0[j] - m*h0d[j]*j1[j]);
        a_n[j] = -(j0d[j]*j1[j] - m*j1d[j]*j0[j])/(h0d[j]*j1[j] - m*j1d[j]*h0[j]);
    }
    free(j0); free(j0d); free(j1); free(j1d); free(h0); free(h0d);
    return 0;
}

/* tr_T, src/mie.f90:728-759: orientation-averaged cross sections */
void orc_tr_T(int nm, const zc *Taa, const zc *Tbb, const zc *Tab, const zc *Tba, double k, double crs[4]) {
    double T1 = 0, T2 = 0;
    for (int mu = 0; mu < nm; ++mu) {
        size_t d = mu + (size_t)nm*mu;
        T1 += creal(Taa[d]) + creal(Tbb[d]) + creal(Tab[d]) + creal(Tba[d]);
        for (int nu = 0; nu < nm; ++nu) {
            size_t o = mu + (size_t)nm*nu;
            T2 += cabs(Taa[o])*cabs(Taa[o]) + cabs(Tbb[o])*cabs(Tbb[o]) + cabs(Tab[o])*cabs(Tab[o]) + cabs(Tba[o])*cabs(Tba[o]);
        }
    }
    crs[0] = -2*PI*T1/(k*k);
    crs[1] = 2*PI*T2/(k*k);
    crs[2] = -2*PI*T1/(k*k) - 2*PI*T2/(k*k);
    crs[3] = T1 + T2;
}
