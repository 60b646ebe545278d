// Geometry helpers and quadrature tables shared by the device set-up
// kernels (setup_device.cu) and host programs that check them.
//
// The quadrature rules are the published ones the reference tabulates
// (src/integration_points.f90): Keast's 24-point tetrahedron rule, the 7-point
// degree-5 triangle rule and the 98 surface nodes of the 5x5x5 lattice on
// [-1,1]^3 (sample_points_cube, src/integration_points.f90:503-805), in the
// reference's point order.
#pragma once
#include <cmath>
#include <cstring>

#include "common.cuh"

constexpr double PI = 3.141592653589793;            // src/common.f90:20
constexpr double F13_D = (double)(1.0f / 3.0f);     // Fortran default-real 1.0/3.0

struct V3 { double x, y, z; };
SCD_HD V3 vsub(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
SCD_HD double vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SCD_HD V3 vcross(V3 a, V3 b) { return V3{a.y * b.z - a.z * b.y, -a.x * b.z + a.z * b.x, a.x * b.y - a.y * b.x}; }
SCD_HD double vdist(V3 r, V3 p) {
    const double a = r.x - p.x, b = r.y - p.y, c = r.z - p.z;
    return sqrt(a * a + b * b + c * c);
}
SCD_HD double tet_vol(const V3 *t) {
    const V3 cr = vcross(vsub(t[1], t[0]), vsub(t[2], t[0]));
    const double dt = vdot(vsub(t[3], t[0]), cr);
    return sqrt(dt * dt) / 6.0;
}
SCD_HD V3 tri_normal(const V3 *tri) {
    const V3 c = vcross(vsub(tri[1], tri[0]), vsub(tri[2], tri[0]));
    const double l = sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
    return V3{c.x / l, c.y / l, c.z / l};
}
// linmap_tri weight factor: twice the triangle area (src/common.f90:1381-1408)
SCD_HD double tri_ww1(const V3 *tri, V3 &a, V3 &b) {
    a = vsub(tri[1], tri[0]);
    b = vsub(tri[2], tri[0]);
    const double aa = a.x * a.x + a.y * a.y + a.z * a.z;
    const double ww0 = aa * b.x, ww1 = aa * b.y, ww2 = aa * b.z;
    const double ab = a.x * b.x + a.y * b.y + a.z * b.z;
    return sqrt((ww0 * b.x + ww1 * b.y + ww2 * b.z) - ab * ab);
}
// faces opposite vertex 1..4 (tetra_face, src/common.f90:296-322): vertex i of face f
SCD_HD int face_vertex(int f, int i) {
    // nibbles, face-major: (1,2,3) (0,3,2) (0,1,3) (0,2,1)
    const unsigned long long tab = 0x123032013021ULL;
    return (int)((tab >> (4 * (11 - (3 * f + i)))) & 0xF);
}

// tables on the host: t5[i] = (xi, eta, zeta, w), r5[i] = (xi, eta, w), ps = cube samples
struct HostQuad {
    double t5[24][4];
    double r5[7][3];
    double ps[98][3];
    HostQuad() {
        const double A[3][2] = {{3.561913862225449e-01, 2.146028712591517e-01},
                                {8.779781243961660e-01, 4.067395853461134e-02},
                                {3.298632957317306e-02, 3.223378901422757e-01}};
        const double W4[3] = {6.653791709694644e-03, 1.679535175886776e-03, 9.226196923942397e-03};
        int p = 0;
        for (int o = 0; o < 3; ++o) {
            const double a = A[o][0], b = A[o][1];
            const double pts[4][3] = {{a, b, b}, {b, b, b}, {b, b, a}, {b, a, b}};
            for (int i = 0; i < 4; ++i, ++p) {
                t5[p][0] = pts[i][0]; t5[p][1] = pts[i][1]; t5[p][2] = pts[i][2]; t5[p][3] = W4[o];
            }
        }
        const double c = 6.366100187501753e-02, d = 2.696723314583159e-01, e = 6.030056647916491e-01;
        const double p12[12][3] = {{d, c, c}, {c, d, c}, {c, c, d}, {e, c, c}, {c, e, c}, {c, c, e},
                                   {c, d, e}, {d, e, c}, {e, c, d}, {c, e, d}, {d, c, e}, {e, d, c}};
        for (int i = 0; i < 12; ++i, ++p) {
            t5[p][0] = p12[i][0]; t5[p][1] = p12[i][1]; t5[p][2] = p12[i][2]; t5[p][3] = 8.035714285714281e-03;
        }
        const double t0 = 3.333333333333330e-01, a1 = 5.971587178977000e-02, b1 = 4.701420641051150e-01;
        const double a2 = 7.974269853530870e-01, b2 = 1.012865073234560e-01;
        const double w1 = 6.619707639425300e-02, w2 = 6.296959027241350e-02;
        const double tri[7][3] = {{t0, t0, 1.125000000000000e-01}, {a1, b1, w1}, {b1, b1, w1}, {b1, a1, w1},
                                  {a2, b2, w2}, {b2, b2, w2}, {b2, a2, w2}};
        std::memcpy(r5, tri, sizeof tri);
        const double v[5] = {-1.0, -0.5, 0.0, 0.5, 1.0};
        int n = 0;
        auto put = [&](double x, double y, double z) { ps[n][0] = x; ps[n][1] = y; ps[n][2] = z; ++n; };
        for (int iy = 4; iy >= 0; --iy) for (int ix = 0; ix < 5; ++ix) put(v[ix], v[iy], -1.0);
        for (int iy = 0; iy < 5; ++iy) for (int ix = 0; ix < 5; ++ix) put(v[ix], v[iy], 1.0);
        for (int iz = 1; iz <= 3; ++iz) for (int ix = 0; ix < 5; ++ix) put(v[ix], -1.0, v[iz]);
        for (int iz = 3; iz >= 1; --iz) for (int ix = 0; ix < 5; ++ix) put(v[ix], 1.0, v[iz]);
        for (int iz = 1; iz <= 3; ++iz) for (int iy = 3; iy >= 1; --iy) put(-1.0, v[iy], v[iz]);
        for (int iz = 1; iz <= 3; ++iz) for (int iy = 1; iy <= 3; ++iy) put(1.0, v[iy], v[iz]);
    }
};
