// Host check of where k_near_build_lin writes the linear-basis blocks
// (lin_tile_positions, scadyn_b200/csrc/lin_setup.cuh) and where
// scd_get_nearzone reads them back.
//
// For diagonal and off-diagonal tiles whose tets are in either order, random
// 12x12 blocks V(t, b) (t <= b) are written into dense emulated tiles through
// lin_tile_positions, and the tiles are applied the way the near-zone kernels
// apply them: rows x columns, and for an off-diagonal tile also transposed.
// The result must equal matmul_Acorr (src/sparse_mat.f90:64-92) on the same
// blocks: Ax[t] += V x[b] and, for t != b, Ax[b] += V^T x[t], with unknowns
// 12 t + 4 c + n.  The first written position of every entry must also give
// the entry back (the export).  Exits non-zero on a failure.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <vector>

#include "lin_setup.cuh"

static unsigned rs = 777u;
static double urand() { rs = rs * 1664525u + 1013904223u; return (rs >> 8) / 16777216.0 - 0.5; }

// one tile: row group tets id1, column group tets id2 (original tet ids);
// diag = same group (id1 == id2)
static int check(const std::vector<int> &id1, const std::vector<int> &id2, bool diag) {
    const int nt1 = (int)id1.size(), nt2 = (int)id2.size();
    std::map<std::pair<int, int>, std::vector<double>> V;   // V[(t, b)], t <= b, entry row + 12 col
    int maxid = 0;
    for (int t : id1) maxid = std::max(maxid, t);
    for (int t : id2) maxid = std::max(maxid, t);
    const int n = 12 * (maxid + 1);
    std::vector<double> A((size_t)n * n, 0.0);
    std::vector<double> tile((size_t)4 * nt1 * 4 * nt2 * 9, 0.0);   // [i][j][el]
    auto T = [&](int i, int j, int el) -> double & { return tile[((size_t)i * 4 * nt2 + j) * 9 + el]; };
    for (int p = 0; p < nt1; ++p)
        for (int q = 0; q < nt2; ++q) {
            if (diag && q < p) continue;
            const int ta = id1[p], tb = id2[q];
            const bool fwd = ta <= tb;
            const int t = fwd ? ta : tb, b = fwd ? tb : ta;
            std::vector<double> v(144);
            for (double &x : v) x = urand();
            V[{t, b}] = v;
            // matmul_Acorr
            for (int col = 0; col < 12; ++col)
                for (int row = 0; row < 12; ++row) {
                    A[(size_t)(12 * t + row) * n + 12 * b + col] += v[row + 12 * col];
                    if (t != b) A[(size_t)(12 * b + col) * n + 12 * t + row] += v[row + 12 * col];
                }
            for (int e = 0; e < 144; ++e) {
                int pos[6];
                const int np = lin_tile_positions(diag, fwd, p, q, e, pos);
                for (int w = 0; w < np; ++w) {
                    if (pos[3 * w] >= 4 * nt1 || pos[3 * w + 1] >= 4 * nt2 || pos[3 * w + 2] >= 9) {
                        printf("position out of the tile\n");
                        return 0;
                    }
                    T(pos[3 * w], pos[3 * w + 1], pos[3 * w + 2]) = v[e];
                }
                if (std::fabs(T(pos[0], pos[1], pos[2]) - v[e]) != 0.0) { printf("export mismatch\n"); return 0; }
            }
        }
    // apply the tile to x (pseudo-tet i of the row group: tet id1[i/4], node i%4)
    std::vector<double> x(n), y(n, 0.0), ref(n, 0.0);
    for (double &v : x) v = urand();
    auto unk = [](int tet, int node, int comp) { return 12 * tet + 4 * comp + node; };
    for (int i = 0; i < 4 * nt1; ++i)
        for (int j = 0; j < 4 * nt2; ++j)
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) {
                    const double m = T(i, j, r + 3 * c);
                    y[unk(id1[i / 4], i % 4, r)] += m * x[unk(id2[j / 4], j % 4, c)];
                    if (!diag) y[unk(id2[j / 4], j % 4, c)] += m * x[unk(id1[i / 4], i % 4, r)];
                }
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) ref[a] += A[(size_t)a * n + b] * x[b];
    double err = 0, mag = 0;
    for (int a = 0; a < n; ++a) { err = std::max(err, std::fabs(y[a] - ref[a])); mag = std::max(mag, std::fabs(ref[a])); }
    const bool ok = err <= 1e-12 * mag;
    printf("%s tile %d x %d tets: max err %.2e of %.2e  %s\n", diag ? "diagonal" : "off-diagonal", nt1, nt2, err, mag,
           ok ? "ok" : "FAIL");
    return ok;
}

int main() {
    int good = 0, all = 0;
    // diagonal tiles: tets in increasing order (slots follow the original order inside a box)
    good += check({0, 1, 2, 3, 4, 5}, {0, 1, 2, 3, 4, 5}, true); ++all;
    good += check({2, 7, 11}, {2, 7, 11}, true); ++all;
    good += check({4}, {4}, true); ++all;
    // off-diagonal tiles with the test tet in either group
    good += check({0, 5, 9}, {3, 4, 12}, false); ++all;
    good += check({10, 11}, {1, 2, 3, 20}, false); ++all;
    good += check({1, 2, 3, 4, 5, 6}, {7, 8}, false); ++all;
    printf("%d of %d tiles ok\n", good, all);
    return good == all ? 0 : 1;
}
