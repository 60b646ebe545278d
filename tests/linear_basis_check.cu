// Host check of the linear-basis pseudo-tet mapping (scadyn_b200/csrc/linear_basis.h):
// the 3x3 blocks expand_linear_blocks makes from 12x12 blocks, placed between
// pseudo-tets with their mirror only between different tets, rebuild the
// near-zone matrix of matmul_Acorr (src/sparse_mat.f90:64-92) in the order
// basis_unknown gives.  Exits non-zero on a mismatch.
#include <complex>
#include <cstdio>
#include <vector>

#include "linear_basis.h"

typedef std::complex<double> zc;

int main() {
    const int T = 5;                                   // tets
    const int32_t ind[] = {1, 1, 1, 3, 2, 5, 4, 4, 3, 5, 5, 5, 2, 2};
    const int B = sizeof(ind) / sizeof(ind[0]) / 2;
    std::vector<double2> sp12((size_t)144 * B);
    unsigned st = 7u;
    for (auto &v : sp12) {
        st = st * 1664525u + 1013904223u; v.x = (st >> 8) / 16777216.0 - 0.5;
        st = st * 1664525u + 1013904223u; v.y = (st >> 8) / 16777216.0 - 0.5;
    }
    const int n = 12 * T;
    std::vector<zc> A((size_t)n * n, 0.0), P((size_t)n * n, 0.0);
    // matmul_Acorr: Ax[a] += V x[b]; if a != b, Ax[b] += V^T x[a]
    for (int b = 0; b < B; ++b) {
        const int a0 = 12 * (ind[2 * b] - 1), b0 = 12 * (ind[2 * b + 1] - 1);
        for (int r = 0; r < 12; ++r)
            for (int c = 0; c < 12; ++c) {
                const double2 v = sp12[144 * b + r + 12 * c];
                A[(size_t)(a0 + r) * n + b0 + c] += zc(v.x, v.y);
                if (a0 != b0) A[(size_t)(b0 + c) * n + a0 + r] += zc(v.x, v.y);
            }
    }
    std::vector<double2> sp3((size_t)144 * B);
    std::vector<int32_t> ind3((size_t)32 * B);
    std::vector<unsigned char> one((size_t)16 * B);
    expand_linear_blocks<double2>(B, sp12.data(), ind, sp3.data(), ind3.data(), one.data());
    for (int e = 0; e < 16 * B; ++e) {
        const int p = ind3[2 * e] - 1, q = ind3[2 * e + 1] - 1;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                const double2 v = sp3[9 * e + r + 3 * c];
                P[(size_t)(3 * p + r) * n + 3 * q + c] += zc(v.x, v.y);
                if (p != q && !one[e]) P[(size_t)(3 * q + c) * n + 3 * p + r] += zc(v.x, v.y);
            }
    }
    int bad = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            const long long oi = basis_unknown(4, i / 3, i % 3), oj = basis_unknown(4, j / 3, j % 3);
            if (P[(size_t)i * n + j] != A[(size_t)oi * n + oj]) ++bad;
        }
    // basis_unknown is a bijection of 0..12T-1
    std::vector<int> hit(n, 0);
    for (int p = 0; p < 4 * T; ++p)
        for (int d = 0; d < 3; ++d) hit[basis_unknown(4, p, d)]++;
    for (int i = 0; i < n; ++i) bad += hit[i] != 1;
    printf("linear basis mapping: %d mismatches\n", bad);
    return bad ? 1 : 0;
}
