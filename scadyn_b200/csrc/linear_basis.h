// Linear basis (mesh%order = 1) as pseudo-tets.
//
// The reference's linear basis has one projector column per (tet, node) --
// S(27, 4T), all four in the tet's box (pfft_projection_lin,
// src/projection.f90:170-338) -- and 12 unknowns per tet ordered (component,
// node): x(12(t-1) + 4c + i) (compute_Ax2, src/gmres_module.f90:88-95,
// 156-165).  Its far field is therefore the constant-basis far field over 4T
// "pseudo-tets" p = 4(t-1) + i, each with its own projector column and the
// three unknowns (x, y, z) of node i.  Its near zone (matmul_Acorr,
// src/sparse_mat.f90:64-92) holds 12x12 blocks V between tets; block (i, j)
// of V restricted to components, V(4c + i, 4c' + j), is the 3x3 block between
// pseudo-tets 4(t1-1)+i and 4(t2-1)+j.  Between different tets the reference
// also applies V^T, which is the mirrored pseudo-tet block transposed, as for
// constant-basis blocks; inside a tet it applies V alone, so those 16 blocks
// are one-sided.  The device kernels run unchanged on pseudo-tets.
#pragma once
#include <stdint.h>

#include "common.cuh"

// position in the reference's unknown vector of component d of basis
// function (pseudo-tet) p, with nb basis functions per tet (1 or 4)
SCD_HD long long basis_unknown(int nb, long long p, int d) {
    return nb == 1 ? 3 * p + d : 12 * (p >> 2) + 4 * d + (p & 3);
}

// 12x12 blocks (column-major V(r, c), r = 4 component + node) between the
// 1-based tets ind[2b], ind[2b+1] -> 16 pseudo-tet 3x3 blocks each (column-
// major), 1-based pseudo-tet pairs, one_sided[e] = 1 for blocks inside a tet
template <typename ST>
inline void expand_linear_blocks(int64_t B, const ST *sp12, const int32_t *ind, ST *sp3, int32_t *ind3,
                                 unsigned char *one_sided) {
    for (int64_t b = 0; b < B; ++b) {
        const int t1 = ind[2 * b] - 1, t2 = ind[2 * b + 1] - 1;
        const ST *V = sp12 + 144 * b;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) {
                const int64_t e = 16 * b + 4 * i + j;
                ind3[2 * e] = 4 * t1 + i + 1;
                ind3[2 * e + 1] = 4 * t2 + j + 1;
                one_sided[e] = t1 == t2;
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q) sp3[9 * e + r + 3 * q] = V[(4 * r + i) + 12 * (4 * q + j)];
            }
    }
}

// Near-zone groups of one projection box holding n basis functions (nb per
// tet, n a multiple of nb): ceil(tets / (gmax / nb)) runs of whole tets whose
// tet counts differ by at most one.  Writes the run sizes (in basis
// functions) to sizes and returns their number.
inline int split_box(int n, int nb, int gmax, int *sizes) {
    const int tets = n / nb, per = gmax / nb;
    if (tets == 0) return 0;
    const int ng = (tets + per - 1) / per;
    for (int g = 0; g < ng; ++g) sizes[g] = nb * (tets / ng + (g < tets % ng ? 1 : 0));
    return ng;
}
