// Host check of the tensor-core near-zone schedule (scadyn_b200/csrc/near_mma.cuh).
//
// For tiles of several shapes it builds the f16 hi/lo planes and x blocks
// with the same element functions the kernels use, then runs every
// instruction of the row and transposed products through an interpreter of
// the tcgen05 no-swizzle operand descriptors (16-bit elements):
//   K-major : element (m, k) at start + (m/8) SBO + (k/8) LBO + (m%8) 16 + (k%8) 2
//   MN-major: element (m, k) at start + (m/8) SBO + (k/8) LBO + (k%8) 16 + (m%8) 2
// with M = 64 accumulators holding row m in lane (m%16) + 32 (m/16).  These
// readings of the descriptors, negate-A, N sub-ranges and accumulate were
// compared bit-exactly with host products on a B200 before this schedule was
// written.  The emulated epilogue must reproduce the complex products A x and
// A^T x of the tile (complex-symmetric near zone, src/sparse_mat.f90:96-123)
// to FP32 accuracy, and no instruction may read past the tile, its x block
// and the ring slack the kernel reserves.  Exits non-zero on a failure.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ctx.h"
#include "near_mma.cuh"

typedef std::complex<double> zc;

static float h2f(uint16_t b) {
    __half_raw r;
    r.x = b;
    return __half2float(__half(r));
}

struct Image {   // a byte image of shared memory
    std::vector<unsigned char> b;
    uint16_t at(size_t off) const {
        if (off + 2 > b.size()) { printf("read past the image at %zu of %zu\n", off, b.size()); exit(3); }
        uint16_t v;
        memcpy(&v, &b[off], 2);
        return v;
    }
};

// D (TMEM [128 lanes][256 columns]) (+)= op(A) op(B) for one instruction
static void emulate(float (*tm)[256], uint32_t dcol, const Image &A, uint32_t a_start, const Image &B, uint32_t b_start,
                    const NzmOp &o, bool acc) {
    for (int m = 0; m < o.M; ++m) {
        const int lane = o.M == 128 ? m : (m % 16) + 32 * (m / 16);
        for (int n = 0; n < o.N; ++n) {
            float s = 0.f;
            for (int k = 0; k < 16; ++k) {
                const size_t ao = o.a_major == 0
                                      ? a_start + (m / 8) * o.a_sbo + (k / 8) * o.a_lbo + (m % 8) * 16 + (k % 8) * 2
                                      : a_start + (m / 8) * o.a_sbo + (k / 8) * o.a_lbo + (k % 8) * 16 + (m % 8) * 2;
                const size_t bo = b_start + (n / 8) * o.b_sbo + (k / 8) * o.b_lbo + (n % 8) * 16 + (k % 8) * 2;
                float av = h2f(A.at(ao));
                if (o.a_neg) av = -av;
                s += av * h2f(B.at(bo));
            }
            float &d = tm[lane][dcol + n];
            d = acc ? d + s : s;
        }
    }
}

static unsigned rs = 12345u;
static double urand() { rs = rs * 1664525u + 1013904223u; return (rs >> 8) / 16777216.0 - 0.5; }

template <int S>
static int check_tile(int n1, int n2, int rg, bool with_skip) {
    constexpr int R = NzmSched<S>::R;
    // complex64 tile in the k_near_groups layout
    NearTile tl{};
    tl.n1 = n1; tl.n2 = n2; tl.data_off = 0;
    std::vector<float2> data((size_t)tile_elems(n1, n2), make_float2(0.f, 0.f));
    std::vector<zc> A((size_t)9 * n1 * n2);
    float amax = 0.f;
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n2; ++j)
            for (int e = 0; e < 9; ++e) {
                // magnitudes over four decades, as near-zone blocks have
                const double sc = std::pow(10.0, -3.0 * (0.5 + urand()));
                const float2 v = make_float2((float)(sc * urand()), (float)(sc * urand()));
                data[tile_at(n1, i, j, e)] = v;
                A[(size_t)(3 * i + e % 3) * 3 * n2 + 3 * j + e / 3] = zc(v.x, v.y);
                amax = std::max(amax, std::max(std::fabs(v.x), std::fabs(v.y)));
            }
    const float sA = nzm_scale_for(amax);
    // x of both groups: columns of stride n, group 1 at slot 0, group 2 at slot n1
    const long long n = 3LL * (n1 + n2);
    std::vector<float2> x((size_t)R * n);
    for (auto &v : x) v = make_float2((float)urand(), (float)urand());
    std::vector<int> skip(R, 0);
    if (with_skip) skip[3] = skip[rg - 1] = 1;
    float sx[R], xinv[R];
    for (int r = 0; r < R; ++r) {
        float m = 0.f;
        for (long long i = 0; i < n; ++i) m = std::max(m, std::max(std::fabs(x[r * n + i].x), std::fabs(x[r * n + i].y)));
        sx[r] = nzm_scale_for(m);
        xinv[r] = 1.f / (sA * sx[r]);
    }
    // planes, x blocks, images
    const uint32_t tb = nzm_tile_bytes(n1, n2), P = tb / 8;
    auto xblock = [&](int s0, int ng) {
        std::vector<unsigned char> b(nzm_xblock_bytes<S>(ng));
        uint16_t *h = (uint16_t *)b.data();
        for (int e = 0; e < 4 * R * nzm_xk(ng); ++e)
            h[e] = nzm_xblock_bits<S>(x.data(), n, 0, rg, skip.data(), sx, s0, ng, e);
        return b;
    };
    const std::vector<unsigned char> x1 = xblock(0, n1), x2 = xblock(n1, n2);
    const uint32_t slack = (nzm_overrun<S>(n1, n2) + 127u) & ~127u;
    Image slot, X1;
    slot.b.assign(tb + x2.size() + slack, 0);
    for (long long e = 0; e < P; ++e) {
        uint16_t v[4];
        nzm_plane_values(tl, data.data(), sA, e, [](int a, int i, int j, int el) { return tile_at(a, i, j, el); }, v);
        for (int p = 0; p < 4; ++p) memcpy(&slot.b[2 * (p * (size_t)P + e)], &v[p], 2);
    }
    memcpy(&slot.b[tb], x2.data(), x2.size());
    X1.b = x1;
    // reads stay inside the tile + x block + slack the kernel reserves; the
    // B operands stay inside their x block
    for (int use = 0; use < 2; ++use)
        for (int kk = 0; kk < nzm_ksteps(use, n1, n2); ++kk)
            for (int s = 0; s < NzmSched<S>::PARTS; ++s)
                for (int q = 0; q < NZM_OPS; ++q) {
                    const NzmOp o = nzm_op_s<S>(use, n1, n2, kk, s, q);
                    const uint32_t bx = (uint32_t)(use ? x1.size() : x2.size());
                    if (nzm_a_end(o) > tb + slack || nzm_b_end(o) > bx) {
                        printf("(%d,%d) use %d kk %d s %d q %d: A end %u > %u or B end %u > %u\n", n1, n2, use, kk, s, q,
                               nzm_a_end(o), tb + slack, nzm_b_end(o), bx);
                        return 0;
                    }
                    // the kernel advances K step 0's descriptors by constant steps
                    const NzmOp o0 = nzm_op_s<S>(use, n1, n2, 0, s, q);
                    if (o.a_off != o0.a_off + kk * nzm_a_step(use, n2) || o.b_off != o0.b_off + kk * NZM_B_STEP) {
                        printf("(%d,%d) use %d kk %d: operand offsets do not advance by the constant steps\n", n1, n2, use, kk);
                        return 0;
                    }
                }
    static float tm[128][256];
    for (auto &row : tm) for (float &v : row) v = NAN;
    // row product into columns 0.., transposed product into columns DCOLS..
    constexpr int DC = NzmSched<S>::DCOLS;
    for (int use = 0; use < 2; ++use) {
        const uint32_t dcol = use ? DC : 0;
        for (int kk = 0; kk < nzm_ksteps(use, n1, n2); ++kk)
            for (int s = 0; s < NzmSched<S>::PARTS; ++s)
                for (int q = 0; q < NZM_OPS; ++q) {
                    const NzmOp o = nzm_op_s<S>(use, n1, n2, kk, s, q);
                    if (use == 0) emulate(tm, dcol + o.d_col, slot, o.a_off, slot, tb + o.b_off, o, !o.first);
                    else emulate(tm, dcol + o.d_col, slot, o.a_off, X1, o.b_off, o, !o.first);
                }
    }
    // epilogue and reference
    double err = 0, ref = 0;
    for (int use = 0; use < 2; ++use) {
        const int M = nzm_M(use, n1, n2), rows = use ? 3 * n2 : 3 * n1, dcol = use ? DC : 0;
        std::vector<int> seen(rows, 0);
        for (int lane = 0; lane < 128; ++lane) {
            const int row = nzm_row_of_lane(M, lane);
            if (row < 0 || row >= rows) continue;
            ++seen[row];
            for (int r = 0; r < rg; ++r) {
                if (skip[r]) continue;
                const float *d = &tm[lane][dcol];
                const zc got = S == 0 ? zc(d[r] * xinv[r], d[R + r] * xinv[r])
                                      : zc((d[r] + d[R + r]) * xinv[r], (d[2 * R + r] + d[3 * R + r]) * xinv[r]);
                zc want = 0;
                if (use == 0)
                    for (int c = 0; c < 3 * n2; ++c) {
                        const float2 xv = x[r * n + 3LL * n1 + c];
                        want += A[(size_t)row * 3 * n2 + c] * zc(xv.x, xv.y);
                    }
                else
                    for (int c = 0; c < 3 * n1; ++c) {
                        const float2 xv = x[r * n + c];
                        want += A[(size_t)c * 3 * n2 + row] * zc(xv.x, xv.y);
                    }
                err = std::max(err, std::abs(got - want));
                ref = std::max(ref, std::abs(want));
            }
        }
        for (int row = 0; row < rows; ++row)
            if (seen[row] != 1) { printf("(%d,%d) use %d: row %d held by %d lanes\n", n1, n2, use, row, seen[row]); return 0; }
    }
    const double rel = err / ref;
    const bool ok = rel < 2e-6;
    printf("schedule %d  tile %2d x %2d  rg %2d%s  M %3d/%3d  rel err %.2e  slack %u  %s\n", S, n1, n2, rg,
           with_skip ? " skip" : "     ", nzm_M(0, n1, n2), nzm_M(1, n1, n2), rel, slack, ok ? "ok" : "FAIL");
    return ok;
}

int main() {
    const int shapes[][2] = {{1, 1}, {3, 5}, {8, 8}, {17, 11}, {21, 21}, {22, 22}, {24, 24}, {24, 7}, {5, 24}, {13, 22}};
    int bad = 0, n = 0;
    for (auto &sh : shapes)
        for (int v = 0; v < 2; ++v) {
            n += 3;
            bad += !check_tile<0>(sh[0], sh[1], v ? 16 : 7, v == 1);
            bad += !check_tile<1>(sh[0], sh[1], v ? 16 : 7, v == 1);
            bad += !check_tile<2>(sh[0], sh[1], v ? 32 : 19, v == 1);
        }
    uint32_t slack = 0;
    for (int a = 1; a <= SCD_GROUP_MAX; ++a)
        for (int b = 1; b <= SCD_GROUP_MAX; ++b)
            slack = std::max({slack, nzm_overrun<0>(a, b), nzm_overrun<1>(a, b), nzm_overrun<2>(a, b)});
    printf("largest overrun over all shapes: %u bytes\n", slack);
    printf("%d of %d tiles ok\n", n - bad, n);
    return bad ? 1 : 0;
}
