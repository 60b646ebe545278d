// Near-zone tile products on the tensor cores (tcgen05.mma kind::f16, FP32
// accumulate in tensor memory): layouts and the instruction schedule, shared
// by the device kernels (near_mma.cu) and a host emulation of the schedule.
//
// A tile couples group g1 (n1 tets, rows 3i + a) to group g2 (n2 tets,
// columns 3j + b); its value A(row, col) is complex.  With a power-of-two
// scale sA the real and imaginary parts are split into f16 pairs,
// A * sA = hi + lo (hi = f16(v), lo = f16(v - hi)), which keeps about 22
// significant bits: the product is as accurate as the complex64 storage it is
// built from.  x is split the same way with a per-right-hand-side scale, and
//   A x ~ hi(A) hi(x) + hi(A) lo(x) + lo(A) hi(x)
// (the lo * lo term is below the FP32 accumulation error).
//
// Operand layouts are the no-swizzle canonical forms of tcgen05 matrix
// descriptors for 16-bit types: 8 x 8 "core matrices" of 8 rows by 16 bytes.
// A plane (rows x cols) stores element (r, c) at nzm_cidx(r, c, cols8):
// cores in (r/8, c/8) order, row-major inside a core.  Read as a K-major
// operand (M = row, K = col; leading offset 128 B between the two 8-column
// cores of a 16-wide K step, stride offset 16*cols8 B between 8-row groups)
// it is A; read as an MN-major operand (M = col, K = row; stride offset
// 128 B between 8-column groups, leading offset 16*cols8 B between 8-row
// groups) it is A^T.  Both readings of the same bytes were checked on a
// B200 for f16 and bf16; kind::tf32 returns zeros for MN-major operands, so
// the 16-bit split is what lets one stored tile serve both products.
#pragma once
#include <cuda_fp16.h>
#include <stdint.h>

#include "common.cuh"

constexpr int NZM_R = 16;              // right-hand sides per pass of schedules 0 and 1
constexpr int NZM_RMAX = 32;           // right-hand sides per pass of schedule 2
constexpr int NZM_N = 2 * NZM_R;       // schedule 0: x-block rows per half (Re x, then Im x)
constexpr int NZM_SPLITS = 3;          // schedule 0: (hi A, hi x), (hi A, lo x), (lo A, hi x)
constexpr int NZM_OPS = 3;             // per A part: Re A X, -Im A Im x, Im A Re x

// Three instruction schedules over the same tile planes:
//  0 ("split"): the x block is a hi half then a lo half, each of NZM_N rows
//    (Re x_r, then Im x_r); per K step 3 splits x 3 ops; accumulator
//    columns [Re y_r | Im y_r].
//  1 ("merged"): the x block is one block of 4R rows (Re x hi, Re x lo,
//    Im x hi, Im x lo); per K step 2 A parts (hi, lo) x 3 ops, each over both
//    x halves at once (6 instead of 9 instructions; lo A lo x is included);
//    accumulator columns [Re y (x hi) | Re y (x lo) | Im y (x hi) | Im y (x lo)],
//    summed pairwise by the epilogue.  Descriptors advance by constant steps.
//  2 ("wide"): schedule 1 with R = 32 right-hand sides per pass: every tile
//    crosses HBM once per 32 right-hand sides instead of 16, with N = 128
//    instructions.  With one buffer for the transposed products (NBUF 1) the
//    row and transposed accumulators take 256 TMEM columns and two CTAs share
//    an SM, one overlapping the other's epilogue; with two (NBUF 2) they take
//    384 of the SM's 512 and one CTA runs per SM.
// NBUF: accumulator buffers of the transposed products; CTAS: CTAs per SM.
#ifndef NZM_WIDE_NB
#define NZM_WIDE_NB 1
#endif
template <int S> struct NzmSched;
template <> struct NzmSched<0> {
    static constexpr int R = NZM_R, PARTS = NZM_SPLITS, DCOLS = 2 * R, NBUF = 2, TMEM = 128, CTAS = 2;
};
template <> struct NzmSched<1> {
    static constexpr int R = NZM_R, PARTS = 2, DCOLS = 4 * R, NBUF = 2, TMEM = 256, CTAS = 2;
};
template <> struct NzmSched<2> {
    static constexpr int R = NZM_RMAX, PARTS = 2, DCOLS = 4 * R, NBUF = NZM_WIDE_NB,
                         TMEM = NZM_WIDE_NB == 1 ? 256 : 512, CTAS = NZM_WIDE_NB == 1 ? 2 : 1;
};

SCD_HD int nzm_ceil8(int v) { return (v + 7) & ~7; }
SCD_HD int nzm_ceil16(int v) { return (v + 15) & ~15; }

// element (r, c) of a 16-bit canonical plane with cols8 (multiple of 8) columns, in halves
SCD_HD long long nzm_cidx(int r, int c, int cols8) {
    return ((((long long)(r >> 3) * (cols8 >> 3) + (c >> 3)) << 6) + ((r & 7) << 3) + (c & 7));
}

// inverse of nzm_cidx: position e (halves, memory order) of a plane with
// cols8 columns -> (row, col)
SCD_HD void nzm_cpos(long long e, int cols8, int &r, int &c) {
    const long long core = e >> 6;
    r = 8 * (int)(core / (cols8 >> 3)) + (int)((e >> 3) & 7);
    c = 8 * (int)(core % (cols8 >> 3)) + (int)(e & 7);
}

// v = hi + lo in f16 (round to nearest), raw bits
SCD_HD void nzm_split(float v, uint16_t &hi, uint16_t &lo) {
    const __half h = __float2half_rn(v);
    const __half l = __float2half_rn(v - __half2float(h));
    hi = ((__half_raw)h).x;
    lo = ((__half_raw)l).x;
}

// power of two that brings a largest magnitude m to [2^13, 2^14)
SCD_HD float nzm_scale_for(float m) {
    if (!(m > 0.f) || !(m <= 3.0e38f)) return 1.f;
    int e;
    frexpf(m, &e);                 // m = f 2^e, f in [0.5, 1)
    return ldexpf(1.f, 14 - e);
}

// ---- tiles: four planes [Re hi, Im hi, Re lo, Im lo], each R1 x C1 halves,
//      R1 = ceil8(3 n1), C1 = ceil8(3 n2), zero outside 3n1 x 3n2
SCD_HD int nzm_rows8(int n1) { return nzm_ceil8(3 * n1); }
SCD_HD int nzm_cols8(int n2) { return nzm_ceil8(3 * n2); }
SCD_HD uint32_t nzm_plane_bytes(int n1, int n2) { return 2u * (uint32_t)nzm_rows8(n1) * (uint32_t)nzm_cols8(n2); }
SCD_HD uint32_t nzm_tile_bytes(int n1, int n2) { return 4u * nzm_plane_bytes(n1, n2); }

// the four plane values at position e of tile tl (complex64 blocks at
// data[tl.data_off + tile_at(...)], the layout of k_near_groups): out =
// {Re hi, Im hi, Re lo, Im lo} of sA * A(row, col), zero outside 3n1 x 3n2
template <typename Tile, typename AtFn>
SCD_HD void nzm_plane_values(const Tile &tl, const float2 *data, float sA, long long e, AtFn at, uint16_t (&out)[4]) {
    int row, col;
    nzm_cpos(e, nzm_cols8(tl.n2), row, col);
    float2 v = make_float2(0.f, 0.f);
    if (row < 3 * tl.n1 && col < 3 * tl.n2) {
        const int i = row / 3, ra = row - 3 * i, j = col / 3, cb = col - 3 * j;
        v = data[tl.data_off + at(tl.n1, i, j, ra + 3 * cb)];
    }
    nzm_split(v.x * sA, out[0], out[2]);
    nzm_split(v.y * sA, out[1], out[3]);
}

// ---- x blocks: per group (n tets) and pass, a K-major B operand of NZM_N
//      rows (Re x_r, r < 16, then Im x_r) by K16 = ceil16(3n) unknowns, hi block
//      then lo block, zero for unknowns >= 3n and for absent right-hand sides
//      (schedule 0); 4R rows by K16 (schedules 1 and 2)
SCD_HD int nzm_xk(int n) { return nzm_ceil16(3 * n); }
SCD_HD uint32_t nzm_xhalf_bytes(int n) { return 2u * NZM_N * (uint32_t)nzm_xk(n); }
template <int S = 0>
SCD_HD uint32_t nzm_xblock_bytes(int n) { return 8u * (uint32_t)NzmSched<S>::R * (uint32_t)nzm_xk(n); }
// element (row, k) of the hi (or lo) block, in halves
SCD_HD long long nzm_xidx(int row, int k, int n) { return nzm_cidx(row, k, nzm_xk(n)); }

// value at position e of a group's x block (before the split): group of ng
// tets from slot s0, right-hand sides r0 .. r0 + rg - 1 of x (columns of
// stride n), scale sx[r]
SCD_HD float nzm_xblock_value(const float2 *x, long long n, int r0, int rg, const int *skip, const float *sx, int s0,
                              int ng, int e) {
    int row, k;
    nzm_cpos(e, nzm_xk(ng), row, k);
    const int r = row % NZM_R, im = row / NZM_R;
    if (r >= rg || k >= 3 * ng || (skip && skip[r0 + r])) return 0.f;
    const float2 xv = x[(long long)(r0 + r) * n + 3LL * s0 + k];
    return (im ? xv.y : xv.x) * sx[r];
}

// f16 bits at position e (halves, 0 <= e < 4 R K16) of a group's x block in
// schedule S's layout (sx holds the pass's R scales)
template <int S>
SCD_HD uint16_t nzm_xblock_bits(const float2 *x, long long n, int r0, int rg, const int *skip, const float *sx, int s0,
                                int ng, int e) {
    const int K = nzm_xk(ng);
    uint16_t hi, lo;
    if constexpr (S == 0) {
        const int half = e / (NZM_N * K);
        nzm_split(nzm_xblock_value(x, n, r0, rg, skip, sx, s0, ng, e - half * NZM_N * K), hi, lo);
        return half ? lo : hi;
    } else {
        constexpr int R = NzmSched<S>::R;
        int row, k;
        nzm_cpos(e, K, row, k);
        const int part = row / R, r = row % R, im = part >> 1, want_lo = part & 1;
        float v = 0.f;
        if (r < rg && k < 3 * ng && !(skip && skip[r0 + r])) {
            const float2 xv = x[(long long)(r0 + r) * n + 3LL * s0 + k];
            v = (im ? xv.y : xv.x) * sx[r];
        }
        nzm_split(v, hi, lo);
        return want_lo ? lo : hi;
    }
}

// ---- products: use 0 = row product D (3n1 rows) += A x(g2), K over 3n2,
//      tile read K-major; use 1 = transposed product D (3n2 rows) = A^T x(g1),
//      K over 3n1, tile read MN-major.  Accumulator columns: [Re y_r | Im y_r].
SCD_HD int nzm_ksteps(int use, int n1, int n2) { return nzm_xk(use ? n1 : n2) / 16; }
SCD_HD int nzm_M(int use, int n1, int n2) { return 3 * (use ? n2 : n1) <= 64 ? 64 : 128; }

struct NzmOp {
    uint32_t a_off, a_lbo, a_sbo;   // bytes; a_off from the tile start
    uint32_t b_off, b_lbo, b_sbo;   // bytes; b_off from the x block start
    int M, N, a_major, a_neg, d_col;
    int first;                      // first instruction of the product: overwrite instead of accumulate
};

// instruction (kk, s, q) of a product in schedules 1 and 2 (R right-hand
// sides): K step kk, A part s (0 hi, 1 lo), op q
//   q 0: D[:, 0:4R)  += Re A * X[0:4R)     (Re and Im of x, hi and lo halves)
//   q 1: D[:, 0:2R)  += -Im A * X[2R:4R)   (Re y gets -Im A Im x)
//   q 2: D[:, 2R:4R) += Im A * X[0:2R)     (Im y gets Im A Re x)
template <int R>
SCD_HD NzmOp nzm_op_merged(int use, int n1, int n2, int kk, int s, int q) {
    const uint32_t C1 = (uint32_t)nzm_cols8(n2);
    const uint32_t plane = nzm_plane_bytes(n1, n2);
    const int im = q != 0;
    NzmOp o;
    const uint32_t pbase = plane * (uint32_t)(2 * s + im);
    if (use == 0) {
        o.a_off = pbase + 256u * kk; o.a_lbo = 128u; o.a_sbo = 16u * C1; o.a_major = 0;
    } else {
        o.a_off = pbase + 32u * C1 * kk; o.a_lbo = 16u * C1; o.a_sbo = 128u; o.a_major = 1;
    }
    const uint32_t xsbo = 16u * (uint32_t)nzm_xk(use ? n1 : n2);
    const uint32_t xbase = 256u * kk;
    o.b_lbo = 128u; o.b_sbo = xsbo;
    if (q == 0) { o.b_off = xbase; o.N = 4 * R; o.d_col = 0; o.a_neg = 0; }
    else if (q == 1) { o.b_off = xbase + (2 * R / 8) * xsbo; o.N = 2 * R; o.d_col = 0; o.a_neg = 1; }
    else { o.b_off = xbase; o.N = 2 * R; o.d_col = 2 * R; o.a_neg = 0; }
    o.M = nzm_M(use, n1, n2);
    o.first = kk == 0 && s == 0 && q == 0;
    return o;
}

// bytes an operand start advances per K step (the same for every instruction of a product)
SCD_HD uint32_t nzm_a_step(int use, int n2) { return use ? 32u * (uint32_t)nzm_cols8(n2) : 256u; }
constexpr uint32_t NZM_B_STEP = 256u;

// instruction (kk, s, q) of a product in schedule 0: K step kk (16 wide), split s, op q
//   q 0: D[:, 0:2R) += Re A * X[0:2R)      (Re y gets Re A Re x, Im y gets Re A Im x)
//   q 1: D[:, 0:R)  += -Im A * X[R:2R)     (Re y gets -Im A Im x)
//   q 2: D[:, R:2R) += Im A * X[0:R)       (Im y gets Im A Re x)
SCD_HD NzmOp nzm_op(int use, int n1, int n2, int kk, int s, int q) {
    const uint32_t C1 = (uint32_t)nzm_cols8(n2);
    const uint32_t plane = nzm_plane_bytes(n1, n2);
    const int a_lo = s == 2, x_lo = s == 1, im = q != 0;
    NzmOp o;
    const uint32_t pbase = plane * (uint32_t)(2 * a_lo + im);
    if (use == 0) {
        o.a_off = pbase + 256u * kk; o.a_lbo = 128u; o.a_sbo = 16u * C1; o.a_major = 0;
    } else {
        o.a_off = pbase + 32u * C1 * kk; o.a_lbo = 16u * C1; o.a_sbo = 128u; o.a_major = 1;
    }
    const int nx = use ? n1 : n2;
    const uint32_t xsbo = 16u * (uint32_t)nzm_xk(nx);
    const uint32_t xbase = nzm_xhalf_bytes(nx) * (uint32_t)x_lo + 256u * kk;
    o.b_lbo = 128u; o.b_sbo = xsbo;
    if (q == 0) { o.b_off = xbase; o.N = NZM_N; o.d_col = 0; o.a_neg = 0; }
    else if (q == 1) { o.b_off = xbase + (NZM_R / 8) * xsbo; o.N = NZM_R; o.d_col = 0; o.a_neg = 1; }
    else { o.b_off = xbase; o.N = NZM_R; o.d_col = NZM_R; o.a_neg = 0; }
    o.M = nzm_M(use, n1, n2);
    o.first = kk == 0 && s == 0 && q == 0;
    return o;
}

template <int S>
SCD_HD NzmOp nzm_op_s(int use, int n1, int n2, int kk, int s, int q) {
    if constexpr (S == 0) return nzm_op(use, n1, n2, kk, s, q);
    else return nzm_op_merged<NzmSched<S>::R>(use, n1, n2, kk, s, q);
}

// last byte (exclusive) an instruction reads, relative to its operand start
SCD_HD uint32_t nzm_a_end(const NzmOp &o) { return o.a_off + (uint32_t)(o.M / 8 - 1) * o.a_sbo + o.a_lbo + 128u; }
SCD_HD uint32_t nzm_b_end(const NzmOp &o) { return o.b_off + (uint32_t)(o.N / 8 - 1) * o.b_sbo + o.b_lbo + 128u; }

// bytes past a tile's end that its products may read (rows beyond 3n1 / 3n2
// up to M and the 8 columns of a half-filled K step): the ring keeps that
// much zeroed slack after its end
template <int S = 0>
SCD_HD uint32_t nzm_overrun(int n1, int n2) {
    uint32_t end = 0;
    for (int use = 0; use < 2; ++use) {
        const int ks = nzm_ksteps(use, n1, n2);
        for (int s = 0; s < NzmSched<S>::PARTS; ++s)
            for (int q = 0; q < NZM_OPS; ++q) {
                const uint32_t e = nzm_a_end(nzm_op_s<S>(use, n1, n2, ks - 1, s, q));
                end = e > end ? e : end;
            }
    }
    const uint32_t tb = nzm_tile_bytes(n1, n2);
    return end > tb ? end - tb : 0u;
}

// accumulator row held by TMEM lane `lane` (0..127) for an M-row product;
// -1 for lanes an M = 64 product leaves unused
SCD_HD int nzm_row_of_lane(int M, int lane) {
    if (M == 128) return lane;
    return (lane & 31) < 16 ? 16 * (lane >> 5) + (lane & 15) : -1;
}

// 32-bit instruction descriptor of kind::f16 with f16 operands, FP32 accumulator
SCD_HD uint32_t nzm_idesc(const NzmOp &o) {
    return (1u << 4) | ((uint32_t)o.a_neg << 13) | ((uint32_t)o.a_major << 15) | ((uint32_t)(o.N >> 3) << 17) |
           ((uint32_t)(o.M >> 4) << 24);
}
// shared-memory matrix descriptor (no swizzle)
SCD_HD uint64_t nzm_sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
