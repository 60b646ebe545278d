// Register-resident line FFT for P = 64 and P = 128 (FFTW sign convention:
// forward exp(-i), unnormalised).  A line of P = N1 * 8 points is handled by
// 8 threads: x[n], n = t + 8k (t < 8, k < N1); X[a + N1 b] (a < N1, b < 8)
//   = sum_t w8^(t b) [ w^(t a) sum_k x[t + 8k] w_N1^(k a) ].
// Stage A: thread t forms the N1-point DFT over k in registers and applies
// the twiddles w^(t a); the values are exchanged through the line's buffer
// (position 8a + t); stage B: thread t forms the 8-point DFTs over t of
// a = t*(N1/8) .. t*(N1/8) + N1/8 - 1 and writes X in natural order.  The
// buffer uses the padded index pidx(i) = i + (i >> 4).  Two exchanges per
// transform, both inside one warp (__syncwarp), instead of two block-wide
// barriers per radix-4 stage.
//
// The phases are separate functions so that a host program can run them
// for all threads of a line in order (the device function interleaves them
// with warp barriers).  tw[i] = exp(-2 pi i i / P), i < P.
#pragma once
#include "common.cuh"

SCD_HD int pidx(int i) { return i + (i >> 4); }

template <bool INV, typename C>
SCD_HD C twiddle_of(const C *tw, int i) {
    C w = tw[i];
    if (INV) w.y = -w.y;
    return w;
}

// in-place 4-point DFT, natural order
template <bool INV, typename C>
SCD_HD void dft4(C &v0, C &v1, C &v2, C &v3) {
    C a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), a3 = csub(v1, v3);
    C ia3;                                                 // (-i or +i) * a3
    ia3.x = INV ? -a3.y : a3.y;
    ia3.y = INV ? a3.x : -a3.x;
    v0 = cadd(a0, a2);
    v2 = csub(a0, a2);
    v1 = cadd(a1, ia3);
    v3 = csub(a1, ia3);
}

// 8-point DFT, natural order: t = t2 + 4 t1, b = b1 + 2 b2;
// X[b1 + 2 b2] = sum_t2 w4^(t2 b2) w8^(t2 b1) sum_t1 u[t2 + 4 t1] (-1)^(t1 b1)
template <int P, bool INV, typename C>
SCD_HD void dft8(C (&u)[8], const C *tw) {
    C z[4][2];
#pragma unroll
    for (int t2 = 0; t2 < 4; ++t2) {
        z[t2][0] = cadd(u[t2], u[t2 + 4]);
        z[t2][1] = csub(u[t2], u[t2 + 4]);
        if (t2) z[t2][1] = cmul(z[t2][1], twiddle_of<INV>(tw, t2 * (P / 8)));
    }
#pragma unroll
    for (int b1 = 0; b1 < 2; ++b1) {
        dft4<INV>(z[0][b1], z[1][b1], z[2][b1], z[3][b1]);
#pragma unroll
        for (int b2 = 0; b2 < 4; ++b2) u[b1 + 2 * b2] = z[b2][b1];
    }
}

// 16-point DFT, natural order: k = k2 + 4 k1, a = a1 + 4 a2;
// X[a1 + 4 a2] = sum_k2 w4^(k2 a2) w16^(k2 a1) sum_k1 v[k2 + 4 k1] w4^(k1 a1)
template <int P, bool INV, typename C>
SCD_HD void dft16(C (&v)[16], const C *tw) {
    C z[4][4];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        C a0 = v[k2], a1 = v[k2 + 4], a2 = v[k2 + 8], a3 = v[k2 + 12];
        dft4<INV>(a0, a1, a2, a3);
        z[k2][0] = a0;
        z[k2][1] = k2 ? cmul(a1, twiddle_of<INV>(tw, k2 * 1 * (P / 16))) : a1;
        z[k2][2] = k2 ? cmul(a2, twiddle_of<INV>(tw, k2 * 2 * (P / 16))) : a2;
        z[k2][3] = k2 ? cmul(a3, twiddle_of<INV>(tw, k2 * 3 * (P / 16))) : a3;
    }
#pragma unroll
    for (int a1 = 0; a1 < 4; ++a1) {
        dft4<INV>(z[0][a1], z[1][a1], z[2][a1], z[3][a1]);
#pragma unroll
        for (int a2 = 0; a2 < 4; ++a2) v[a1 + 4 * a2] = z[a2][a1];
    }
}

template <int P> struct RegFft {
    static_assert(P == 64 || P == 128, "register line FFT: P = 64 or 128");
    static constexpr int N2 = 8, N1 = P / 8, PER = N1 / 8;
};

template <int P, bool INV, typename C>
SCD_HD void regfft_dftA(C (&v)[P / 8], const C *tw) {
    if constexpr (P == 128) dft16<P, INV>(v, tw);
    else dft8<P, INV>(v, tw);
}

// stage A for thread t: load, N1-point DFT, twiddles w^(t a)
template <int P, bool INV, typename C>
SCD_HD void regfft_A(const C *s, const C *tw, int t, C (&v)[P / 8]) {
    constexpr int N1 = P / 8;
#pragma unroll
    for (int k = 0; k < N1; ++k) v[k] = s[pidx(t + 8 * k)];
    regfft_dftA<P, INV>(v, tw);
#pragma unroll
    for (int a = 1; a < N1; ++a)
        if (t) v[a] = cmul(v[a], twiddle_of<INV>(tw, t * a));
}

template <int P, typename C>
SCD_HD void regfft_A_store(C *s, int t, const C (&v)[P / 8]) {
#pragma unroll
    for (int a = 0; a < P / 8; ++a) s[pidx(8 * a + t)] = v[a];
}

// stage B for thread t: the 8-point DFTs over t of its PER values of a
template <int P, bool INV, typename C>
SCD_HD void regfft_B(const C *s, const C *tw, int t, C (&u)[RegFft<P>::PER][8]) {
    constexpr int PER = RegFft<P>::PER;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int a = t * PER + p;
#pragma unroll
        for (int m = 0; m < 8; ++m) u[p][m] = s[pidx(8 * a + m)];
        dft8<P, INV>(u[p], tw);
    }
}

template <int P, typename C>
SCD_HD void regfft_B_store(C *s, int t, const C (&u)[RegFft<P>::PER][8]) {
    constexpr int PER = RegFft<P>::PER, N1 = P / 8;
#pragma unroll
    for (int p = 0; p < PER; ++p)
#pragma unroll
        for (int b = 0; b < 8; ++b) s[pidx(t * PER + p + N1 * b)] = u[p][b];
}

#ifdef __CUDACC__
// the whole transform of one line held in s by its 8 threads (t = 0..7,
// all in one warp)
template <int P, bool INV, typename C>
__device__ __forceinline__ void fft_line_reg(C *s, const C *tw, int t) {
    C v[P / 8];
    regfft_A<P, INV>(s, tw, t, v);
    __syncwarp();
    regfft_A_store<P>(s, t, v);
    __syncwarp();
    C u[RegFft<P>::PER][8];
    regfft_B<P, INV>(s, tw, t, u);
    __syncwarp();
    regfft_B_store<P>(s, t, u);
    __syncwarp();
}
#endif
