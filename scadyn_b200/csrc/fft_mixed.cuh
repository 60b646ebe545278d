// Register line FFT for 5-smooth lengths P = T * N1 (T threads per line,
// T in {4, 8}, T | N1), FFTW sign convention (forward exp(-i),
// unnormalised), used for padded FFT lengths that are not 64 or 128.
//
// x[n], n = t + T k (t < T, k < N1);  X[a + N1 b] (a < N1, b < T)
//   = sum_t w_T^(t b) [ w_P^(t a) sum_k x[t + T k] w_N1^(k a) ].
// Stage A: thread t forms the N1-point DFT over k in registers (mixed radix
// 4/2/3/5, recursive decimation in time, twiddles read from the line's
// table tw[i] = exp(-2 pi i i / P)), then multiplies by w_P^(t a) and stores
// at position T a + t of the line buffer; stage B: thread t forms the T-point
// DFTs over t of a = t PER .. t PER + PER - 1 (PER = N1 / T) and writes X in
// natural order.  The buffer uses the padded index pidx(i) = i + (i >> 4).
// The phases are separate functions, so a host program can run the T
// threads of a line in order.
#pragma once
#include "common.cuh"
#include "fft_reg.cuh"

// exp(-/+ 2 pi i e / N) for an N dividing P, from the P-point table
template <int P, int N, bool INV, typename C>
SCD_HD C tw_n(const C *tw, int e) {
    static_assert(P % N == 0, "twiddle table");
    return twiddle_of<INV>(tw, (e % N) * (P / N));
}

template <int N> struct FirstRadix {
    static constexpr int r = N % 4 == 0 && N != 8 ? 4 : N % 2 == 0 ? 2 : N % 3 == 0 ? 3 : N % 5 == 0 ? 5 : 0;
};

// in-place DFT of length N (natural order) for N = 2^a 3^b 5^c, on v[off + stride*m], m < N
template <int P, int N, bool INV, typename C, int LEN>
SCD_HD void dft_mixed(C (&v)[LEN], int off, int stride, const C *tw) {
    if constexpr (N == 1) {
        return;
    } else if constexpr (N == 2) {
        const C a = v[off], b = v[off + stride];
        v[off] = cadd(a, b);
        v[off + stride] = csub(a, b);
    } else if constexpr (N == 4) {
        dft4<INV>(v[off], v[off + stride], v[off + 2 * stride], v[off + 3 * stride]);
    } else if constexpr (N == 3 || N == 5) {
        // direct sum (small prime radix)
        C x[N], y[N];
#pragma unroll
        for (int j = 0; j < N; ++j) x[j] = v[off + j * stride];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            C s = x[0];
#pragma unroll
            for (int j = 1; j < N; ++j) s = cadd(s, cmul(x[j], tw_n<P, N, INV>(tw, j * k)));
            y[k] = s;
        }
#pragma unroll
        for (int k = 0; k < N; ++k) v[off + k * stride] = y[k];
    } else {
        constexpr int R = FirstRadix<N>::r;
        static_assert(R != 0, "length must be 5-smooth");
        constexpr int M = N / R;
        // sub-DFTs of length M over the residues j: elements j + R m
        C t[N];
#pragma unroll
        for (int j = 0; j < R; ++j)
#pragma unroll
            for (int m = 0; m < M; ++m) t[j * M + m] = v[off + (j + R * m) * stride];
#pragma unroll
        for (int j = 0; j < R; ++j) dft_mixed<P, M, INV>(t, j * M, 1, tw);
        // twiddles w_N^(j k1), then R-point DFTs across j
#pragma unroll
        for (int j = 1; j < R; ++j)
#pragma unroll
            for (int k1 = 1; k1 < M; ++k1) t[j * M + k1] = cmul(t[j * M + k1], tw_n<P, N, INV>(tw, j * k1));
#pragma unroll
        for (int k1 = 0; k1 < M; ++k1) {
            C u[R];
#pragma unroll
            for (int j = 0; j < R; ++j) u[j] = t[j * M + k1];
            dft_mixed<P, R, INV>(u, 0, 1, tw);
#pragma unroll
            for (int k2 = 0; k2 < R; ++k2) v[off + (k1 + M * k2) * stride] = u[k2];
        }
    }
}

template <int P, int T> struct MixFft {
    static_assert(T == 4 || T == 8, "threads per line");
    static constexpr int N1 = P / T, PER = N1 / T;
    static_assert(N1 * T == P && PER * T == N1, "P = T * N1 with T | N1");
};

// stage A for thread t: load, N1-point DFT, twiddles w_P^(t a)
template <int P, int T, bool INV, typename C>
SCD_HD void mixfft_A(const C *s, const C *tw, int t, C (&v)[P / T]) {
    constexpr int N1 = P / T;
#pragma unroll
    for (int k = 0; k < N1; ++k) v[k] = s[pidx(t + T * k)];
    dft_mixed<P, N1, INV>(v, 0, 1, tw);
#pragma unroll
    for (int a = 1; a < N1; ++a)
        if (t) v[a] = cmul(v[a], twiddle_of<INV>(tw, t * a));
}

template <int P, int T, typename C>
SCD_HD void mixfft_A_store(C *s, int t, const C (&v)[P / T]) {
#pragma unroll
    for (int a = 0; a < P / T; ++a) s[pidx(T * a + t)] = v[a];
}

// stage B for thread t: the T-point DFTs over t of its PER values of a
template <int P, int T, bool INV, typename C>
SCD_HD void mixfft_B(const C *s, const C *tw, int t, C (&u)[MixFft<P, T>::PER][T]) {
    constexpr int PER = MixFft<P, T>::PER;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int a = t * PER + p;
#pragma unroll
        for (int m = 0; m < T; ++m) u[p][m] = s[pidx(T * a + m)];
        dft_mixed<P, T, INV>(u[p], 0, 1, tw);
    }
}

template <int P, int T, typename C>
SCD_HD void mixfft_B_store(C *s, int t, const C (&u)[MixFft<P, T>::PER][T]) {
    constexpr int PER = MixFft<P, T>::PER, N1 = P / T;
#pragma unroll
    for (int p = 0; p < PER; ++p)
#pragma unroll
        for (int b = 0; b < T; ++b) s[pidx(t * PER + p + N1 * b)] = u[p][b];
}

#ifdef __CUDACC__
// the whole transform of one line held in s by its T threads (t = 0..T-1,
// one warp)
template <int P, int T, bool INV, typename C>
__device__ __forceinline__ void fft_line_mixed(C *s, const C *tw, int t) {
    C v[P / T];
    mixfft_A<P, T, INV>(s, tw, t, v);
    __syncwarp();
    mixfft_A_store<P, T>(s, t, v);
    __syncwarp();
    C u[MixFft<P, T>::PER][T];
    mixfft_B<P, T, INV>(s, tw, t, u);
    __syncwarp();
    mixfft_B_store<P, T>(s, t, u);
    __syncwarp();
}
#endif
