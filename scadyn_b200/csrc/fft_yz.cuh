// The y and z passes of the pruned FFT convolution fused into one kernel,
// one CTA per (x column, grid): the (y, z) plane of an x-transformed grid is
// held in shared memory and transformed along y (length PY, zero padded from
// Ny), then along z (length PZ, zero padded from Nz) in chunks of KC lines,
// multiplied by the Green spectrum, transformed back along z and y, and its
// Ny x Nz corner is written back in place.  Replaces the three passes y
// forward, z (forward, x Fg, inverse), y inverse (FFT3d_2 / IFFT3d_2,
// src/possu.f90:140-289, with the product of src/gmres_module.f90:104...):
// the plane crosses HBM once each way instead of six times, and the z lines
// are never strided in global memory.
//
// Global layout of an x-transformed grid (rg = 4 r + g): Wt[rg][x][z][y],
// x < Px, z < Nz, y < Ny (y fastest), written by the x forward pass and read
// by the x inverse pass.  The Green spectrum is the octant of Fg (even in
// every axis) pre-scaled by 1/(Px Py Pz), transposed for this pass to
// Fyz[(fx Hy + fy) Hz + fz], H = P/2 + 1.
//
// Shared memory (elements of C): twiddles twy[PY], twz[PZ]; the plane
// A[NzR][LSY] (row z holds the y line, padded index pidx); the chunk
// B[KC][LSZ] (row l holds the z line of ky = ky0 + l).  NzR = Nz rounded up
// to a multiple of 8, so that a warp's lines are either all real or all
// padding rows (the line transforms are warp-synchronous).
//
// Line transforms are the register transforms of fft_reg.cuh (P = 64, 128,
// 8 threads per line) and fft_mixed.cuh (P = 80, 96 with 4 threads, 192 with
// 8).  The phases below are host-callable so that a host program can run the
// whole pass thread by thread and check it (tests/fft_yz_check.cu).
#pragma once
#include "common.cuh"
#include "fft_mixed.cuh"
#include "fft_reg.cuh"

constexpr int YZ_THREADS = 256;

// Line stride in shared memory: at least the padded line (pidx range), and
// such that the lines a half-warp transforms together fall in disjoint
// 8-byte bank pairs: with 8 threads per line a half-warp holds 2 lines, each
// touching 8 consecutive pairs per access, so the stride is 8 mod 16 pairs;
// with 4 threads it holds 4 lines of 4 pairs, so 4 or 12 mod 16.
constexpr int yz_line_stride(int P, int tpl) {
    int L = P + (P >> 4) + 1;
    while (tpl == 8 ? (L % 16 != 8) : (L % 16 != 4 && L % 16 != 12)) ++L;
    return L;
}

template <int P> struct YzLine {
    static constexpr bool REG = P == 64 || P == 128;
    static constexpr bool MIX = P == 80 || P == 96 || P == 192;
    static constexpr bool OK = REG || MIX;
    static constexpr int TPL = REG ? 8 : (P % 64 == 0 ? 8 : 4);   // threads per line
    static constexpr int LS = yz_line_stride(P, TPL);               // line stride
    static constexpr int LINES = YZ_THREADS / TPL;                  // lines per round
};

// Chunk copies between the plane's columns and the z lines run over 4 x 4
// tiles (4 consecutive lines ky by 4 consecutive z per half-warp): the plane
// side reads 4 runs of 4 contiguous elements, the chunk side writes 4 runs of
// 4, instead of 16 elements one line stride apart on one side.
SCD_HD void yz_tile4(int e, int nl, int &l, int &z) {
    const int w = e & 15, blk = e >> 4, nbl = nl >> 2;
    l = ((blk % nbl) << 2) + (w & 3);
    z = ((blk / nbl) << 2) + (w >> 2);
}

struct YzDims {
    int Nx, Ny, Nz, NzR;   // grid nodes, Nz rounded up to a multiple of 8
    int Px;                // x FFT length
    int Hx, Hy, Hz;        // octant sizes P/2 + 1
};

SCD_HD int yz_fold(int u, int P) { return u <= P - u ? u : P - u; }
SCD_HD int yz_round8(int n) { return (n + 7) & ~7; }

// shared-memory elements of one CTA
template <int PY, int PZ>
SCD_HD long long yz_smem_elems(int NzR) {
    return (long long)PY + PZ + (long long)NzR * YzLine<PY>::LS + (long long)YzLine<PZ>::LINES * YzLine<PZ>::LS;
}

// plane load: A[z][y] = Wp[z Ny + y] for z < Nz, y < Ny, zero elsewhere
// (the y padding and the rows Nz..NzR-1)
template <int PY, typename C>
SCD_HD void yz_load(int tid, C *A, const C *Wp, const YzDims &D) {
    constexpr int LSY = YzLine<PY>::LS;
    for (int e = tid; e < D.NzR * PY; e += YZ_THREADS) {
        const int z = e / PY, y = e - z * PY;
        A[z * LSY + pidx(y)] = (z < D.Nz && y < D.Ny) ? Wp[(long long)z * D.Ny + y] : czero<C>();
    }
}

// plane store: Wp[z Ny + y] = A[z][y] for z < Nz, y < Ny
template <int PY, typename C>
SCD_HD void yz_store(int tid, const C *A, C *Wp, const YzDims &D) {
    constexpr int LSY = YzLine<PY>::LS;
    const int n = D.Nz * D.Ny;
    for (int e = tid; e < n; e += YZ_THREADS) {
        const int z = e / D.Ny, y = e - z * D.Ny;
        Wp[e] = A[z * LSY + pidx(y)];
    }
}

// chunk load: B[l][z] = A[z][ky0 + l] for z < Nz and ky0 + l < PY, zero
// elsewhere (the z padding and lines past PY)
template <int PY, int PZ, typename C>
SCD_HD void yz_zload(int tid, const C *A, C *B, int ky0, const YzDims &D) {
    constexpr int LSY = YzLine<PY>::LS, LSZ = YzLine<PZ>::LS, KC = YzLine<PZ>::LINES;
    static_assert(KC % 4 == 0 && PZ % 4 == 0, "4 x 4 tiles");
    for (int e = tid; e < KC * PZ; e += YZ_THREADS) {
        int l, z;
        yz_tile4(e, KC, l, z);
        const int ky = ky0 + l;
        B[l * LSZ + pidx(z)] = (z < D.Nz && ky < PY) ? A[z * LSY + pidx(ky)] : czero<C>();
    }
}

// chunk store: A[z][ky0 + l] = B[l][z] for z < Nz and ky0 + l < PY
template <int PY, int PZ, typename C>
SCD_HD void yz_zstore(int tid, C *A, const C *B, int ky0, const YzDims &D) {
    constexpr int LSY = YzLine<PY>::LS, LSZ = YzLine<PZ>::LS, KC = YzLine<PZ>::LINES;
    const int n = KC * ((D.Nz + 3) & ~3);
    for (int e = tid; e < n; e += YZ_THREADS) {
        int l, z;
        yz_tile4(e, KC, l, z);
        const int ky = ky0 + l;
        if (ky < PY && z < D.Nz) A[z * LSY + pidx(ky)] = B[l * LSZ + pidx(z)];
    }
}

// the Green product of a chunk: B[l][kz] *= Fyz(fx, fold(ky), fold(kz)),
// each line by its own TZ threads (thread t of line l = tid / TZ takes kz = t,
// t + TZ, ...), so that the line's transforms before and after it need only
// a warp synchronisation (a warp holds whole lines)
template <int PY, int PZ, typename C>
SCD_HD void yz_green(int tid, C *B, const C *Fyz, int fx, int ky0, const YzDims &D) {
    constexpr int LSZ = YzLine<PZ>::LS, TZ = YzLine<PZ>::TPL;
    const int l = tid / TZ, t = tid - l * TZ, ky = ky0 + l;
    if (ky >= PY) return;
    const C *Fr = Fyz + ((long long)fx * D.Hy + yz_fold(ky, PY)) * D.Hz;
    for (int kz = t; kz < PZ; kz += TZ) B[l * LSZ + pidx(kz)] = cmul(Fr[yz_fold(kz, PZ)], B[l * LSZ + pidx(kz)]);
}

// one line transform run on the host: every thread of the line, phase by
// phase, as the warp does
template <int P, bool INV, typename C>
void yz_line_host(C *s, const C *tw) {
    if constexpr (YzLine<P>::REG) {
        constexpr int PER = RegFft<P>::PER;
        C v[8][P / 8];
        for (int t = 0; t < 8; ++t) regfft_A<P, INV>(s, tw, t, v[t]);
        for (int t = 0; t < 8; ++t) regfft_A_store<P>(s, t, v[t]);
        C u[8][PER][8];
        for (int t = 0; t < 8; ++t) regfft_B<P, INV>(s, tw, t, u[t]);
        for (int t = 0; t < 8; ++t) regfft_B_store<P>(s, t, u[t]);
    } else {
        constexpr int T = YzLine<P>::TPL, PER = MixFft<P, T>::PER;
        C v[T][P / T];
        for (int t = 0; t < T; ++t) mixfft_A<P, T, INV>(s, tw, t, v[t]);
        for (int t = 0; t < T; ++t) mixfft_A_store<P, T>(s, t, v[t]);
        C u[T][PER][T];
        for (int t = 0; t < T; ++t) mixfft_B<P, T, INV>(s, tw, t, u[t]);
        for (int t = 0; t < T; ++t) mixfft_B_store<P, T>(s, t, u[t]);
    }
}

// the whole fused pass of one plane on the host (x column x, grid rg): the
// same phases, in the kernel's order, with the CTA's threads run in turn
template <int PY, int PZ, typename C>
void yz_plane_host(C *Wp, const C *Fyz, const C *twy, const C *twz, int x, const YzDims &D, C *smem) {
    constexpr int LSY = YzLine<PY>::LS, LSZ = YzLine<PZ>::LS, KC = YzLine<PZ>::LINES;
    C *A = smem + PY + PZ, *B = A + (long long)D.NzR * LSY;
    for (int t = 0; t < YZ_THREADS; ++t) yz_load<PY>(t, A, Wp, D);
    for (int l = 0; l < D.NzR; ++l) yz_line_host<PY, false>(A + l * LSY, twy);
    const int fx = yz_fold(x, D.Px);
    for (int ky0 = 0; ky0 < PY; ky0 += KC) {
        for (int t = 0; t < YZ_THREADS; ++t) yz_zload<PY, PZ>(t, A, B, ky0, D);
        for (int l = 0; l < KC; ++l) yz_line_host<PZ, false>(B + l * LSZ, twz);
        for (int t = 0; t < YZ_THREADS; ++t) yz_green<PY, PZ>(t, B, Fyz, fx, ky0, D);
        for (int l = 0; l < KC; ++l) yz_line_host<PZ, true>(B + l * LSZ, twz);
        for (int t = 0; t < YZ_THREADS; ++t) yz_zstore<PY, PZ>(t, A, B, ky0, D);
    }
    for (int l = 0; l < D.NzR; ++l) yz_line_host<PY, true>(A + l * LSY, twy);
    for (int t = 0; t < YZ_THREADS; ++t) yz_store<PY>(t, A, Wp, D);
}

#ifdef __CUDACC__
template <int P, bool INV, typename C>
__device__ __forceinline__ void yz_line_dev(C *s, const C *tw, int t) {
    if constexpr (YzLine<P>::REG) fft_line_reg<P, INV, C>(s, tw, t);
    else fft_line_mixed<P, YzLine<P>::TPL, INV, C>(s, tw, t);
}

// the NzR y lines of the plane, LINES per round; a warp's lines are all
// below NzR or all above it (NzR and the lines per warp are multiples of
// 8 and 4), so the warp-synchronous transform is never split
template <int PY, bool INV, typename C>
__device__ __forceinline__ void yz_ylines_dev(C *A, const C *tw, int NzR) {
    constexpr int TPL = YzLine<PY>::TPL, LS = YzLine<PY>::LS, LINES = YzLine<PY>::LINES;
    const int tid = threadIdx.x;
    for (int l0 = 0; l0 < NzR; l0 += LINES) {
        const int l = l0 + tid / TPL;
        if (l < NzR) yz_line_dev<PY, INV, C>(A + l * LS, tw, tid % TPL);
    }
}

// one CTA per (x, rg): grid (Px, 4 nrhs); dynamic shared memory
// yz_smem_elems<PY, PZ>(NzR) elements of C
template <int PY, int PZ, typename C>
__global__ void __launch_bounds__(YZ_THREADS)
k_fft_yz(C *__restrict__ Wt, const C *__restrict__ Fyz, const C *__restrict__ twy_g, const C *__restrict__ twz_g,
         YzDims D, const int *done) {
    const int x = blockIdx.x, rg = blockIdx.y;
    if (done && done[rg >> 2]) return;
    constexpr int LSY = YzLine<PY>::LS, LSZ = YzLine<PZ>::LS, KC = YzLine<PZ>::LINES, TZ = YzLine<PZ>::TPL;
    extern __shared__ __align__(16) unsigned char yz_raw[];
    C *twy = reinterpret_cast<C *>(yz_raw), *twz = twy + PY, *A = twz + PZ, *B = A + D.NzR * LSY;
    const int tid = threadIdx.x;
    for (int i = tid; i < PY; i += YZ_THREADS) twy[i] = twy_g[i];
    for (int i = tid; i < PZ; i += YZ_THREADS) twz[i] = twz_g[i];
    C *Wp = Wt + ((long long)rg * D.Px + x) * D.Nz * D.Ny;
    yz_load<PY>(tid, A, Wp, D);
    __syncthreads();
    yz_ylines_dev<PY, false>(A, twy, D.NzR);
    __syncthreads();
    const int fx = yz_fold(x, D.Px);
    for (int ky0 = 0; ky0 < PY; ky0 += KC) {
        yz_zload<PY, PZ>(tid, A, B, ky0, D);
        __syncthreads();
        yz_line_dev<PZ, false, C>(B + (tid / TZ) * LSZ, twz, tid % TZ);
        __syncwarp();   // a warp holds whole lines (YZ_THREADS / TZ lines, 32 / TZ per warp)
        yz_green<PY, PZ>(tid, B, Fyz, fx, ky0, D);
        __syncwarp();
        yz_line_dev<PZ, true, C>(B + (tid / TZ) * LSZ, twz, tid % TZ);
        __syncthreads();
        yz_zstore<PY, PZ>(tid, A, B, ky0, D);
        __syncthreads();
    }
    yz_ylines_dev<PY, true>(A, twy, D.NzR);
    __syncthreads();
    yz_store<PY>(tid, A, Wp, D);
}

// Fyz[(fx Hy + fy) Hz + fz] = Fo[(fz Hy + fy) Hx + fx]
template <typename C>
__global__ void k_green_yz(const C *__restrict__ Fo, C *__restrict__ Fyz, int Hx, int Hy, int Hz) {
    const long long n = (long long)Hx * Hy * Hz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int fz = (int)(i % Hz);
        const long long r = i / Hz;
        const int fy = (int)(r % Hy), fx = (int)(r / Hy);
        Fyz[i] = Fo[((long long)fz * Hy + fy) * Hx + fx];
    }
}
#endif
