// The pFFT matvec on the device: anterpolation onto the grid, the pruned
// FFT convolution with the Green's function, interpolation back to the tets,
// and the near-zone correction.  Restates compute_Ax2
// (src/gmres_module.f90:57-176) for the constant basis with the three
// cross-component convolutions (:122-144) merged into one by linearity:
//   Y_dd  = S  . G*(S^T x_d)                 d = x, y, z
//   Y2_e  = S_e . G*(Sx^T x_x + Sy^T x_y + Sz^T x_z)
//   Ax    = A_near x + (Y2 - k^2 Y)
// All vectors are slot ordered (tets sorted by cube); see ctx.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include <type_traits>

#include "ctx.h"
#include "fft_mixed.cuh"
#include "fft_reg.cuh"
#include "fft_yz.cuh"
#include "linear_basis.h"

namespace {

constexpr int WARPS_PER_CTA = 4;
// anterpolation of eight or more right-hand sides with one CTA per cube
// (k_scatter_cta) instead of one warp
#ifndef SCD_SG_CTA
#define SCD_SG_CTA 1
#endif
// resident CTAs per SM the complex64 interpolation kernel is compiled for
// (its register cap): at C2 with 32 right-hand sides 0.75 ms with 3 (160
// registers), 0.90 with 1 (174), 1.07 with 4 or 5 (spills)
#ifndef SCD_GATHER_MINB
#define SCD_GATHER_MINB 3
#endif

// slot order <-> the reference's unknown order (nb basis functions per tet:
// 1, or 4 for the linear basis, see linear_basis.h)
__global__ void k_permute_in(const cd *__restrict__ xo, cd *__restrict__ xs, const int *__restrict__ perm,
                             int T, long long ld, int nb) {
    const int r = blockIdx.y;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3LL * T; i += (long long)gridDim.x * blockDim.x) {
        long long s = i / 3, d = i - 3 * s;
        xs[r * ld + i] = xo[r * ld + basis_unknown(nb, perm[s], (int)d)];
    }
}

__global__ void k_permute_out(const cd *__restrict__ xs, cd *__restrict__ xo, const int *__restrict__ perm,
                              int T, long long ld, int nb) {
    const int r = blockIdx.y;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3LL * T; i += (long long)gridDim.x * blockDim.x) {
        long long s = i / 3, d = i - 3 * s;
        xo[r * ld + basis_unknown(nb, perm[s], (int)d)] = xs[r * ld + i];
    }
}

// ---------------------------------------------------------------- scatter
// Anterpolation (sparse_T_matmul, src/sparse.f90:13-43), one warp per
// (cube, span of rspan right-hand sides): lane j < 27 accumulates the four
// box-node sums of node j over the cube's tets, SC_RG right-hand sides at a
// time (projector values are read once per group of SC_RG and stay in L1 for
// the next group of the span).  The spans are the grid's y index; rspan is a
// multiple of SC_RG.  Projectors are stored P[(g*27 + j)*T + slot].
// bpart[((r*ncubes + c)*4 + g)*27 + j].
template <typename C, int SC_RG>
__global__ void __launch_bounds__(32 * WARPS_PER_CTA)
k_scatter(const C *__restrict__ x, long long ld, const C *__restrict__ P, int T,
          const int *__restrict__ cube_off, int ncubes, C *__restrict__ bpart, const int *skip, int nrhs, int rspan) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * WARPS_PER_CTA + warp;
    if (c >= ncubes || lane >= 27) return;
    const int s0 = cube_off[c], s1 = cube_off[c + 1];
    const C *P0 = P + (size_t)lane * T, *PX = P + (size_t)(27 + lane) * T;
    const C *PY = P + (size_t)(54 + lane) * T, *PZ = P + (size_t)(81 + lane) * T;
    const int rend = min(nrhs, (int)(blockIdx.y + 1) * rspan);
    for (int r0 = blockIdx.y * rspan; r0 < rend; r0 += SC_RG) {
        C acc[SC_RG][4];
#pragma unroll
        for (int q = 0; q < SC_RG; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = czero<C>();
#pragma unroll 4
        for (int s = s0; s < s1; ++s) {
            const C p0 = P0[s], px = PX[s], py = PY[s], pz = PZ[s];
#pragma unroll
            for (int q = 0; q < SC_RG; ++q) {
                const int r = r0 + q;
                if (r < nrhs) {
                    const C *xr = x + r * ld + 3LL * s;
                    const C x0 = xr[0], x1 = xr[1], x2 = xr[2];
                    cfma(acc[q][0], p0, x0);
                    cfma(acc[q][1], p0, x1);
                    cfma(acc[q][2], p0, x2);
                    cfma(acc[q][3], px, x0);
                    cfma(acc[q][3], py, x1);
                    cfma(acc[q][3], pz, x2);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < SC_RG; ++q) {
            const int r = r0 + q;
            if (r < nrhs && !(skip && skip[r])) {
                C *o = bpart + ((long long)r * ncubes + c) * 4 * 27 + lane;
                o[0] = acc[q][0];
                o[27] = acc[q][1];
                o[54] = acc[q][2];
                o[81] = acc[q][3];
            }
        }
    }
}

// The same anterpolation for many right-hand sides, one CTA per (cube, span
// of right-hand sides): the cube's projector rows are staged in shared
// memory by the whole CTA (coalesced over the cube's tets, NTC at a time),
// and the four warps take SR right-hand sides each per round, lane j < 27
// summing node j over the tets in ascending order from shared memory -- the
// order of k_scatter, so a column gives the same bits through either.  The
// row stride NTC + 1 keeps the lanes' reads of one tet in distinct banks.
constexpr int SCB = 128;
template <typename C, int NTC, int SR>
__global__ void __launch_bounds__(SCB)
k_scatter_cta(const C *__restrict__ x, long long ld, const C *__restrict__ P, int T, const int *__restrict__ cube_off,
              int ncubes, C *__restrict__ bpart, const int *skip, int nrhs, int rspan) {
    __shared__ C Ps[108][NTC + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x;
    const int s0 = cube_off[c], nt = cube_off[c + 1] - s0;
    const int rlo = blockIdx.y * rspan, rhi = min(nrhs, rlo + rspan);
    const int nround = (rhi - rlo + 4 * SR - 1) / (4 * SR);
    const bool one = nt <= NTC;
    auto stage = [&](int t0) {
        const int m = min(NTC, nt - t0);
        for (int e = threadIdx.x; e < 108 * m; e += SCB) {
            const int row = e / m, t = e - row * m;
            Ps[row][t] = P[(size_t)row * T + s0 + t0 + t];
        }
    };
    if (one && nt > 0) stage(0);
    __syncthreads();
    for (int rd = 0; rd < nround; ++rd) {
        const int rb = rlo + (rd * 4 + warp) * SR;
        C acc[SR][4];
#pragma unroll
        for (int q = 0; q < SR; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = czero<C>();
        for (int t0 = 0; t0 < nt; t0 += NTC) {
            if (!one) {
                __syncthreads();
                stage(t0);
                __syncthreads();
            }
            const int m = min(NTC, nt - t0);
            if (lane < 27) {
                for (int t = 0; t < m; ++t) {
                    const C p0 = Ps[lane][t], px = Ps[27 + lane][t], py = Ps[54 + lane][t], pz = Ps[81 + lane][t];
                    const long long s = s0 + t0 + t;
#pragma unroll
                    for (int q = 0; q < SR; ++q) {
                        const int r = rb + q;
                        if (r < rhi) {
                            const C *xr = x + r * ld + 3LL * s;
                            const C x0 = xr[0], x1 = xr[1], x2 = xr[2];
                            cfma(acc[q][0], p0, x0);
                            cfma(acc[q][1], p0, x1);
                            cfma(acc[q][2], p0, x2);
                            cfma(acc[q][3], px, x0);
                            cfma(acc[q][3], py, x1);
                            cfma(acc[q][3], pz, x2);
                        }
                    }
                }
            }
        }
        if (lane < 27) {
#pragma unroll
            for (int q = 0; q < SR; ++q) {
                const int r = rb + q;
                if (r < rhi && !(skip && skip[r])) {
                    C *o = bpart + ((long long)r * ncubes + c) * 4 * 27 + lane;
                    o[0] = acc[q][0];
                    o[27] = acc[q][1];
                    o[54] = acc[q][2];
                    o[81] = acc[q][3];
                }
            }
        }
    }
}

// -------------------------------------------------------------------- FFT
// Radix-4 Stockham (with a final radix-2 stage for odd log2 P) on lines held
// in shared memory, FFTW sign convention (forward exp(-i)), unnormalised.
// TPL = P/4 threads cooperate on a line; all lines of a CTA advance together.
template <int P> struct Log2 { static constexpr int v = 1 + Log2<P / 2>::v; };
template <> struct Log2<1> { static constexpr int v = 0; };

template <bool INV, typename C>
__device__ __forceinline__ void radix4(C &v0, C &v1, C &v2, C &v3) {
    C a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), a3 = csub(v1, v3);
    // forward: X1 = a1 - i a3 ; X3 = a1 + i a3
    C ia3;                                                 // (+i or -i) * a3
    ia3.x = INV ? -a3.y : a3.y;
    ia3.y = INV ? a3.x : -a3.x;
    v0 = cadd(a0, a2);
    v2 = csub(a0, a2);
    v1 = cadd(a1, ia3);
    v3 = csub(a1, ia3);
}

// in-line padding pidx(i) = i + (i >> 4) (fft_reg.cuh): one spare slot per
// 16 complex values spreads the strided Stockham writes over the banks

template <bool INV, typename C>
__device__ __forceinline__ C twid(const C *tw, int i) {
    C w = tw[i];
    return INV ? cconj(w) : w;
}

template <int P, bool INV, typename C>
__device__ __forceinline__ void fft_line(C *s, const C *tw, int t) {
    constexpr int L = Log2<P>::v;
    constexpr int NB = P / 4;
    int Ns = 1;
#pragma unroll
    for (int st = 0; st < L / 2; ++st) {
        const int j = t;
        C v0 = s[pidx(j)], v1 = s[pidx(j + NB)], v2 = s[pidx(j + 2 * NB)], v3 = s[pidx(j + 3 * NB)];
        const int kk = j & (Ns - 1);
        if (Ns > 1) {
            const int step = P / (Ns * 4);
            v1 = cmul(v1, twid<INV, C>(tw, kk * step));
            v2 = cmul(v2, twid<INV, C>(tw, 2 * kk * step));
            v3 = cmul(v3, twid<INV, C>(tw, 3 * kk * step));
        }
        radix4<INV, C>(v0, v1, v2, v3);
        __syncthreads();
        const int idx = (j / Ns) * Ns * 4 + kk;
        s[pidx(idx)] = v0;
        s[pidx(idx + Ns)] = v1;
        s[pidx(idx + 2 * Ns)] = v2;
        s[pidx(idx + 3 * Ns)] = v3;
        __syncthreads();
        Ns *= 4;
    }
    if (L & 1) {   // radix-2 stage, Ns = P/2: butterflies j = t, t + NB
        C a[2], b[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = t + q * NB;
            a[q] = s[pidx(j)];
            b[q] = cmul(s[pidx(j + P / 2)], twid<INV, C>(tw, j));
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = t + q * NB;
            s[pidx(j)] = cadd(a[q], b[q]);
            s[pidx(j + P / 2)] = csub(a[q], b[q]);
        }
        __syncthreads();
    }
}

// Line FFT of the passes: register-resident 8-thread transform for P = 64
// and 128 (fft_reg.cuh), register-resident mixed-radix transform with 4 or 8
// threads for the 5-smooth lengths below (fft_mixed.cuh), shared-memory
// radix-4 Stockham for other powers of two.
// (N1 = P / threads <= 24 keeps the FP64 transforms within the register file)
template <int P> constexpr bool fft_mixed_len() { return P == 80 || P == 96 || P == 192; }
// lines per CTA halved until the line buffers fit 44 KB of static shared memory
constexpr int fft_fit_lpb(int lpb, int ls, int es) { return (lpb > 1 && lpb * ls * es > 44 * 1024) ? fft_fit_lpb(lpb / 2, ls, es) : lpb; }
template <int P, typename Cx> struct FftCfg {
    static constexpr bool REG = P == 64 || P == 128;
    static constexpr bool MIX = !REG && fft_mixed_len<P>();
    static constexpr int LS = P + (P >> 4) + 1;              // padded line stride (bank spread)
    static constexpr int TPL = REG ? 8 : MIX ? (P % 64 == 0 ? 8 : 4) : P / 4;   // threads per line
    static constexpr int LPB = REG ? (sizeof(Cx) == 16 ? 16 : 32)
                               : MIX ? fft_fit_lpb(256 / TPL / (sizeof(Cx) == 16 ? 2 : 1), LS, (int)sizeof(Cx))
                                     : ((256 / TPL) > 0 ? 256 / TPL : 1);   // lines per CTA
    static constexpr int THREADS = TPL * LPB;
};

template <int P, bool INV, typename Cx>
__device__ __forceinline__ void fft_line_any(Cx *s, const Cx *tw, int t) {
    if constexpr (FftCfg<P, Cx>::REG) {
        fft_line_reg<P, INV, Cx>(s, tw, t);
        __syncthreads();   // the passes' next loops read every line of the CTA
    } else if constexpr (FftCfg<P, Cx>::MIX) {
        fft_line_mixed<P, FftCfg<P, Cx>::TPL, INV, Cx>(s, tw, t);
        __syncthreads();
    } else {
        fft_line<P, INV, Cx>(s, tw, t);
    }
}

struct GridDims {
    int Nx, Ny, Nz, Px, Py, Pz, Hx, Hy, Hz, ncx, ncy, ncz, ncubes;
};

__device__ __forceinline__ int fold(int u, int P) { return u <= P - u ? u : P - u; }

// node value of grid g at node (x,y,z) from the box partial sums: every box
// whose 3x3x3 node block contains the node contributes its local sum
template <typename C>
__device__ __forceinline__ C node_value(const C *__restrict__ bp, const GridDims &G, int g, int x, int y, int z) {
    int bxs[2], axs[2], nbx = 0, bys[2], ays[2], nby = 0, bzs[2], azs[2], nbz = 0;
    int b = x >> 1;
    if (b < G.ncx) { bxs[nbx] = b; axs[nbx++] = x - 2 * b; }
    if (!(x & 1) && x >= 2 && b - 1 < G.ncx) { bxs[nbx] = b - 1; axs[nbx++] = 2; }
    b = y >> 1;
    if (b < G.ncy) { bys[nby] = b; ays[nby++] = y - 2 * b; }
    if (!(y & 1) && y >= 2 && b - 1 < G.ncy) { bys[nby] = b - 1; ays[nby++] = 2; }
    b = z >> 1;
    if (b < G.ncz) { bzs[nbz] = b; azs[nbz++] = z - 2 * b; }
    if (!(z & 1) && z >= 2 && b - 1 < G.ncz) { bzs[nbz] = b - 1; azs[nbz++] = 2; }
    C v = czero<C>();
    for (int iz = 0; iz < nbz; ++iz)
        for (int iy = 0; iy < nby; ++iy)
            for (int ix = 0; ix < nbx; ++ix) {
                const int box = bxs[ix] + G.ncx * (bys[iy] + G.ncy * bzs[iz]);
                const int j = axs[ix] + 3 * ays[iy] + 9 * azs[iz];
                v = cadd(v, bp[((long long)box * 4 + g) * 27 + j]);
            }
    return v;
}

// X forward: lines (y < Ny, z < Nz) of grid (g, r); node assembly on load,
// zero padding x >= Nx.  W[(rg)][(z*Py + y)*Px + x] for the three-pass
// y/z chain, or (TL) the fused y-z pass's layout Wt[rg][x][z][y] (fft_yz.cuh):
// a CTA's lines are consecutive (z, y), so for every x its outputs are one
// contiguous run.
template <int P, typename Cx, bool TL>
__global__ void __launch_bounds__(FftCfg<P, Cx>::THREADS)
k_fft_x_fwd(const Cx *__restrict__ bpart, Cx *__restrict__ W, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P, Cx>;
    __shared__ Cx sh[Cf::LPB * Cf::LS];
    __shared__ Cx tw[P];
    const int rg = blockIdx.y;                 // r*4 + g
    const int g = rg & 3, r = rg >> 2;
    const Cx *bp = bpart + (long long)r * G.ncubes * 4 * 27;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int nlines = G.Ny * G.Nz;
    const int line0 = blockIdx.x * Cf::LPB;
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int l = e / P, x = e - l * P, line = line0 + l;
        Cx v = czero<Cx>();
        if (line < nlines && x < G.Nx) {
            const int y = line % G.Ny, z = line / G.Ny;
            v = node_value<Cx>(bp, G, g, x, y, z);
        }
        sh[l * Cf::LS + pidx(x)] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / Cf::TPL, t = threadIdx.x - l * Cf::TPL;
    fft_line_any<P, false, Cx>(sh + l * Cf::LS, tw, t);
    if constexpr (TL) {
        Cx *Wr = W + (long long)rg * P * nlines;
        for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
            const int x = e / Cf::LPB, ll = e - x * Cf::LPB, line = line0 + ll;
            if (line < nlines) Wr[(long long)x * nlines + line] = sh[ll * Cf::LS + pidx(x)];
        }
    } else {
        Cx *Wr = W + (long long)rg * G.Px * G.Py * G.Nz;
        for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
            const int ll = e / P, x = e - ll * P, line = line0 + ll;
            if (line < nlines) {
                const int y = line % G.Ny, z = line / G.Ny;
                Wr[((long long)z * G.Py + y) * G.Px + x] = sh[ll * Cf::LS + pidx(x)];
            }
        }
    }
}

// Y pass: lines (x < Px, z < Nz); forward reads y < Ny and writes y < Py,
// inverse reads y < Py and writes y < Ny.  A CTA takes LPB consecutive x.
template <int P, bool INV, typename Cx>
__global__ void __launch_bounds__(FftCfg<P, Cx>::THREADS)
k_fft_y(Cx *__restrict__ W, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P, Cx>;
    __shared__ Cx sh[Cf::LPB * Cf::LS];
    __shared__ Cx tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int xblocks = (G.Px + Cf::LPB - 1) / Cf::LPB;
    const int z = blockIdx.x / xblocks, x0 = (blockIdx.x - z * xblocks) * Cf::LPB;
    Cx *Wr = W + (long long)rg * G.Px * G.Py * G.Nz + (long long)z * G.Py * G.Px;
    const int nin = INV ? G.Py : G.Ny, nout = INV ? G.Ny : G.Py;
    // sh layout [line][y]
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int y = e / Cf::LPB, l = e - y * Cf::LPB, x = x0 + l;
        Cx v = czero<Cx>();
        if (y < nin && x < G.Px) v = Wr[(long long)y * G.Px + x];
        sh[l * Cf::LS + pidx(y)] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / Cf::TPL, t = threadIdx.x - l * Cf::TPL;
    fft_line_any<P, INV, Cx>(sh + l * Cf::LS, tw, t);
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int y = e / Cf::LPB, ll = e - y * Cf::LPB, x = x0 + ll;
        if (y < nout && x < G.Px) Wr[(long long)y * G.Px + x] = sh[ll * Cf::LS + pidx(y)];
    }
}

// Z pass: lines (x < Px, y < Py), forward FFT of z < Nz (zero padded), times
// the Green octant Fo (folded by evenness), inverse FFT, keep z < Nz.
template <int P, typename Cx>
__global__ void __launch_bounds__(FftCfg<P, Cx>::THREADS)
k_fft_z(Cx *__restrict__ W, const Cx *__restrict__ Fo, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P, Cx>;
    __shared__ Cx sh[Cf::LPB * Cf::LS];
    __shared__ Cx tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int xblocks = (G.Px + Cf::LPB - 1) / Cf::LPB;
    const int y = blockIdx.x / xblocks, x0 = (blockIdx.x - y * xblocks) * Cf::LPB;
    const long long plane = (long long)G.Px * G.Py;
    Cx *Wr = W + (long long)rg * plane * G.Nz + (long long)y * G.Px;
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int z = e / Cf::LPB, l = e - z * Cf::LPB, x = x0 + l;
        Cx v = czero<Cx>();
        if (z < G.Nz && x < G.Px) v = Wr[(long long)z * plane + x];
        sh[l * Cf::LS + pidx(z)] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / Cf::TPL, t = threadIdx.x - l * Cf::TPL;
    fft_line_any<P, false, Cx>(sh + l * Cf::LS, tw, t);
    const int fy = fold(y, G.Py);
    // consecutive threads take consecutive lines (x), so the octant reads of
    // one z plane are contiguous
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int z = e / Cf::LPB, ll = e - z * Cf::LPB, x = x0 + ll;
        if (x < G.Px) {
            const Cx f = __ldg(&Fo[((long long)fold(z, G.Pz) * G.Hy + fy) * G.Hx + fold(x, G.Px)]);
            sh[ll * Cf::LS + pidx(z)] = cmul(f, sh[ll * Cf::LS + pidx(z)]);
        }
    }
    __syncthreads();
    fft_line_any<P, true, Cx>(sh + l * Cf::LS, tw, t);
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int z = e / Cf::LPB, ll = e - z * Cf::LPB, x = x0 + ll;
        if (z < G.Nz && x < G.Px) Wr[(long long)z * plane + x] = sh[ll * Cf::LS + pidx(z)];
    }
}

// X inverse: lines (y < Ny, z < Nz), keep x < Nx, write the result grid
// R[(rg)][(z*Ny + y)*Nx + x]; the input in the three-pass layout or (TL) the
// fused y-z pass's Wt[rg][x][z][y]
template <int P, typename Cx, bool TL>
__global__ void __launch_bounds__(FftCfg<P, Cx>::THREADS)
k_fft_x_inv(const Cx *__restrict__ W, Cx *__restrict__ R, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P, Cx>;
    __shared__ Cx sh[Cf::LPB * Cf::LS];
    __shared__ Cx tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int nlines = G.Ny * G.Nz;
    const int line0 = blockIdx.x * Cf::LPB;
    if constexpr (TL) {
        const Cx *Wr = W + (long long)rg * P * nlines;
        for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
            const int x = e / Cf::LPB, l = e - x * Cf::LPB, line = line0 + l;
            sh[l * Cf::LS + pidx(x)] = line < nlines ? Wr[(long long)x * nlines + line] : czero<Cx>();
        }
    } else {
        const Cx *Wr = W + (long long)rg * G.Px * G.Py * G.Nz;
        for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
            const int l = e / P, x = e - l * P, line = line0 + l;
            Cx v = czero<Cx>();
            if (line < nlines) {
                const int y = line % G.Ny, z = line / G.Ny;
                v = Wr[((long long)z * G.Py + y) * G.Px + x];
            }
            sh[l * Cf::LS + pidx(x)] = v;
        }
    }
    __syncthreads();
    const int l = threadIdx.x / Cf::TPL, t = threadIdx.x - l * Cf::TPL;
    fft_line_any<P, true, Cx>(sh + l * Cf::LS, tw, t);
    Cx *Rr = R + (long long)rg * G.Nx * G.Ny * G.Nz;
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int ll = e / P, x = e - ll * P, line = line0 + ll;
        if (line < nlines && x < G.Nx) {
            const int y = line % G.Ny, z = line / G.Ny;
            Rr[((long long)z * G.Ny + y) * G.Nx + x] = sh[ll * Cf::LS + pidx(x)];
        }
    }
}

// ------------------------------------------------------------ near zone
// Row sums y(g1) += M x(g2) and, for off-diagonal tiles, column sums
// y(g2) += M^T x(g1) (transpose, not conjugate: the operator is complex
// symmetric, src/sparse_mat.f90:113-116).  M(3i+a, 3j+b) is entry (a,b) of
// block (i,j), at tile_at(n1, i, j, a + 3b) (see NearTile).
//
// One CTA per group g: it walks the tiles (g, g2), g2 >= g, in tile order,
// keeping the group's row sums in registers across them, so every group has
// a single row slot; each off-diagonal tile's column sums go to that tile's
// partial slot of g2.  k_gather adds the slots in a fixed order.
//
// Tiles stream through a shared-memory ring filled by a producer thread: a
// tile's blocks and its x segment arrive by bulk copies (TMA engine,
// completion counted in bytes on the slot's "full" mbarrier) at the ring's
// head, so as many tiles are in flight as their sizes allow (up to NZ_SLOTS).
// The x segments come from xT, the right-hand sides interleaved per unknown
// (k_xpose), so a group's x is one contiguous run x[3j+b][r].  Consumer
// warps release a tile on its slot's "empty" barrier; there is no CTA-wide
// barrier in the tile loop, so row and column warps run independently.  Warps [0, HT) hold row items (quad q, block row
// i): a 3 x U register tile of row sums for right-hand sides Uq..Uq+U-1.
// Warps [HT, 2HT) hold column items (q, block column j).  Lanes run over i
// (resp. j), so with the odd plane stride both sides read the tile without
// bank conflicts, and x is a broadcast.
//
// Every sum runs in one canonical order -- row sums: tiles in order, then
// j = 0..n2-1, then b = 0..2; column sums: i = 0..n1-1, then a = 0..2 --
// for any number of right-hand sides and any U, so a column's result does
// not depend on the batch it is solved in.
constexpr int NZ_QMAX = 4;             // quads of right-hand sides per pass
constexpr int NZ_SLOTS = 8;                 // tiles in flight at most (mbarrier pairs)
constexpr int NZ_META = 272;                // bytes of barriers, ring offsets and the stop flag
constexpr size_t NZ_SMEM_2CTA = 113 * 1024; // dynamic shared memory per CTA that lets two CTAs share an SM
constexpr size_t NZ_SMEM_4CTA = 56 * 1024;  // ... four CTAs
// With one right-hand side a tile's sums are short dependent chains, so the
// kernel is latency-bound per tile: four CTAs per SM (registers and ring
// bounded to fit) keep four tiles in progress.  With register tiles of four
// right-hand sides the compiler is left free (two CTAs fit).
template <int U> constexpr int NZ_MIN_CTAS = U == 1 ? 4 : 1;
constexpr size_t NZ_SMEM_MAX = 227 * 1024;
constexpr int NZ_MAX_THREADS = 2 * 32 * ((SCD_GROUP_MAX * NZ_QMAX + 31) / 32) + 32;

struct NearPass {
    const NearTile *tiles;
    const int *grp_tile, *grp_off;
    const long long *pslot_base;
    const void *data;
    const void *xT;          // [pass][3T][RG]
    long long n;             // 3T
    void *part;
    long long part_len;
    const int *skip;
    int nrhs, nq, half, rg_stride;   // rg_stride: right-hand sides per xT row (nq*U, or 2 for a lone complex64 one)
    uint32_t x1_bytes;       // x(g) buffer (multiple of 16)
    uint32_t ring_bytes;     // tile ring (multiple of 16, at least one tile with its x segment)
    int *err;
};

// x (nrhs columns of stride ld) -> xT[p][k][RG]: the RG right-hand sides of
// pass p interleaved per unknown k, zero beyond nrhs
template <typename C>
__global__ void k_xpose(const C *__restrict__ x, long long ld, long long n, int nrhs, int PS, int RG, C *__restrict__ xT) {
    const long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int p = blockIdx.y;
    if (k >= n) return;
    C *dst = xT + ((long long)p * n + k) * RG;
    for (int r = 0; r < RG; ++r) {
        const int rr = p * PS + r;
        dst[r] = (r < PS && rr < nrhs) ? x[(long long)rr * ld + k] : czero<C>();
    }
}

// U consecutive values of C from shared address addr (16-byte aligned when
// C is complex64 and U is even)
template <typename C, int U>
__device__ __forceinline__ void load_xu(uint32_t addr, C (&xu)[U]) {
    if constexpr (sizeof(C) == 8 && U % 2 == 0) {
#pragma unroll
        for (int u = 0; u < U; u += 2) lds_c2(addr + 8 * u, xu[u], xu[u + 1]);
    } else {
#pragma unroll
        for (int u = 0; u < U; ++u) xu[u] = lds_c(addr + (uint32_t)sizeof(C) * u, C{});
    }
}

// partial sums p = 0..NS-1 -> p0 + p1 (NS = 2): NP partials in the lane, or
// one per lane over L adjacent lanes (lane 0 of each pair gets the total;
// every lane of the warp must call it)
template <typename C> __device__ __forceinline__ C shfl_down_c(C v, int d, int width) {
    v.x = __shfl_down_sync(0xffffffffu, v.x, d, width);
    v.y = __shfl_down_sync(0xffffffffu, v.y, d, width);
    return v;
}
template <typename C, int U, int NP, int L>
__device__ __forceinline__ void combine_split(const C (&p)[NP][3][U], C (&tot)[3][U]) {
#pragma unroll
    for (int q = 0; q < 3; ++q)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if constexpr (NP == 2) {
                tot[q][u] = cadd(p[0][q][u], p[1][q][u]);
            } else if constexpr (L == 2) {
                tot[q][u] = cadd(p[0][q][u], shfl_down_c(p[0][q][u], 1, 2));
            } else {
                tot[q][u] = p[0][q][u];
            }
        }
}

// NS (1 or 2) splits every row and column sum into NS partial sums over the
// j (row) or i (column) residues mod NS, added in order at the end: with one
// right-hand side (U = 1) NS lanes share a row or column, one partial each;
// with U = 4 one lane keeps all NS partials.  Either way the sums are formed
// in the same order, so a column stays bit-identical alone and in a batch.
template <typename ST, typename C, int U, int NS>
__global__ void __launch_bounds__(NZ_MAX_THREADS, NZ_MIN_CTAS<U>) k_near_groups(NearPass a) {
    static_assert(NS == 1 || NS == 2, "split");
    constexpr int L = U == 1 ? NS : 1;     // lanes per row or column
    constexpr int NP = NS / L;             // partial sums per lane
    extern __shared__ __align__(128) unsigned char nz_sh[];
    uint64_t *full = reinterpret_cast<uint64_t *>(nz_sh);
    uint64_t *empty = full + NZ_SLOTS;
    // per slot, written by the producer before the slot's arrive: ring offset,
    // n2 and column partial slot of the tile (consumers read no tile table)
    int *toff = reinterpret_cast<int *>(nz_sh + 16 * NZ_SLOTS);
    int *tn2 = toff + NZ_SLOTS;
    long long *tcol = reinterpret_cast<long long *>(nz_sh + 24 * NZ_SLOTS);
    // raised by the first wait that gives up: the producer issues no more
    // copies, the consumers skip the remaining tiles (still arriving on their
    // barriers), and the kernel returns with a.err set
    volatile int *stop = reinterpret_cast<volatile int *>(nz_sh + 32 * NZ_SLOTS);
    C *const X1 = reinterpret_cast<C *>(nz_sh + NZ_META);                 // x(g)
    unsigned char *const ring = nz_sh + NZ_META + a.x1_bytes;
    const ST *data = static_cast<const ST *>(a.data);
    const C *xT = static_cast<const C *>(a.xT);
    C *part = static_cast<C *>(a.part);

    const int g = blockIdx.x;
    const int t0 = a.grp_tile[g], t1 = a.grp_tile[g + 1];
    const int s1 = a.grp_off[g], n1 = a.grp_off[g + 1] - s1;
    const int ld1 = n1 | 1;
    const int RG = a.rg_stride;     // xT row length
    const int PS = a.nq * U;        // right-hand sides per pass
    const int HT = a.half;
    const int ncw = 2 * HT / 32;                 // consumer warps
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int k = 0; k < NZ_SLOTS; ++k) {
            mbar_init(&full[k], 1);              // the producer's arrive (with the tile's bytes)
            mbar_init(&empty[k], ncw);
        }
        *stop = 0;
        mbar_fence_init();
    }
    __syncthreads();

    if (warp == ncw) {
        // ------------------------------------------------------ producer
        // ring accounting: `used` bytes are reserved by the `count` tiles in
        // flight (a tile that wraps also reserves the unused end of the ring);
        // tiles are released in order, oldest first
        if (lane == 0) {
            const uint32_t R = a.ring_bytes;
            uint32_t head = 0, used = 0;
            uint32_t resv[NZ_SLOTS] = {};
            int oldest = 0, count = 0, ord = 0;
            int last[NZ_SLOTS];                  // latest tile issued into each slot
            for (int k = 0; k < NZ_SLOTS; ++k) last[k] = -1;
            bool halt = false;
            auto release_oldest = [&]() {
                const int k = oldest % NZ_SLOTS;
                if (!mbar_wait_or(&empty[k], (uint32_t)((oldest / NZ_SLOTS) & 1), a.err, stop)) halt = true;
                used -= resv[k];
                ++oldest;
                --count;
            };
            for (int r0 = 0; r0 < a.nrhs && !halt; r0 += PS) {
                const C *xp = xT + (long long)(r0 / PS) * a.n * RG;
                while (count > 0 && !halt) release_oldest();   // X1 is rewritten: the previous pass must be done
                for (int t = t0; t < t1 && !halt; ++t, ++ord) {
                    const NearTile &tl = a.tiles[t];
                    const uint32_t mb = (uint32_t)(tile_elems(tl.n1, tl.n2) * (long long)sizeof(ST));
                    const uint32_t xb = (uint32_t)(3 * tl.n2 * RG * sizeof(C));
                    const uint32_t x1b = t == t0 ? (uint32_t)(3 * n1 * RG * sizeof(C)) : 0u;
                    const uint32_t S = mb + xb;
                    bool fit = head + S <= R;
                    uint32_t res = fit ? S : (R - head) + S;
                    while (count > 0 && !halt && (count == NZ_SLOTS || used + res > R)) release_oldest();
                    if (halt || *stop) { halt = true; break; }
                    if (count == 0) { head = 0; used = 0; fit = true; res = S; }
                    const uint32_t st = fit ? head : 0u;
                    const int k = ord % NZ_SLOTS;
                    toff[k] = (int)st;
                    tn2[k] = tl.n2;
                    tcol[k] = tl.col_off;
                    mbar_expect_tx(&full[k], S + x1b);
                    bulk_g2s(ring + st, data + tl.data_off, mb, &full[k]);
                    bulk_g2s(ring + st + mb, xp + 3LL * tl.s2 * RG, xb, &full[k]);
                    if (x1b) bulk_g2s(X1, xp + 3LL * s1 * RG, x1b, &full[k]);
                    head = st + S;
                    used += res;
                    resv[k] = res;
                    last[k] = ord;
                    ++count;
                }
            }
            if (halt) {
                // a wait gave up: tell the consumers, then let every copy
                // still landing in the ring finish before the CTA exits
                *stop = 1;
                for (int k = 0; k < NZ_SLOTS; ++k)
                    if (last[k] >= 0) mbar_wait(&full[k], (uint32_t)((last[k] / NZ_SLOTS) & 1), a.err);
            }
        }
        return;
    }

    // ---------------------------------------------------------- consumers
    const bool rowside = warp < HT / 32;
    const int it = rowside ? threadIdx.x : threadIdx.x - HT;
    const bool row_item = rowside && it < n1 * a.nq * L;
    const int rq = row_item ? it / (n1 * L) : 0;
    const int ri = row_item ? (it - rq * n1 * L) / L : 0, hl = row_item ? (it - rq * n1 * L) % L : 0;
    int ord = 0;
    for (int r0 = 0; r0 < a.nrhs; r0 += PS) {
        const int rg = min(PS, a.nrhs - r0);
        C accs[NP][3][U];
#pragma unroll
        for (int p = 0; p < NP; ++p)
#pragma unroll
            for (int q = 0; q < 3; ++q)
#pragma unroll
                for (int u = 0; u < U; ++u) accs[p][q][u] = czero<C>();
        C (&acc)[3][U] = accs[0];
        for (int t = t0; t < t1; ++t, ++ord) {
            const int kslot = ord % NZ_SLOTS;
            bool ok = !*stop && mbar_wait_or(&full[kslot], (uint32_t)((ord / NZ_SLOTS) & 1), a.err, stop);
            ok = __all_sync(0xffffffffu, ok);   // the warp skips or computes as one (shuffles below)
            if (!ok) {
                *stop = 1;
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty[kslot]);
                continue;
            }
            const int n2 = tn2[kslot];
            const int tof = toff[kslot];
            const long long tcoff = tcol[kslot];
            const uint32_t M = smem_addr(ring + tof);
            const uint32_t X2 = M + (uint32_t)(tile_elems(n1, n2) * (long long)sizeof(ST));
            constexpr uint32_t SB = sizeof(ST), CB = sizeof(C);
            const uint32_t mrow = SB * ld1, xrow = CB * RG;   // bytes between planes / x rows
            if (rowside) {
                if (row_item) {
                    uint32_t mp = M + SB * ri;            // plane (9j + 3b), lane i
                    uint32_t xp = X2 + CB * U * rq;       // x row 3j + b
                    // one j: the three b-planes into partial pp
                    auto row_j = [&](C (&pp)[3][U]) {
#pragma unroll
                        for (int b = 0; b < 3; ++b) {
                            C xu[U];
                            load_xu<C, U>(xp, xu);
                            const C mm[3] = {as_c<C>(lds_c(mp, ST{})), as_c<C>(lds_c(mp + mrow, ST{})),
                                             as_c<C>(lds_c(mp + 2 * mrow, ST{}))};
                            mac3<C, U>(pp, mm, xu);
                            mp += 3 * mrow;
                            xp += xrow;
                        }
                    };
                    if constexpr (NP == 1) {
                        // lane hl takes j = hl, hl + L, ...
                        mp += hl * 9 * mrow;
                        xp += hl * 3 * xrow;
                        for (int j = hl; j < n2; j += L) {
                            row_j(acc);
                            mp += (L - 1) * 9 * mrow;
                            xp += (L - 1) * 3 * xrow;
                        }
                    } else {
                        for (int j = 0; j < n2; j += 2) {
                            row_j(accs[0]);
                            if (j + 1 < n2) row_j(accs[1]);
                        }
                    }
                }
            } else if (NS == 1 && tcoff >= 0 && it < n2 * a.nq) {
                const int q = it / n2, j = it - q * n2;
                C cacc[3][U];
#pragma unroll
                for (int b = 0; b < 3; ++b)
#pragma unroll
                    for (int u = 0; u < U; ++u) cacc[b][u] = czero<C>();
                const uint32_t mj = M + SB * 9 * j * ld1;
                uint32_t xp = smem_addr(X1) + CB * U * q;   // x row 3i + a
                for (int i = 0; i < n1; ++i) {
#pragma unroll
                    for (int aa = 0; aa < 3; ++aa) {
                        C xu[U];
                        load_xu<C, U>(xp, xu);
                        const uint32_t mp = mj + aa * mrow + SB * i;
                        const C mm[3] = {as_c<C>(lds_c(mp, ST{})), as_c<C>(lds_c(mp + 3 * mrow, ST{})),
                                         as_c<C>(lds_c(mp + 6 * mrow, ST{}))};
                        mac3<C, U>(cacc, mm, xu);
                        xp += xrow;
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int r = U * q + u;
                    if (r < rg && !(a.skip && a.skip[r0 + r])) {
                        C *pc = part + (r0 + r) * a.part_len + tcoff + 3 * j;
                        pc[0] = cacc[0][u];
                        pc[1] = cacc[1][u];
                        pc[2] = cacc[2][u];
                    }
                }
            } else if (NS > 1 && tcoff >= 0) {
                // split column sums: partial p over i = p, p + NS, ...; the
                // lanes of a column are adjacent (all lanes join the shuffle)
                const bool col_item = it < n2 * a.nq * L;
                const int q = col_item ? it / (n2 * L) : 0;
                const int j = col_item ? (it - q * n2 * L) / L : 0, cl = col_item ? (it - q * n2 * L) % L : 0;
                C cps[NP][3][U];
#pragma unroll
                for (int p = 0; p < NP; ++p)
#pragma unroll
                    for (int b = 0; b < 3; ++b)
#pragma unroll
                        for (int u = 0; u < U; ++u) cps[p][b][u] = czero<C>();
                if (col_item) {
                    const uint32_t mj = M + SB * 9 * j * ld1;
                    const uint32_t x0 = smem_addr(X1) + CB * U * q;   // x row 3i + a
                    auto col_i = [&](int i, C (&pp)[3][U]) {
                        uint32_t xp = x0 + 3 * i * xrow;
#pragma unroll
                        for (int aa = 0; aa < 3; ++aa) {
                            C xu[U];
                            load_xu<C, U>(xp, xu);
                            const uint32_t mp = mj + aa * mrow + SB * i;
                            const C mm[3] = {as_c<C>(lds_c(mp, ST{})), as_c<C>(lds_c(mp + 3 * mrow, ST{})),
                                             as_c<C>(lds_c(mp + 6 * mrow, ST{}))};
                            mac3<C, U>(pp, mm, xu);
                            xp += xrow;
                        }
                    };
                    if constexpr (NP == 1) {
                        for (int i = cl; i < n1; i += L) col_i(i, cps[0]);
                    } else {
                        for (int i = 0; i < n1; i += 2) {
                            col_i(i, cps[0]);
                            if (i + 1 < n1) col_i(i + 1, cps[1]);
                        }
                    }
                }
                C ctot[3][U];
                combine_split<C, U, NP, L>(cps, ctot);
                if (col_item && cl == 0) {
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int r = U * q + u;
                        if (r < rg && !(a.skip && a.skip[r0 + r])) {
                            C *pc = part + (r0 + r) * a.part_len + tcoff + 3 * j;
                            pc[0] = ctot[0][u];
                            pc[1] = ctot[1][u];
                            pc[2] = ctot[2][u];
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[kslot]);
        }
        if constexpr (NS > 1) {
            if (rowside) {
                // all row-side lanes take part in the combination (shuffles)
                C tot[3][U];
                combine_split<C, U, NP, L>(accs, tot);
#pragma unroll
                for (int q = 0; q < 3; ++q)
#pragma unroll
                    for (int u = 0; u < U; ++u) acc[q][u] = tot[q][u];
            }
        }
        if (row_item && hl == 0) {
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int r = U * rq + u;
                if (r < rg && !(a.skip && a.skip[r0 + r])) {
                    C *pr = part + (r0 + r) * a.part_len + a.pslot_base[g] + 3 * ri;
                    pr[0] = acc[0][u];
                    pr[1] = acc[1][u];
                    pr[2] = acc[2][u];
                }
            }
        }
    }
}

// ---------------------------------------------------------------- gather
// Interpolation (sparse_eps_matmul, src/sparse.f90:47-77) and final
// assembly (src/gmres_module.f90:148-170), one warp per (near-zone group,
// span of rspan right-hand sides), one lane per tet, GA_RG right-hand sides
// at a time: the 27 box-node values of the four result grids are staged in
// shared memory, each lane forms its tet's six 27-term sums from the
// projector rows P[(g*27 + j)*T + slot] (coalesced across lanes; they stay
// in L1 for the next group of the span), adds the group's near-zone partial
// slots in slot order and writes Ax = near + (Y2 - k^2 Y).  The spans are the
// grid's y index; rspan is a multiple of GA_RG.
template <typename C, int GA_RG>
__global__ void __launch_bounds__(32 * WARPS_PER_CTA, sizeof(C) == 8 ? SCD_GATHER_MINB : 1)
k_gather(const C *__restrict__ Rg, const C *__restrict__ P, int T, const int *__restrict__ grp_off,
         const int *__restrict__ grp_cube, int ngroups, GridDims G, typename CReal<C>::type k2,
         const C *__restrict__ part, long long part_len, const long long *__restrict__ pslot_base,
         const int *__restrict__ pslot_cnt, C *__restrict__ y, long long ld, const int *skip, int nrhs,
         int rspan) {
    __shared__ C Rs[WARPS_PER_CTA][GA_RG][4][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int gq = blockIdx.x * WARPS_PER_CTA + warp;
    if (gq >= ngroups) return;
    const int s0 = grp_off[gq], s1 = grp_off[gq + 1];
    const int nc = s1 - s0;
    const int c = grp_cube[gq];
    const int bx = c % G.ncx, by = (c / G.ncx) % G.ncy, bz = c / (G.ncx * G.ncy);
    const long long NN = (long long)G.Nx * G.Ny * G.Nz;
    const long long pbase = pslot_base[gq];
    const int nslot = pslot_cnt[gq];
    long long node = 0;
    if (lane < 27) {
        const int a = lane % 3, b = (lane / 3) % 3, cc = lane / 9;
        node = ((long long)(2 * bz + cc) * G.Ny + (2 * by + b)) * G.Nx + (2 * bx + a);
    }
    const int rend = min(nrhs, (int)(blockIdx.y + 1) * rspan);
    for (int r0 = blockIdx.y * rspan; r0 < rend; r0 += GA_RG) {
        __syncwarp();
        if (lane < 27) {
#pragma unroll
            for (int q = 0; q < GA_RG; ++q) {
                const int r = r0 + q;
                if (r < nrhs) {
                    const C *Rr = Rg + (long long)r * 4 * NN;
#pragma unroll
                    for (int g = 0; g < 4; ++g) Rs[warp][q][g][lane] = Rr[g * NN + node];
                }
            }
        }
        __syncwarp();
        for (int sl = lane; sl < nc; sl += 32) {
            const int s = s0 + sl;
            C acc[GA_RG][6];
#pragma unroll
            for (int q = 0; q < GA_RG; ++q)
#pragma unroll
                for (int v = 0; v < 6; ++v) acc[q][v] = czero<C>();
#pragma unroll 3
            for (int j = 0; j < 27; ++j) {
                const C p0 = P[(size_t)j * T + s], px = P[(size_t)(27 + j) * T + s];
                const C py = P[(size_t)(54 + j) * T + s], pz = P[(size_t)(81 + j) * T + s];
#pragma unroll
                for (int q = 0; q < GA_RG; ++q) {
                    cfma(acc[q][0], p0, Rs[warp][q][0][j]);
                    cfma(acc[q][1], p0, Rs[warp][q][1][j]);
                    cfma(acc[q][2], p0, Rs[warp][q][2][j]);
                    const C r3 = Rs[warp][q][3][j];
                    cfma(acc[q][3], px, r3);
                    cfma(acc[q][4], py, r3);
                    cfma(acc[q][5], pz, r3);
                }
            }
            // far field first (acc dies), then the partial slots of all
            // right-hand sides of the round in one sweep over the slots, so
            // that 3 GA_RG independent loads are in flight per slot; each sum
            // still runs over the slots in order
            C far[GA_RG][3], nz[GA_RG][3];
            bool on[GA_RG];
#pragma unroll
            for (int q = 0; q < GA_RG; ++q) {
                const int r = r0 + q;
                on[q] = r < nrhs && !(skip && skip[r]);
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    far[q][d] = csub_scaled(acc[q][3 + d], k2, acc[q][d]);
                    nz[q][d] = czero<C>();
                }
            }
            const C *pr0 = part + pbase + 3 * sl;
#pragma unroll 2
            for (int t = 0; t < nslot; ++t) {
                const C *pt = pr0 + (long long)t * 3 * nc;
#pragma unroll
                for (int q = 0; q < GA_RG; ++q) {
                    if (!on[q]) continue;
                    const C *pq = pt + (r0 + q) * part_len;
#pragma unroll
                    for (int d = 0; d < 3; ++d) nz[q][d] = cadd(nz[q][d], pq[d]);
                }
            }
#pragma unroll
            for (int q = 0; q < GA_RG; ++q) {
                if (!on[q]) continue;
                C *yr = y + (r0 + q) * ld + 3LL * s;
#pragma unroll
                for (int d = 0; d < 3; ++d) yr[d] = cadd(nz[q][d], far[q][d]);
            }
        }
    }
}

__global__ void k_twiddles(cd *tw, int P) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < P) {
        double s, c;
        sincospi(-2.0 * (double)i / (double)P, &s, &c);
        tw[i] = cmk(c, s);
    }
}

__global__ void k_narrow(const cd *in, cf *out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = make_float2((float)in[i].x, (float)in[i].y);
}

GridDims dims_of(const scd_ctx *c) {
    GridDims G;
    G.Nx = c->Nx; G.Ny = c->Ny; G.Nz = c->Nz;
    G.Px = c->Px; G.Py = c->Py; G.Pz = c->Pz;
    G.Hx = c->Hx; G.Hy = c->Hy; G.Hz = c->Hz;
    G.ncx = c->ncx; G.ncy = c->ncy; G.ncz = c->ncz; G.ncubes = c->ncubes;
    return G;
}

// operator copies and work buffers of one precision
template <typename C> struct Res;
template <> struct Res<cd> {
    static const cd *P(scd_ctx *c) { return c->d_P; }
    static const cd *Fo(scd_ctx *c) { return c->d_Fo; }
    static const cd *Fyz(scd_ctx *c) { return c->d_Fyz; }
    static const cd *tw(scd_ctx *c, int a) { return c->d_tw[a]; }
    static cd *bpart(scd_ctx *c) { return c->d_bpart; }
    static cd *W(scd_ctx *c) { return c->d_W; }
    static cd *R(scd_ctx *c) { return c->d_R; }
    static cd *part(scd_ctx *c) { return c->d_nzpart; }
    static cd *xT(scd_ctx *c) { return c->d_xT; }
};
template <> struct Res<cf> {
    static const cf *P(scd_ctx *c) { return c->f_P; }
    static const cf *Fo(scd_ctx *c) { return c->f_Fo; }
    static const cf *Fyz(scd_ctx *c) { return c->f_Fyz; }
    static const cf *tw(scd_ctx *c, int a) { return c->f_tw[a]; }
    static cf *bpart(scd_ctx *c) { return c->f_bpart; }
    static cf *W(scd_ctx *c) { return c->f_W; }
    static cf *R(scd_ctx *c) { return c->f_R; }
    static cf *part(scd_ctx *c) { return c->f_nzpart; }
    static cf *xT(scd_ctx *c) { return c->f_xT; }
};

template <int P, typename C>
void fft_x_fwd_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw, bool tl) {
    using Cf = FftCfg<P, C>;
    dim3 grid((G.Ny * G.Nz + Cf::LPB - 1) / Cf::LPB, nrg);
    if (tl) k_fft_x_fwd<P, C, true><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::bpart(c), Res<C>::W(c), tw, G, done);
    else k_fft_x_fwd<P, C, false><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::bpart(c), Res<C>::W(c), tw, G, done);
}
template <int P, bool INV, typename C>
void fft_y_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw) {
    using Cf = FftCfg<P, C>;
    dim3 grid(((G.Px + Cf::LPB - 1) / Cf::LPB) * G.Nz, nrg);
    k_fft_y<P, INV, C><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), tw, G, done);
}
template <int P, typename C>
void fft_z_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw) {
    using Cf = FftCfg<P, C>;
    dim3 grid(((G.Px + Cf::LPB - 1) / Cf::LPB) * G.Py, nrg);
    k_fft_z<P, C><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), Res<C>::Fo(c), tw, G, done);
}
template <int P, typename C>
void fft_x_inv_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw, bool tl) {
    using Cf = FftCfg<P, C>;
    dim3 grid((G.Ny * G.Nz + Cf::LPB - 1) / Cf::LPB, nrg);
    if (tl) k_fft_x_inv<P, C, true><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), Res<C>::R(c), tw, G, done);
    else k_fft_x_inv<P, C, false><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), Res<C>::R(c), tw, G, done);
}

// the fused y-z pass (fft_yz.cuh) for one (PY, PZ) pair
template <int PY, int PZ, typename C>
void fft_yz_t(scd_ctx *c, const GridDims &G, int nrg, const int *done) {
    if constexpr (YzLine<PY>::OK && YzLine<PZ>::OK) {
        YzDims D;
        D.Nx = G.Nx; D.Ny = G.Ny; D.Nz = G.Nz; D.NzR = yz_round8(G.Nz);
        D.Px = G.Px; D.Hx = G.Hx; D.Hy = G.Hy; D.Hz = G.Hz;
        const size_t sh = sizeof(C) * (size_t)yz_smem_elems<PY, PZ>(D.NzR);
        cudaFuncSetAttribute(k_fft_yz<PY, PZ, C>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
        k_fft_yz<PY, PZ, C><<<dim3(G.Px, nrg), YZ_THREADS, sh, c->st>>>(Res<C>::W(c), Res<C>::Fyz(c), Res<C>::tw(c, 1),
                                                                       Res<C>::tw(c, 2), D, done);
    }
}

template <int PY, typename C>
void fft_yz_pz(scd_ctx *c, const GridDims &G, int nrg, const int *done) {
    switch (G.Pz) {
        case 64: fft_yz_t<PY, 64, C>(c, G, nrg, done); break;
        case 80: fft_yz_t<PY, 80, C>(c, G, nrg, done); break;
        case 96: fft_yz_t<PY, 96, C>(c, G, nrg, done); break;
        case 128: fft_yz_t<PY, 128, C>(c, G, nrg, done); break;
        case 192: fft_yz_t<PY, 192, C>(c, G, nrg, done); break;
        default: break;
    }
}

template <typename C>
void fft_yz(scd_ctx *c, const GridDims &G, int nrg, const int *done) {
    switch (G.Py) {
        case 64: fft_yz_pz<64, C>(c, G, nrg, done); break;
        case 80: fft_yz_pz<80, C>(c, G, nrg, done); break;
        case 96: fft_yz_pz<96, C>(c, G, nrg, done); break;
        case 128: fft_yz_pz<128, C>(c, G, nrg, done); break;
        case 192: fft_yz_pz<192, C>(c, G, nrg, done); break;
        default: break;
    }
}

constexpr bool yz_len_ok(int P) { return P == 64 || P == 80 || P == 96 || P == 128 || P == 192; }

// shared-memory bytes of the fused y-z pass for the context's lengths
template <typename C>
size_t yz_smem_bytes(const scd_ctx *c) {
    const int NzR = yz_round8(c->Nz);
    auto tpl = [](int P) { return (P == 64 || P == 128 || P % 64 == 0) ? 8 : 4; };
    auto lines = [&](int P) { return YZ_THREADS / tpl(P); };
    auto ls = [&](int P) { return yz_line_stride(P, tpl(P)); };
    return sizeof(C) * (size_t)(c->Py + c->Pz + (long long)NzR * ls(c->Py) + (long long)lines(c->Pz) * ls(c->Pz));
}

// whether the complex64 (or FP64) chain takes the fused y-z pass: both lengths
// have warp-synchronous line transforms and the CTA fits shared memory
template <typename C>
bool use_yz(const scd_ctx *c) {
    if (!c->yz_on || !yz_len_ok(c->Py) || !yz_len_ok(c->Pz)) return false;
    return yz_smem_bytes<C>(c) <= (size_t)(227 * 1024);
}

// the transposed Green octant of the fused pass, built from Fo once per
// Green spectrum; false (three-pass chain) if it cannot be allocated
template <typename C>
bool ensure_fyz(scd_ctx *c) {
    constexpr bool single = std::is_same<C, cf>::value;
    bool &ready = single ? c->fyz_ready_f : c->fyz_ready;
    if (ready) return true;
    C *&buf = *reinterpret_cast<C **>(single ? (void *)&c->f_Fyz : (void *)&c->d_Fyz);
    const long long no = (long long)c->Hx * c->Hy * c->Hz;
    if (!buf && cudaMalloc((void **)&buf, sizeof(C) * (size_t)no) != cudaSuccess) {
        cudaGetLastError();
        buf = nullptr;
        return false;
    }
    k_green_yz<C><<<(unsigned)std::min<long long>((no + 255) / 256, 4096), 256, 0, c->st>>>(Res<C>::Fo(c), buf, c->Hx,
                                                                                          c->Hy, c->Hz);
    ready = true;
    return true;
}

#define SCD_DISPATCH_P(PV, CALL)                     \
    switch (PV) {                                    \
        case 8: CALL(8); break;                      \
        case 16: CALL(16); break;                    \
        case 32: CALL(32); break;                    \
        case 64: CALL(64); break;                    \
        case 128: CALL(128); break;                  \
        case 80: CALL(80); break;                    \
        case 96: CALL(96); break;                    \
        case 192: CALL(192); break;                  \
        case 256: CALL(256); break;                  \
        case 512: CALL(512); break;                  \
        default: break;                              \
    }

template <typename C>
void fft_chain_t(scd_ctx *c, const C *x, int nrhs, const int *done) {
    const GridDims G = dims_of(c);
    {
        const unsigned gx = (unsigned)((c->ncubes + WARPS_PER_CTA - 1) / WARPS_PER_CTA);
        const C *P = Res<C>::P(c);
        // spans of right-hand sides per warp (c->scatter_span, 0 = all of them)
        auto span = [&](int rg) { int sp = c->scatter_span > 0 ? c->scatter_span : nrhs; return (sp + rg - 1) / rg * rg; };
        if (nrhs >= 8 && SCD_SG_CTA) {
            // one CTA per cube (projector rows shared through shared memory)
            constexpr int NTC = sizeof(C) == 8 ? 32 : 16;
            const int sp = span(4);
            k_scatter_cta<C, NTC, 4><<<dim3((unsigned)c->ncubes, (nrhs + sp - 1) / sp), SCB, 0, c->st>>>(
                x, c->n, P, c->T, c->d_cube_off, c->ncubes, Res<C>::bpart(c), done, nrhs, sp);
        } else if (nrhs >= 8) {
            const int sp = span(8);
            k_scatter<C, 8><<<dim3(gx, (nrhs + sp - 1) / sp), 32 * WARPS_PER_CTA, 0, c->st>>>(
                x, c->n, P, c->T, c->d_cube_off, c->ncubes, Res<C>::bpart(c), done, nrhs, sp);
        } else if (nrhs >= 4) {
            const int sp = span(4);
            k_scatter<C, 4><<<dim3(gx, (nrhs + sp - 1) / sp), 32 * WARPS_PER_CTA, 0, c->st>>>(
                x, c->n, P, c->T, c->d_cube_off, c->ncubes, Res<C>::bpart(c), done, nrhs, sp);
        } else {
            const int sp = span(1);
            k_scatter<C, 1><<<dim3(gx, (nrhs + sp - 1) / sp), 32 * WARPS_PER_CTA, 0, c->st>>>(
                x, c->n, P, c->T, c->d_cube_off, c->ncubes, Res<C>::bpart(c), done, nrhs, sp);
        }
    }
    const int nrg = 4 * nrhs;
    const bool tl = use_yz<C>(c) && ensure_fyz<C>(c);
#define XF(PP) fft_x_fwd_t<PP, C>(c, G, nrg, done, Res<C>::tw(c, 0), tl)
#define YF(PP) fft_y_t<PP, false, C>(c, G, nrg, done, Res<C>::tw(c, 1))
#define ZC(PP) fft_z_t<PP, C>(c, G, nrg, done, Res<C>::tw(c, 2))
#define YI(PP) fft_y_t<PP, true, C>(c, G, nrg, done, Res<C>::tw(c, 1))
#define XI(PP) fft_x_inv_t<PP, C>(c, G, nrg, done, Res<C>::tw(c, 0), tl)
    SCD_DISPATCH_P(c->Px, XF)
    if (tl) {
        fft_yz<C>(c, G, nrg, done);
    } else {
        SCD_DISPATCH_P(c->Py, YF)
        SCD_DISPATCH_P(c->Pz, ZC)
        SCD_DISPATCH_P(c->Py, YI)
    }
    SCD_DISPATCH_P(c->Px, XI)
#undef XF
#undef YF
#undef ZC
#undef YI
#undef XI
    c->launches += tl ? 4 : 6;
}

template <typename ST, typename C, int U, int NS>
void near_launch(scd_ctx *c, const ST *data, const C *x, int nrhs, const int *done) {
    NearPass a;
    a.tiles = c->d_tiles; a.grp_tile = c->d_grp_tile; a.grp_off = c->d_grp_off; a.pslot_base = c->d_pslot_base;
    a.data = data; a.xT = Res<C>::xT(c); a.n = c->n; a.part = Res<C>::part(c); a.part_len = c->part_len;
    a.skip = done; a.nrhs = nrhs;
    a.err = c->d_kerr;
    const int nq = U == 1 ? 1 : std::min(NZ_QMAX, (nrhs + U - 1) / U);
    a.nq = nq;
    a.half = 32 * ((c->max_per_group * a.nq * (U == 1 ? NS : 1) + 31) / 32);   // lanes per side
    // xT rows are whole 16-byte units (bulk-copy granularity)
    a.rg_stride = nq * U;
    while ((a.rg_stride * sizeof(C)) % 16) ++a.rg_stride;
    a.x1_bytes = (uint32_t)(3 * c->max_per_group * a.rg_stride * sizeof(C));
    // the ring fills what two CTAs per SM leave, and must hold the largest tile with its x
    const size_t max_tile = (size_t)c->max_tile_store * sizeof(ST) + a.x1_bytes;
    size_t ring = ((U == 1 ? NZ_SMEM_4CTA : NZ_SMEM_2CTA) - NZ_META - a.x1_bytes) / 16 * 16;
    if (ring < max_tile) ring = std::min((NZ_SMEM_MAX - NZ_META - a.x1_bytes) / 16 * 16, (max_tile + 15) / 16 * 16 * 2);
    if (ring < max_tile) {
        // cannot happen with groups of at most SCD_GROUP_MAX slots; reported
        // by near_status instead of overrunning the ring
        c->near_cfg_err = 1;
        return;
    }
    a.ring_bytes = (uint32_t)ring;
    {
        const int npass = (nrhs + nq * U - 1) / (nq * U);
        dim3 g((unsigned)((c->n + 255) / 256), npass);
        k_xpose<C><<<g, 256, 0, c->st>>>(x, c->n, c->n, nrhs, nq * U, a.rg_stride, Res<C>::xT(c));
        c->launches += 1;
    }
    const size_t sh = NZ_META + a.x1_bytes + a.ring_bytes;
    cudaFuncSetAttribute(k_near_groups<ST, C, U, NS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    if (c->timing) cudaEventRecord(c->ev[6], c->st);
    k_near_groups<ST, C, U, NS><<<c->ngroups, 2 * a.half + 32, sh, c->st>>>(a);
    if (c->timing) cudaEventRecord(c->ev[7], c->st);
}

template <typename ST, typename C>
void near_dispatch(scd_ctx *c, const ST *data, const C *x, int nrhs, const int *done) {
    // near_split 2 (the default): two partial sums per row and column (two
    // lanes each at one right-hand side, both in one lane at four) for the
    // FP64 matvec, the same arithmetic per sum at U = 1 and U = 4, so a column
    // keeps its bits alone and in a batch; the complex64 matvec of the mixed
    // form keeps one sum per lane (its U = 4 kernel would lose occupancy to
    // the second set of accumulators)
    if (c->near_split == 2 && std::is_same<C, cd>::value) {
        if (nrhs == 1) near_launch<ST, C, 1, 2>(c, data, x, nrhs, done);
        else near_launch<ST, C, 4, 2>(c, data, x, nrhs, done);
    } else {
        if (nrhs == 1) near_launch<ST, C, 1, 1>(c, data, x, nrhs, done);
        else near_launch<ST, C, 4, 1>(c, data, x, nrhs, done);
    }
}

template <typename C>
void near_t(scd_ctx *c, const C *x, int nrhs, const int *done) {
    if (c->ngroups == 0) return;
    if constexpr (std::is_same<C, cf>::value) {
        if (c->nzm_on && c->nzm_ready) {
            near_mma_run(c, x, nrhs, done);
            return;
        }
    }
    if (c->near_prec == SCD_STORE_C64) near_dispatch<cf, C>(c, (const cf *)c->d_tdata, x, nrhs, done);
    else near_dispatch<cd, C>(c, (const cd *)c->d_tdata, x, nrhs, done);
    c->launches += 1;
}

template <typename C>
void gather_t(scd_ctx *c, C *y, int nrhs, const int *done) {
    const GridDims G = dims_of(c);
    const unsigned gx = (unsigned)((c->ngroups + WARPS_PER_CTA - 1) / WARPS_PER_CTA);
    if (c->ngroups == 0) return;
    typedef typename CReal<C>::type R;
    const R k2 = (R)(c->k * c->k);
    // spans of right-hand sides per warp (c->gather_span, 0 = all of them)
    auto span = [&](int rg) { int sp = c->gather_span > 0 ? c->gather_span : nrhs; return (sp + rg - 1) / rg * rg; };
    if (nrhs >= 4) {
        const int sp = span(4);
        k_gather<C, 4><<<dim3(gx, (nrhs + sp - 1) / sp), 32 * WARPS_PER_CTA, 0, c->st>>>(
            Res<C>::R(c), Res<C>::P(c), c->T, c->d_grp_off, c->d_grp_cube, c->ngroups, G, k2, Res<C>::part(c),
            c->part_len, c->d_pslot_base, c->d_pslot_cnt, y, c->n, done, nrhs, sp);
    } else {
        const int sp = span(1);
        k_gather<C, 1><<<dim3(gx, (nrhs + sp - 1) / sp), 32 * WARPS_PER_CTA, 0, c->st>>>(
            Res<C>::R(c), Res<C>::P(c), c->T, c->d_grp_off, c->d_grp_cube, c->ngroups, G, k2, Res<C>::part(c),
            c->part_len, c->d_pslot_base, c->d_pslot_cnt, y, c->n, done, nrhs, sp);
    }
    c->launches += 1;
}

template <typename C>
void run_matvec_t(scd_ctx *c, const C *x, C *y, int nrhs, const int *done) {
    if (c->timing) cudaEventRecord(c->ev[0], c->st);
    {
        NvtxRange r("near zone");
        near_t<C>(c, x, nrhs, done);
    }
    if (c->timing) cudaEventRecord(c->ev[1], c->st);
    {
        NvtxRange r("fft convolutions");
        fft_chain_t<C>(c, x, nrhs, done);
    }
    if (c->timing) cudaEventRecord(c->ev[2], c->st);
    {
        NvtxRange r("gather");
        gather_t<C>(c, y, nrhs, done);
    }
    if (c->timing) cudaEventRecord(c->ev[3], c->st);
}

}  // namespace

// twiddle table exp(-2 pi i j / P), j < P
int build_twiddles(scd_ctx *c, int P, cd **out) {
    cudaError_t e = cudaMalloc(out, sizeof(cd) * P);
    if (e != cudaSuccess) return check_cuda(c, e, "twiddles");
    k_twiddles<<<(P + 255) / 256, 256, 0, c->st>>>(*out, P);
    return check_cuda(c, cudaGetLastError(), "twiddles");
}

// complex64 copies of the projectors, the Green octant and the twiddles for
// the mixed-precision inner solves (rounded from the FP64 operator)
int ensure_single(scd_ctx *c) {
    // the tensor-core near zone reads complex64 tiles; by default a context
    // with complex128 storage keeps the CUDA-core kernel, an explicit request
    // is an error (near_mma_prepare)
    if (c->nzm_on && !c->nzm_ready && c->have_near && c->ngroups > 0 &&
        (c->near_prec == SCD_STORE_C64 || c->d.near_kernel != SCD_NEAR_DEFAULT)) {
        const int rc = near_mma_prepare(c);
        if (rc) return rc;
    }
    if (c->f_ready) return SCD_OK;
    const long long np = 4LL * 27 * c->T, no = (long long)c->Hx * c->Hy * c->Hz;
    auto al = [&](cf **p, long long n) -> int {
        if (*p) { cudaFree(*p); *p = nullptr; }
        if (cudaMalloc(p, sizeof(cf) * (size_t)std::max<long long>(n, 1)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, SCD_OOM, "complex64 operator copy");
        }
        return SCD_OK;
    };
    int rc;
    if ((rc = al(&c->f_P, np)) || (rc = al(&c->f_Fo, no))) return rc;
    k_narrow<<<1024, 256, 0, c->st>>>(c->d_P, c->f_P, np);
    k_narrow<<<1024, 256, 0, c->st>>>(c->d_Fo, c->f_Fo, no);
    const int Ps[3] = {c->Px, c->Py, c->Pz};
    for (int a = 0; a < 3; ++a) {
        if ((rc = al(&c->f_tw[a], Ps[a]))) return rc;
        k_narrow<<<(Ps[a] + 255) / 256, 256, 0, c->st>>>(c->d_tw[a], c->f_tw[a], Ps[a]);
    }
    rc = check_cuda(c, cudaStreamSynchronize(c->st), "complex64 operator copy");
    if (!rc) c->f_ready = true;
    return rc;
}

int ensure_work_single(scd_ctx *c, int nrhs) {
    if (c->f_cap >= nrhs && c->f_W) return SCD_OK;
    const size_t r = (size_t)nrhs;
    auto al = [&](cf **p, size_t n) -> int {
        if (*p) { cudaFree(*p); *p = nullptr; }
        if (cudaMalloc(p, sizeof(cf) * std::max<size_t>(n, 1)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, SCD_OOM, "complex64 work buffers (%d right-hand sides)", nrhs);
        }
        return SCD_OK;
    };
    int rc;
    if ((rc = al(&c->f_bpart, r * c->ncubes * 4 * 27)) || (rc = al(&c->f_W, r * 4 * (size_t)c->Px * c->Py * c->Nz)) ||
        (rc = al(&c->f_R, r * 4 * (size_t)c->Nx * c->Ny * c->Nz)) ||
        (rc = al(&c->f_nzpart, r * (size_t)std::max<long long>(c->part_len, 1))) ||
        (rc = al(&c->f_xT, (size_t)xt_columns(nrhs) * c->n)))
        return rc;
    c->f_cap = nrhs;
    return SCD_OK;
}

void launch_permute_in(scd_ctx *c, const cd *x_orig, cd *x_slot, int nrhs, long long ld) {
    dim3 grid((unsigned)std::min<long long>((3LL * c->T + 255) / 256, 4096), nrhs);
    k_permute_in<<<grid, 256, 0, c->st>>>(x_orig, x_slot, c->d_perm, c->T, ld, c->nb);
}

void launch_permute_out(scd_ctx *c, const cd *x_slot, cd *x_orig, int nrhs, long long ld) {
    dim3 grid((unsigned)std::min<long long>((3LL * c->T + 255) / 256, 4096), nrhs);
    k_permute_out<<<grid, 256, 0, c->st>>>(x_slot, x_orig, c->d_perm, c->T, ld, c->nb);
}

void launch_fft_chain(scd_ctx *c, const cd *x, int nrhs, const int *done) { fft_chain_t<cd>(c, x, nrhs, done); }
void launch_near(scd_ctx *c, const cd *x, int nrhs, const int *done) { near_t<cd>(c, x, nrhs, done); }
void launch_gather(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done) {
    (void)x;
    gather_t<cd>(c, y, nrhs, done);
}
void run_matvec(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done) { run_matvec_t<cd>(c, x, y, nrhs, done); }
void run_matvec(scd_ctx *c, const cf *x, cf *y, int nrhs, const int *done) { run_matvec_t<cf>(c, x, y, nrhs, done); }
