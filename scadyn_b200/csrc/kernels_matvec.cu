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

#include "ctx.h"

namespace {

constexpr int WARPS_PER_CTA = 4;

__global__ void k_permute_in(const cd *__restrict__ xo, cd *__restrict__ xs, const int *__restrict__ perm,
                             int T, long long ld) {
    const int r = blockIdx.y;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3LL * T; i += (long long)gridDim.x * blockDim.x) {
        long long s = i / 3, d = i - 3 * s;
        xs[r * ld + i] = xo[r * ld + 3LL * perm[s] + d];
    }
}

__global__ void k_permute_out(const cd *__restrict__ xs, cd *__restrict__ xo, const int *__restrict__ perm,
                              int T, long long ld) {
    const int r = blockIdx.y;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < 3LL * T; i += (long long)gridDim.x * blockDim.x) {
        long long s = i / 3, d = i - 3 * s;
        xo[r * ld + 3LL * perm[s] + d] = xs[r * ld + i];
    }
}

// ---------------------------------------------------------------- scatter
// Anterpolation (sparse_T_matmul, src/sparse.f90:13-43), one warp per cube:
// lane j < 27 accumulates the four box-node sums of node j over the cube's
// tets, for a group of right-hand sides at a time (projector values are read
// once per group).  Projectors are stored P[(g*27 + j)*T + slot].
// bpart[((r*ncubes + c)*4 + g)*27 + j].
template <typename C, int SC_RG>
__global__ void __launch_bounds__(32 * WARPS_PER_CTA)
k_scatter(const C *__restrict__ x, long long ld, const C *__restrict__ P, int T,
          const int *__restrict__ cube_off, int ncubes, C *__restrict__ bpart, const int *skip, int nrhs) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * WARPS_PER_CTA + warp;
    if (c >= ncubes || lane >= 27) return;
    const int s0 = cube_off[c], s1 = cube_off[c + 1];
    const C *P0 = P + (size_t)lane * T, *PX = P + (size_t)(27 + lane) * T;
    const C *PY = P + (size_t)(54 + lane) * T, *PZ = P + (size_t)(81 + lane) * T;
    for (int r0 = 0; r0 < nrhs; r0 += SC_RG) {
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

// in-line padding: one spare slot per 16 complex values spreads the
// strided Stockham writes over the shared-memory banks
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }

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

template <int P> struct FftCfg {
    static constexpr int TPL = P / 4;                        // threads per line
    static constexpr int LPB = (256 / TPL) > 0 ? 256 / TPL : 1;   // lines per CTA
    static constexpr int THREADS = TPL * LPB;
    static constexpr int LS = P + (P >> 4) + 1;              // padded line stride (bank spread)
};

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
// zero padding x >= Nx.  W[(rg)][(z*Py + y)*Px + x]
template <int P, typename Cx>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_x_fwd(const Cx *__restrict__ bpart, Cx *__restrict__ W, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P>;
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
    fft_line<P, false, Cx>(sh + l * Cf::LS, tw, t);
    Cx *Wr = W + (long long)rg * G.Px * G.Py * G.Nz;
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int ll = e / P, x = e - ll * P, line = line0 + ll;
        if (line < nlines) {
            const int y = line % G.Ny, z = line / G.Ny;
            Wr[((long long)z * G.Py + y) * G.Px + x] = sh[ll * Cf::LS + pidx(x)];
        }
    }
}

// Y pass: lines (x < Px, z < Nz); forward reads y < Ny and writes y < Py,
// inverse reads y < Py and writes y < Ny.  A CTA takes LPB consecutive x.
template <int P, bool INV, typename Cx>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_y(Cx *__restrict__ W, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P>;
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
    fft_line<P, INV, Cx>(sh + l * Cf::LS, tw, t);
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int y = e / Cf::LPB, ll = e - y * Cf::LPB, x = x0 + ll;
        if (y < nout && x < G.Px) Wr[(long long)y * G.Px + x] = sh[ll * Cf::LS + pidx(y)];
    }
}

// Z pass: lines (x < Px, y < Py), forward FFT of z < Nz (zero padded), times
// the Green octant Fo (folded by evenness), inverse FFT, keep z < Nz.
template <int P, typename Cx>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_z(Cx *__restrict__ W, const Cx *__restrict__ Fo, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P>;
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
    fft_line<P, false, Cx>(sh + l * Cf::LS, tw, t);
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
    fft_line<P, true, Cx>(sh + l * Cf::LS, tw, t);
    for (int e = threadIdx.x; e < Cf::LPB * P; e += blockDim.x) {
        const int z = e / Cf::LPB, ll = e - z * Cf::LPB, x = x0 + ll;
        if (z < G.Nz && x < G.Px) Wr[(long long)z * plane + x] = sh[ll * Cf::LS + pidx(z)];
    }
}

// X inverse: lines (y < Ny, z < Nz), keep x < Nx, write the result grid
// R[(rg)][(z*Ny + y)*Nx + x]
template <int P, typename Cx>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_x_inv(const Cx *__restrict__ W, Cx *__restrict__ R, const Cx *__restrict__ twg, GridDims G, const int *done) {
    if (done && done[blockIdx.y >> 2]) return;
    using Cf = FftCfg<P>;
    __shared__ Cx sh[Cf::LPB * Cf::LS];
    __shared__ Cx tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int nlines = G.Ny * G.Nz;
    const int line0 = blockIdx.x * Cf::LPB;
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
    __syncthreads();
    const int l = threadIdx.x / Cf::TPL, t = threadIdx.x - l * Cf::TPL;
    fft_line<P, true, Cx>(sh + l * Cf::LS, tw, t);
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
// Row sums y(c1) += M x(c2) and, for off-diagonal tiles, column sums
// y(c2) += M^T x(c1) (transpose, not conjugate: the operator is complex
// symmetric, src/sparse_mat.f90:113-116).  M(3i+a, 3j+b) is entry (a,b) of
// block (i,j), stored at D[(i*n2 + j)*9 + a + 3b].  Results go to per-cube
// partial slots that k_gather adds in a fixed order (deterministic).
constexpr int NZ_MAXN = 64;            // tets per cube supported (two lanes' worth)

// One warp per tile (4 tiles per CTA).  Tile rows stream through a
// two-row shared-memory ring with cp.async (coalesced 8/16-byte copies): row
// i+1 is in flight while row i is used.  Lane j takes block (i, j) from
// shared memory and applies it to RG right-hand sides; each row sum is
// reduced across the warp (xor tree), column j accumulates in lane j over the
// rows in order.  The arithmetic of one right-hand side is the same for every
// RG, so a column's result does not depend on the batch it is solved in.
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

template <typename ST>
__device__ __forceinline__ void copy_row_async(ST *dst, const ST *src, int nel, int lane) {
    for (int e = lane; e < nel; e += 32) {
        if (sizeof(ST) == 8) cp_async8(dst + e, src + e);
        else cp_async16(dst + e, src + e);
    }
    cp_async_commit();
}

constexpr int NZ_WARPS = 4;

template <typename ST, typename C, int U, int RG>
__global__ void __launch_bounds__(32 * NZ_WARPS)
k_near_warp(const NearTile *__restrict__ tiles, int ntiles, const ST *__restrict__ data, const C *__restrict__ x,
            long long ld, const int *__restrict__ cube_off, C *__restrict__ part, long long part_len,
            const int *skip, int nrhs, int row_cap) {
    extern __shared__ __align__(16) unsigned char nz_sh[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int t = blockIdx.x * NZ_WARPS + warp;
    if (t >= ntiles) return;
    ST *ring = (ST *)nz_sh + (size_t)warp * 2 * row_cap;       // two rows of this warp
    const NearTile tl = tiles[t];
    const int n1 = tl.n1, n2 = tl.n2;
    const int s1 = cube_off[tl.c1], s2 = cube_off[tl.c2];
    const ST *D = data + tl.data_off * 9;
    const bool offd = tl.col_off >= 0;
    const int nel = 9 * n2;
    for (int r0 = 0; r0 < nrhs; r0 += RG) {
        bool act[RG];
        C y[RG][U][3], ca[RG][U][3];
#pragma unroll
        for (int rr = 0; rr < RG; ++rr) {
            const int r = r0 + rr;
            act[rr] = r < nrhs && !(skip && skip[r]);
            const C *x2 = x + r * ld + 3LL * s2;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = lane + 32 * u;
                ca[rr][u][0] = ca[rr][u][1] = ca[rr][u][2] = czero<C>();
                y[rr][u][0] = y[rr][u][1] = y[rr][u][2] = czero<C>();
                if (act[rr] && j < n2) { y[rr][u][0] = x2[3 * j]; y[rr][u][1] = x2[3 * j + 1]; y[rr][u][2] = x2[3 * j + 2]; }
            }
        }
        __syncwarp();
        copy_row_async(ring, D, nel, lane);
        for (int i = 0; i < n1; ++i) {
            ST *cur = ring + (size_t)(i & 1) * row_cap;
            if (i + 1 < n1) {
                copy_row_async(ring + (size_t)((i + 1) & 1) * row_cap, D + (size_t)(i + 1) * nel, nel, lane);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncwarp();
            C m[U][9];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int j = lane + 32 * u;
#pragma unroll
                for (int q = 0; q < 9; ++q) m[u][q] = (j < n2) ? as_c<C>(cur[9 * j + q]) : czero<C>();
            }
            __syncwarp();      // the ring slot may be refilled after this
#pragma unroll
            for (int rr = 0; rr < RG; ++rr) {
                if (!act[rr]) continue;           // uniform across the warp
                const C *x1 = x + (r0 + rr) * ld + 3LL * s1;
                const C xa0 = x1[3 * i], xa1 = x1[3 * i + 1], xa2 = x1[3 * i + 2];
                C t0 = czero<C>(), t1 = t0, t2 = t0;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    cfma(t0, m[u][0], y[rr][u][0]); cfma(t1, m[u][1], y[rr][u][0]); cfma(t2, m[u][2], y[rr][u][0]);
                    cfma(t0, m[u][3], y[rr][u][1]); cfma(t1, m[u][4], y[rr][u][1]); cfma(t2, m[u][5], y[rr][u][1]);
                    cfma(t0, m[u][6], y[rr][u][2]); cfma(t1, m[u][7], y[rr][u][2]); cfma(t2, m[u][8], y[rr][u][2]);
                    if (offd) {
                        cfma(ca[rr][u][0], m[u][0], xa0); cfma(ca[rr][u][0], m[u][1], xa1); cfma(ca[rr][u][0], m[u][2], xa2);
                        cfma(ca[rr][u][1], m[u][3], xa0); cfma(ca[rr][u][1], m[u][4], xa1); cfma(ca[rr][u][1], m[u][5], xa2);
                        cfma(ca[rr][u][2], m[u][6], xa0); cfma(ca[rr][u][2], m[u][7], xa1); cfma(ca[rr][u][2], m[u][8], xa2);
                    }
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    t0.x += __shfl_xor_sync(0xffffffffu, t0.x, o);
                    t0.y += __shfl_xor_sync(0xffffffffu, t0.y, o);
                    t1.x += __shfl_xor_sync(0xffffffffu, t1.x, o);
                    t1.y += __shfl_xor_sync(0xffffffffu, t1.y, o);
                    t2.x += __shfl_xor_sync(0xffffffffu, t2.x, o);
                    t2.y += __shfl_xor_sync(0xffffffffu, t2.y, o);
                }
                C *pr = part + (r0 + rr) * part_len + tl.row_off + 3 * i;
                if (lane == 0) pr[0] = t0;
                else if (lane == 1) pr[1] = t1;
                else if (lane == 2) pr[2] = t2;
            }
        }
        if (offd) {
#pragma unroll
            for (int rr = 0; rr < RG; ++rr) {
                if (!act[rr]) continue;
                C *pc = part + (r0 + rr) * part_len + tl.col_off;
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int j = lane + 32 * u;
                    if (j < n2) {
                        pc[3 * j] = ca[rr][u][0];
                        pc[3 * j + 1] = ca[rr][u][1];
                        pc[3 * j + 2] = ca[rr][u][2];
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------- gather
// Interpolation (sparse_eps_matmul, src/sparse.f90:47-77) and final
// assembly (src/gmres_module.f90:148-170), one warp per cube, one lane per
// tet: the 27 box-node values of the four result grids are staged in shared
// memory for a group of right-hand sides, each lane forms its tet's six
// 27-term sums from the projector rows P[(g*27 + j)*T + slot] (coalesced
// across lanes), adds the cube's near-zone partial slots in slot order and
// writes Ax = near + (Y2 - k^2 Y).
template <typename C, int GA_RG>
__global__ void __launch_bounds__(32 * WARPS_PER_CTA)
k_gather(const C *__restrict__ Rg, const C *__restrict__ P, int T, const int *__restrict__ cube_off, GridDims G,
         typename CReal<C>::type k2, const C *__restrict__ part, long long part_len,
         const long long *__restrict__ pslot_base, const int *__restrict__ pslot_cnt, C *__restrict__ y, long long ld,
         const int *skip, int nrhs) {
    __shared__ C Rs[WARPS_PER_CTA][GA_RG][4][27];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * WARPS_PER_CTA + warp;
    if (c >= G.ncubes) return;
    const int s0 = cube_off[c], s1 = cube_off[c + 1];
    if (s0 == s1) return;
    const int nc = s1 - s0;
    const int bx = c % G.ncx, by = (c / G.ncx) % G.ncy, bz = c / (G.ncx * G.ncy);
    const long long NN = (long long)G.Nx * G.Ny * G.Nz;
    const long long pbase = pslot_base[c];
    const int nslot = pslot_cnt[c];
    long long node = 0;
    if (lane < 27) {
        const int a = lane % 3, b = (lane / 3) % 3, cc = lane / 9;
        node = ((long long)(2 * bz + cc) * G.Ny + (2 * by + b)) * G.Nx + (2 * bx + a);
    }
    for (int r0 = 0; r0 < nrhs; r0 += GA_RG) {
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
#pragma unroll
            for (int q = 0; q < GA_RG; ++q) {
                const int r = r0 + q;
                if (r >= nrhs || (skip && skip[r])) continue;
                const C *pr = part + r * part_len + pbase + 3 * sl;
                C *yr = y + r * ld + 3LL * s;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    C nz = czero<C>();
#pragma unroll 8
                    for (int t = 0; t < nslot; ++t) nz = cadd(nz, pr[(long long)t * 3 * nc + d]);
                    const C far = csub_scaled(acc[q][3 + d], k2, acc[q][d]);
                    yr[d] = cadd(nz, far);
                }
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
    static const cd *tw(scd_ctx *c, int a) { return c->d_tw[a]; }
    static cd *bpart(scd_ctx *c) { return c->d_bpart; }
    static cd *W(scd_ctx *c) { return c->d_W; }
    static cd *R(scd_ctx *c) { return c->d_R; }
    static cd *part(scd_ctx *c) { return c->d_nzpart; }
};
template <> struct Res<cf> {
    static const cf *P(scd_ctx *c) { return c->f_P; }
    static const cf *Fo(scd_ctx *c) { return c->f_Fo; }
    static const cf *tw(scd_ctx *c, int a) { return c->f_tw[a]; }
    static cf *bpart(scd_ctx *c) { return c->f_bpart; }
    static cf *W(scd_ctx *c) { return c->f_W; }
    static cf *R(scd_ctx *c) { return c->f_R; }
    static cf *part(scd_ctx *c) { return c->f_nzpart; }
};

template <int P, typename C>
void fft_x_fwd_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw) {
    using Cf = FftCfg<P>;
    dim3 grid((G.Ny * G.Nz + Cf::LPB - 1) / Cf::LPB, nrg);
    k_fft_x_fwd<P, C><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::bpart(c), Res<C>::W(c), tw, G, done);
}
template <int P, bool INV, typename C>
void fft_y_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw) {
    using Cf = FftCfg<P>;
    dim3 grid(((G.Px + Cf::LPB - 1) / Cf::LPB) * G.Nz, nrg);
    k_fft_y<P, INV, C><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), tw, G, done);
}
template <int P, typename C>
void fft_z_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw) {
    using Cf = FftCfg<P>;
    dim3 grid(((G.Px + Cf::LPB - 1) / Cf::LPB) * G.Py, nrg);
    k_fft_z<P, C><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), Res<C>::Fo(c), tw, G, done);
}
template <int P, typename C>
void fft_x_inv_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const C *tw) {
    using Cf = FftCfg<P>;
    dim3 grid((G.Ny * G.Nz + Cf::LPB - 1) / Cf::LPB, nrg);
    k_fft_x_inv<P, C><<<grid, Cf::THREADS, 0, c->st>>>(Res<C>::W(c), Res<C>::R(c), tw, G, done);
}

#define SCD_DISPATCH_P(PV, CALL)                     \
    switch (PV) {                                    \
        case 8: CALL(8); break;                      \
        case 16: CALL(16); break;                    \
        case 32: CALL(32); break;                    \
        case 64: CALL(64); break;                    \
        case 128: CALL(128); break;                  \
        case 256: CALL(256); break;                  \
        case 512: CALL(512); break;                  \
        default: break;                              \
    }

template <typename C>
void fft_chain_t(scd_ctx *c, const C *x, int nrhs, const int *done) {
    const GridDims G = dims_of(c);
    {
        dim3 grid((c->ncubes + WARPS_PER_CTA - 1) / WARPS_PER_CTA);
        const C *P = Res<C>::P(c);
        if (nrhs >= 8)
            k_scatter<C, 8><<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(x, c->n, P, c->T, c->d_cube_off, c->ncubes,
                                                                    Res<C>::bpart(c), done, nrhs);
        else if (nrhs >= 4)
            k_scatter<C, 4><<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(x, c->n, P, c->T, c->d_cube_off, c->ncubes,
                                                                    Res<C>::bpart(c), done, nrhs);
        else
            k_scatter<C, 1><<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(x, c->n, P, c->T, c->d_cube_off, c->ncubes,
                                                                    Res<C>::bpart(c), done, nrhs);
    }
    const int nrg = 4 * nrhs;
#define XF(PP) fft_x_fwd_t<PP, C>(c, G, nrg, done, Res<C>::tw(c, 0))
#define YF(PP) fft_y_t<PP, false, C>(c, G, nrg, done, Res<C>::tw(c, 1))
#define ZC(PP) fft_z_t<PP, C>(c, G, nrg, done, Res<C>::tw(c, 2))
#define YI(PP) fft_y_t<PP, true, C>(c, G, nrg, done, Res<C>::tw(c, 1))
#define XI(PP) fft_x_inv_t<PP, C>(c, G, nrg, done, Res<C>::tw(c, 0))
    SCD_DISPATCH_P(c->Px, XF)
    SCD_DISPATCH_P(c->Py, YF)
    SCD_DISPATCH_P(c->Pz, ZC)
    SCD_DISPATCH_P(c->Py, YI)
    SCD_DISPATCH_P(c->Px, XI)
#undef XF
#undef YF
#undef ZC
#undef YI
#undef XI
    c->launches += 6;
}

template <typename ST, typename C, int U>
void near_dispatch_u(scd_ctx *c, const ST *data, const C *x, int nrhs, const int *done) {
    const int row_cap = 9 * c->max_per_cube;
    const size_t sh = sizeof(ST) * 2 * (size_t)row_cap * NZ_WARPS;
    const int grid = (c->ntiles + NZ_WARPS - 1) / NZ_WARPS;
    C *part = Res<C>::part(c);
    if (nrhs >= 4) {
        cudaFuncSetAttribute(k_near_warp<ST, C, U, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
        k_near_warp<ST, C, U, 4><<<grid, 32 * NZ_WARPS, sh, c->st>>>(c->d_tiles, c->ntiles, data, x, c->n,
                                                                    c->d_cube_off, part, c->part_len, done, nrhs, row_cap);
    } else if (nrhs >= 2) {
        cudaFuncSetAttribute(k_near_warp<ST, C, U, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
        k_near_warp<ST, C, U, 2><<<grid, 32 * NZ_WARPS, sh, c->st>>>(c->d_tiles, c->ntiles, data, x, c->n,
                                                                    c->d_cube_off, part, c->part_len, done, nrhs, row_cap);
    } else {
        cudaFuncSetAttribute(k_near_warp<ST, C, U, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
        k_near_warp<ST, C, U, 1><<<grid, 32 * NZ_WARPS, sh, c->st>>>(c->d_tiles, c->ntiles, data, x, c->n,
                                                                    c->d_cube_off, part, c->part_len, done, nrhs, row_cap);
    }
}

template <typename C>
void near_t(scd_ctx *c, const C *x, int nrhs, const int *done) {
    if (c->ntiles == 0) return;
    const bool u1 = c->max_per_cube <= 32;
    if (c->near_prec == SCD_STORE_C64) {
        if (u1) near_dispatch_u<cf, C, 1>(c, (const cf *)c->d_tdata, x, nrhs, done);
        else near_dispatch_u<cf, C, 2>(c, (const cf *)c->d_tdata, x, nrhs, done);
    } else {
        if (u1) near_dispatch_u<cd, C, 1>(c, (const cd *)c->d_tdata, x, nrhs, done);
        else near_dispatch_u<cd, C, 2>(c, (const cd *)c->d_tdata, x, nrhs, done);
    }
    c->launches += 1;
}

template <typename C>
void gather_t(scd_ctx *c, C *y, int nrhs, const int *done) {
    const GridDims G = dims_of(c);
    dim3 grid((c->ncubes + WARPS_PER_CTA - 1) / WARPS_PER_CTA);
    typedef typename CReal<C>::type R;
    const R k2 = (R)(c->k * c->k);
    if (nrhs >= 4)
        k_gather<C, 4><<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(Res<C>::R(c), Res<C>::P(c), c->T, c->d_cube_off, G, k2,
                                                               Res<C>::part(c), c->part_len, c->d_pslot_base,
                                                               c->d_pslot_cnt, y, c->n, done, nrhs);
    else
        k_gather<C, 1><<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(Res<C>::R(c), Res<C>::P(c), c->T, c->d_cube_off, G, k2,
                                                               Res<C>::part(c), c->part_len, c->d_pslot_base,
                                                               c->d_pslot_cnt, y, c->n, done, nrhs);
    c->launches += 1;
}

template <typename C>
void run_matvec_t(scd_ctx *c, const C *x, C *y, int nrhs, const int *done) {
    if (c->timing) cudaEventRecord(c->ev[0], c->st);
    near_t<C>(c, x, nrhs, done);
    if (c->timing) cudaEventRecord(c->ev[1], c->st);
    fft_chain_t<C>(c, x, nrhs, done);
    if (c->timing) cudaEventRecord(c->ev[2], c->st);
    gather_t<C>(c, y, nrhs, done);
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
        (rc = al(&c->f_nzpart, r * (size_t)std::max<long long>(c->part_len, 1))))
        return rc;
    c->f_cap = nrhs;
    return SCD_OK;
}

void launch_permute_in(scd_ctx *c, const cd *x_orig, cd *x_slot, int nrhs, long long ld) {
    dim3 grid((unsigned)std::min<long long>((3LL * c->T + 255) / 256, 4096), nrhs);
    k_permute_in<<<grid, 256, 0, c->st>>>(x_orig, x_slot, c->d_perm, c->T, ld);
}

void launch_permute_out(scd_ctx *c, const cd *x_slot, cd *x_orig, int nrhs, long long ld) {
    dim3 grid((unsigned)std::min<long long>((3LL * c->T + 255) / 256, 4096), nrhs);
    k_permute_out<<<grid, 256, 0, c->st>>>(x_slot, x_orig, c->d_perm, c->T, ld);
}

void launch_fft_chain(scd_ctx *c, const cd *x, int nrhs, const int *done) { fft_chain_t<cd>(c, x, nrhs, done); }
void launch_near(scd_ctx *c, const cd *x, int nrhs, const int *done) { near_t<cd>(c, x, nrhs, done); }
void launch_gather(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done) {
    (void)x;
    gather_t<cd>(c, y, nrhs, done);
}
void run_matvec(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done) { run_matvec_t<cd>(c, x, y, nrhs, done); }
void run_matvec(scd_ctx *c, const cf *x, cf *y, int nrhs, const int *done) { run_matvec_t<cf>(c, x, y, nrhs, done); }
