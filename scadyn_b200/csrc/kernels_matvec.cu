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
// tets.  bpart[((r*ncubes + c)*4 + g)*27 + j].
__global__ void k_scatter(const cd *__restrict__ x, long long ld, const cd *__restrict__ P, int T,
                          const int *__restrict__ cube_off, int ncubes, cd *__restrict__ bpart,
                          const int *done) {
    if (done && *done) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * WARPS_PER_CTA + warp;
    const int r = blockIdx.y;
    if (c >= ncubes) return;
    const cd *xr = x + r * ld;
    const long long TT = 27LL * T;
    cd a0 = cmk(0, 0), a1 = a0, a2 = a0, a3 = a0;
    if (lane < 27) {
        const int s0 = cube_off[c], s1 = cube_off[c + 1];
        for (int s = s0; s < s1; ++s) {
            const cd x0 = xr[3LL * s], x1 = xr[3LL * s + 1], x2 = xr[3LL * s + 2];
            const long long o = 27LL * s + lane;
            const cd p0 = P[o], px = P[TT + o], py = P[2 * TT + o], pz = P[3 * TT + o];
            cfma(a0, p0, x0);
            cfma(a1, p0, x1);
            cfma(a2, p0, x2);
            cfma(a3, px, x0);
            cfma(a3, py, x1);
            cfma(a3, pz, x2);
        }
        cd *o = bpart + ((long long)r * ncubes + c) * 4 * 27 + lane;
        o[0] = a0;
        o[27] = a1;
        o[54] = a2;
        o[81] = a3;
    }
}

// -------------------------------------------------------------------- FFT
// Radix-4 Stockham (with a final radix-2 stage for odd log2 P) on lines held
// in shared memory, FFTW sign convention (forward exp(-i)), unnormalised.
// TPL = P/4 threads cooperate on a line; all lines of a CTA advance together.
template <int P> struct Log2 { static constexpr int v = 1 + Log2<P / 2>::v; };
template <> struct Log2<1> { static constexpr int v = 0; };

template <bool INV>
__device__ __forceinline__ void radix4(cd &v0, cd &v1, cd &v2, cd &v3) {
    cd a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), a3 = csub(v1, v3);
    // forward: X1 = a1 - i a3 ; X3 = a1 + i a3
    cd ia3 = INV ? cmk(-a3.y, a3.x) : cmk(a3.y, -a3.x);   // (+i or -i) * a3
    v0 = cadd(a0, a2);
    v2 = csub(a0, a2);
    v1 = cadd(a1, ia3);
    v3 = csub(a1, ia3);
}

template <bool INV>
__device__ __forceinline__ cd twid(const cd *tw, int i) {
    cd w = tw[i];
    return INV ? cconj(w) : w;
}

template <int P, bool INV>
__device__ __forceinline__ void fft_line(cd *s, const cd *tw, int t) {
    constexpr int L = Log2<P>::v;
    constexpr int NB = P / 4;
    int Ns = 1;
#pragma unroll
    for (int st = 0; st < L / 2; ++st) {
        const int j = t;
        cd v0 = s[j], v1 = s[j + NB], v2 = s[j + 2 * NB], v3 = s[j + 3 * NB];
        const int kk = j & (Ns - 1);
        if (Ns > 1) {
            const int step = P / (Ns * 4);
            v1 = cmul(v1, twid<INV>(tw, kk * step));
            v2 = cmul(v2, twid<INV>(tw, 2 * kk * step));
            v3 = cmul(v3, twid<INV>(tw, 3 * kk * step));
        }
        radix4<INV>(v0, v1, v2, v3);
        __syncthreads();
        const int idx = (j / Ns) * Ns * 4 + kk;
        s[idx] = v0;
        s[idx + Ns] = v1;
        s[idx + 2 * Ns] = v2;
        s[idx + 3 * Ns] = v3;
        __syncthreads();
        Ns *= 4;
    }
    if (L & 1) {   // radix-2 stage, Ns = P/2: butterflies j = t, t + NB
        cd a[2], b[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = t + q * NB;
            a[q] = s[j];
            b[q] = cmul(s[j + P / 2], twid<INV>(tw, j));
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int j = t + q * NB;
            s[j] = cadd(a[q], b[q]);
            s[j + P / 2] = csub(a[q], b[q]);
        }
        __syncthreads();
    }
}

template <int P> struct FftCfg {
    static constexpr int TPL = P / 4;                        // threads per line
    static constexpr int LPB = (256 / TPL) > 0 ? 256 / TPL : 1;   // lines per CTA
    static constexpr int THREADS = TPL * LPB;
    static constexpr int LS = P + 1;                         // padded line stride (bank spread)
};

struct GridDims {
    int Nx, Ny, Nz, Px, Py, Pz, Hx, Hy, Hz, ncx, ncy, ncz, ncubes;
};

__device__ __forceinline__ int fold(int u, int P) { return u <= P - u ? u : P - u; }

// node value of grid g at node (x,y,z) from the box partial sums: every box
// whose 3x3x3 node block contains the node contributes its local sum
__device__ __forceinline__ cd node_value(const cd *__restrict__ bp, const GridDims &G, int g, int x, int y, int z) {
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
    cd v = cmk(0, 0);
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
template <int P>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_x_fwd(const cd *__restrict__ bpart, cd *__restrict__ W, const cd *__restrict__ twg, GridDims G, const int *done) {
    if (done && *done) return;
    using C = FftCfg<P>;
    __shared__ cd sh[C::LPB * C::LS];
    __shared__ cd tw[P];
    const int rg = blockIdx.y;                 // r*4 + g
    const int g = rg & 3, r = rg >> 2;
    const cd *bp = bpart + (long long)r * G.ncubes * 4 * 27;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int nlines = G.Ny * G.Nz;
    const int line0 = blockIdx.x * C::LPB;
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int l = e / P, x = e - l * P, line = line0 + l;
        cd v = cmk(0, 0);
        if (line < nlines && x < G.Nx) {
            const int y = line % G.Ny, z = line / G.Ny;
            v = node_value(bp, G, g, x, y, z);
        }
        sh[l * C::LS + x] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / C::TPL, t = threadIdx.x - l * C::TPL;
    fft_line<P, false>(sh + l * C::LS, tw, t);
    cd *Wr = W + (long long)rg * G.Px * G.Py * G.Nz;
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int ll = e / P, x = e - ll * P, line = line0 + ll;
        if (line < nlines) {
            const int y = line % G.Ny, z = line / G.Ny;
            Wr[((long long)z * G.Py + y) * G.Px + x] = sh[ll * C::LS + x];
        }
    }
}

// Y pass: lines (x < Px, z < Nz); forward reads y < Ny and writes y < Py,
// inverse reads y < Py and writes y < Ny.  A CTA takes LPB consecutive x.
template <int P, bool INV>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_y(cd *__restrict__ W, const cd *__restrict__ twg, GridDims G, const int *done) {
    if (done && *done) return;
    using C = FftCfg<P>;
    __shared__ cd sh[C::LPB * C::LS];
    __shared__ cd tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int xblocks = (G.Px + C::LPB - 1) / C::LPB;
    const int z = blockIdx.x / xblocks, x0 = (blockIdx.x - z * xblocks) * C::LPB;
    cd *Wr = W + (long long)rg * G.Px * G.Py * G.Nz + (long long)z * G.Py * G.Px;
    const int nin = INV ? G.Py : G.Ny, nout = INV ? G.Ny : G.Py;
    // sh layout [line][y]
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int y = e / C::LPB, l = e - y * C::LPB, x = x0 + l;
        cd v = cmk(0, 0);
        if (y < nin && x < G.Px) v = Wr[(long long)y * G.Px + x];
        sh[l * C::LS + y] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / C::TPL, t = threadIdx.x - l * C::TPL;
    fft_line<P, INV>(sh + l * C::LS, tw, t);
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int y = e / C::LPB, ll = e - y * C::LPB, x = x0 + ll;
        if (y < nout && x < G.Px) Wr[(long long)y * G.Px + x] = sh[ll * C::LS + y];
    }
}

// Z pass: lines (x < Px, y < Py), forward FFT of z < Nz (zero padded), times
// the Green octant Fo (folded by evenness), inverse FFT, keep z < Nz.
template <int P>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_z(cd *__restrict__ W, const cd *__restrict__ Fo, const cd *__restrict__ twg, GridDims G, const int *done) {
    if (done && *done) return;
    using C = FftCfg<P>;
    __shared__ cd sh[C::LPB * C::LS];
    __shared__ cd tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int xblocks = (G.Px + C::LPB - 1) / C::LPB;
    const int y = blockIdx.x / xblocks, x0 = (blockIdx.x - y * xblocks) * C::LPB;
    const long long plane = (long long)G.Px * G.Py;
    cd *Wr = W + (long long)rg * plane * G.Nz + (long long)y * G.Px;
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int z = e / C::LPB, l = e - z * C::LPB, x = x0 + l;
        cd v = cmk(0, 0);
        if (z < G.Nz && x < G.Px) v = Wr[(long long)z * plane + x];
        sh[l * C::LS + z] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / C::TPL, t = threadIdx.x - l * C::TPL;
    fft_line<P, false>(sh + l * C::LS, tw, t);
    const int fy = fold(y, G.Py);
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int ll = e / P, z = e - ll * P, x = x0 + ll;
        if (x < G.Px) {
            const cd f = Fo[((long long)fold(z, G.Pz) * G.Hy + fy) * G.Hx + fold(x, G.Px)];
            sh[ll * C::LS + z] = cmul(f, sh[ll * C::LS + z]);
        }
    }
    __syncthreads();
    fft_line<P, true>(sh + l * C::LS, tw, t);
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int z = e / C::LPB, ll = e - z * C::LPB, x = x0 + ll;
        if (z < G.Nz && x < G.Px) Wr[(long long)z * plane + x] = sh[ll * C::LS + z];
    }
}

// X inverse: lines (y < Ny, z < Nz), keep x < Nx, write the result grid
// R[(rg)][(z*Ny + y)*Nx + x]
template <int P>
__global__ void __launch_bounds__(FftCfg<P>::THREADS)
k_fft_x_inv(const cd *__restrict__ W, cd *__restrict__ R, const cd *__restrict__ twg, GridDims G, const int *done) {
    if (done && *done) return;
    using C = FftCfg<P>;
    __shared__ cd sh[C::LPB * C::LS];
    __shared__ cd tw[P];
    const int rg = blockIdx.y;
    for (int i = threadIdx.x; i < P; i += blockDim.x) tw[i] = twg[i];
    const int nlines = G.Ny * G.Nz;
    const int line0 = blockIdx.x * C::LPB;
    const cd *Wr = W + (long long)rg * G.Px * G.Py * G.Nz;
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int l = e / P, x = e - l * P, line = line0 + l;
        cd v = cmk(0, 0);
        if (line < nlines) {
            const int y = line % G.Ny, z = line / G.Ny;
            v = Wr[((long long)z * G.Py + y) * G.Px + x];
        }
        sh[l * C::LS + x] = v;
    }
    __syncthreads();
    const int l = threadIdx.x / C::TPL, t = threadIdx.x - l * C::TPL;
    fft_line<P, true>(sh + l * C::LS, tw, t);
    cd *Rr = R + (long long)rg * G.Nx * G.Ny * G.Nz;
    for (int e = threadIdx.x; e < C::LPB * P; e += blockDim.x) {
        const int ll = e / P, x = e - ll * P, line = line0 + ll;
        if (line < nlines && x < G.Nx) {
            const int y = line % G.Ny, z = line / G.Ny;
            Rr[((long long)z * G.Ny + y) * G.Nx + x] = sh[ll * C::LS + x];
        }
    }
}

// ------------------------------------------------------------ near zone
// One CTA per tile: row sums y(c1) += M x(c2) and, for off-diagonal tiles,
// column sums y(c2) += M^T x(c1) (transpose, not conjugate: the operator is
// complex symmetric, src/sparse_mat.f90:113-116).  Results go to per-cube
// partial slots; k_gather adds them in a fixed order (deterministic).
template <typename ST>
__global__ void __launch_bounds__(128)
k_near_tiles(const NearTile *__restrict__ tiles, const ST *__restrict__ data, const cd *__restrict__ x,
             long long ld, const int *__restrict__ cube_off, cd *__restrict__ part, long long part_len,
             const int *done) {
    if (done && *done) return;
    extern __shared__ cd xs_sh[];
    const NearTile tl = tiles[blockIdx.x];
    const int r = blockIdx.y;
    const cd *xr = x + r * ld;
    cd *pr = part + r * part_len;
    const int s1 = cube_off[tl.c1], s2 = cube_off[tl.c2];
    cd *x1 = xs_sh, *x2 = xs_sh + 3 * tl.n1;
    for (int i = threadIdx.x; i < 3 * tl.n1; i += blockDim.x) x1[i] = xr[3LL * s1 + i];
    for (int i = threadIdx.x; i < 3 * tl.n2; i += blockDim.x) x2[i] = xr[3LL * s2 + i];
    __syncthreads();
    const ST *D = data + tl.data_off * 9;
    for (int row = threadIdx.x; row < 3 * tl.n1; row += blockDim.x) {
        const int i = row / 3, a = row - 3 * i;
        cd acc = cmk(0, 0);
        const ST *Bi = D + (long long)i * tl.n2 * 9 + a;
        for (int j = 0; j < tl.n2; ++j) {
            const ST *b = Bi + 9 * j;
            cfma(acc, widen(b[0]), x2[3 * j]);
            cfma(acc, widen(b[3]), x2[3 * j + 1]);
            cfma(acc, widen(b[6]), x2[3 * j + 2]);
        }
        pr[tl.row_off + row] = acc;
    }
    if (tl.col_off >= 0) {
        for (int col = threadIdx.x; col < 3 * tl.n2; col += blockDim.x) {
            const int j = col / 3, b = col - 3 * j;
            cd acc = cmk(0, 0);
            const ST *Bj = D + (long long)j * 9 + 3 * b;
            for (int i = 0; i < tl.n1; ++i) {
                const ST *q = Bj + (long long)i * tl.n2 * 9;
                cfma(acc, widen(q[0]), x1[3 * i]);
                cfma(acc, widen(q[1]), x1[3 * i + 1]);
                cfma(acc, widen(q[2]), x1[3 * i + 2]);
            }
            pr[tl.col_off + col] = acc;
        }
    }
}

// ---------------------------------------------------------------- gather
// Interpolation (sparse_eps_matmul, src/sparse.f90:47-77) and final
// assembly (src/gmres_module.f90:148-170), one warp per cube: lane j < 27
// holds the four result-grid values at node j of the cube's box; per tet the
// six 27-term dot products are reduced across the warp.  The near-zone
// partial slots of the cube are added in slot order.
__global__ void k_gather(const cd *__restrict__ Rg, const cd *__restrict__ P, int T,
                         const int *__restrict__ cube_off, GridDims G, double k2,
                         const cd *__restrict__ part, long long part_len,
                         const long long *__restrict__ pslot_base, const int *__restrict__ pslot_cnt,
                         cd *__restrict__ y, long long ld, const int *done) {
    if (done && *done) return;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * WARPS_PER_CTA + warp;
    const int r = blockIdx.y;
    if (c >= G.ncubes) return;
    const int s0 = cube_off[c], s1 = cube_off[c + 1];
    if (s0 == s1) return;
    const int bx = c % G.ncx, by = (c / G.ncx) % G.ncy, bz = c / (G.ncx * G.ncy);
    const long long NN = (long long)G.Nx * G.Ny * G.Nz;
    const cd *Rr = Rg + (long long)r * 4 * NN;
    cd R0 = cmk(0, 0), R1 = R0, R2 = R0, R3 = R0;
    if (lane < 27) {
        const int a = lane % 3, b = (lane / 3) % 3, cc = lane / 9;
        const long long node = ((long long)(2 * bz + cc) * G.Ny + (2 * by + b)) * G.Nx + (2 * bx + a);
        R0 = Rr[node];
        R1 = Rr[NN + node];
        R2 = Rr[2 * NN + node];
        R3 = Rr[3 * NN + node];
    }
    const long long TT = 27LL * T;
    const int nc = s1 - s0;
    const cd *pr = part + r * part_len + pslot_base[c];
    const int nslot = pslot_cnt[c];
    cd *yr = y + r * ld;
    for (int s = s0; s < s1; ++s) {
        double v[12];
        if (lane < 27) {
            const long long o = 27LL * s + lane;
            const cd p0 = P[o], px = P[TT + o], py = P[2 * TT + o], pz = P[3 * TT + o];
            const cd t0 = cmul(p0, R0), t1 = cmul(p0, R1), t2 = cmul(p0, R2);
            const cd u0 = cmul(px, R3), u1 = cmul(py, R3), u2 = cmul(pz, R3);
            v[0] = t0.x; v[1] = t0.y; v[2] = t1.x; v[3] = t1.y; v[4] = t2.x; v[5] = t2.y;
            v[6] = u0.x; v[7] = u0.y; v[8] = u1.x; v[9] = u1.y; v[10] = u2.x; v[11] = u2.y;
        } else {
#pragma unroll
            for (int q = 0; q < 12; ++q) v[q] = 0.0;
        }
#pragma unroll
        for (int q = 0; q < 12; ++q) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
        }
        if (lane < 3) {
            const int d = lane;
            cd far = cmk(v[6 + 2 * d] - k2 * v[2 * d], v[7 + 2 * d] - k2 * v[2 * d + 1]);
            cd nz = cmk(0, 0);
            const int li = 3 * (s - s0) + d;
            for (int q = 0; q < nslot; ++q) nz = cadd(nz, pr[(long long)q * 3 * nc + li]);
            yr[3LL * s + d] = cadd(nz, far);
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

GridDims dims_of(const scd_ctx *c) {
    GridDims G;
    G.Nx = c->Nx; G.Ny = c->Ny; G.Nz = c->Nz;
    G.Px = c->Px; G.Py = c->Py; G.Pz = c->Pz;
    G.Hx = c->Hx; G.Hy = c->Hy; G.Hz = c->Hz;
    G.ncx = c->ncx; G.ncy = c->ncy; G.ncz = c->ncz; G.ncubes = c->ncubes;
    return G;
}

}  // namespace

// twiddle table exp(-2 pi i j / P), j < P
int build_twiddles(scd_ctx *c, int P, cd **out) {
    cudaError_t e = cudaMalloc(out, sizeof(cd) * P);
    if (e != cudaSuccess) return check_cuda(c, e, "twiddles");
    k_twiddles<<<(P + 255) / 256, 256, 0, c->st>>>(*out, P);
    return check_cuda(c, cudaGetLastError(), "twiddles");
}

namespace {

template <int P>
void fft_x_fwd_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const cd *tw) {
    using C = FftCfg<P>;
    dim3 grid((G.Ny * G.Nz + C::LPB - 1) / C::LPB, nrg);
    k_fft_x_fwd<P><<<grid, C::THREADS, 0, c->st>>>(c->d_bpart, c->d_W, tw, G, done);
}
template <int P, bool INV>
void fft_y_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const cd *tw) {
    using C = FftCfg<P>;
    dim3 grid(((G.Px + C::LPB - 1) / C::LPB) * G.Nz, nrg);
    k_fft_y<P, INV><<<grid, C::THREADS, 0, c->st>>>(c->d_W, tw, G, done);
}
template <int P>
void fft_z_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const cd *tw) {
    using C = FftCfg<P>;
    dim3 grid(((G.Px + C::LPB - 1) / C::LPB) * G.Py, nrg);
    k_fft_z<P><<<grid, C::THREADS, 0, c->st>>>(c->d_W, c->d_Fo, tw, G, done);
}
template <int P>
void fft_x_inv_t(scd_ctx *c, const GridDims &G, int nrg, const int *done, const cd *tw) {
    using C = FftCfg<P>;
    dim3 grid((G.Ny * G.Nz + C::LPB - 1) / C::LPB, nrg);
    k_fft_x_inv<P><<<grid, C::THREADS, 0, c->st>>>(c->d_W, c->d_R, tw, G, done);
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

}  // namespace

void launch_permute_in(scd_ctx *c, const cd *x_orig, cd *x_slot, int nrhs, long long ld) {
    dim3 grid((unsigned)std::min<long long>((3LL * c->T + 255) / 256, 4096), nrhs);
    k_permute_in<<<grid, 256, 0, c->st>>>(x_orig, x_slot, c->d_perm, c->T, ld);
}

void launch_permute_out(scd_ctx *c, const cd *x_slot, cd *x_orig, int nrhs, long long ld) {
    dim3 grid((unsigned)std::min<long long>((3LL * c->T + 255) / 256, 4096), nrhs);
    k_permute_out<<<grid, 256, 0, c->st>>>(x_slot, x_orig, c->d_perm, c->T, ld);
}

void launch_fft_chain(scd_ctx *c, const cd *x, int nrhs, const int *done) {
    const GridDims G = dims_of(c);
    {
        dim3 grid((c->ncubes + WARPS_PER_CTA - 1) / WARPS_PER_CTA, nrhs);
        k_scatter<<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(x, c->n, c->d_P, c->T, c->d_cube_off, c->ncubes,
                                                          c->d_bpart, done);
    }
    const int nrg = 4 * nrhs;
#define XF(P) fft_x_fwd_t<P>(c, G, nrg, done, c->d_tw[0])
#define YF(P) fft_y_t<P, false>(c, G, nrg, done, c->d_tw[1])
#define ZC(P) fft_z_t<P>(c, G, nrg, done, c->d_tw[2])
#define YI(P) fft_y_t<P, true>(c, G, nrg, done, c->d_tw[1])
#define XI(P) fft_x_inv_t<P>(c, G, nrg, done, c->d_tw[0])
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

void launch_near(scd_ctx *c, const cd *x, int nrhs, const int *done) {
    if (c->ntiles == 0) return;
    dim3 grid(c->ntiles, nrhs);
    size_t sh = sizeof(cd) * 6 * (size_t)c->max_per_cube;
    if (c->near_prec == SCD_STORE_C64)
        k_near_tiles<cf><<<grid, 128, sh, c->st>>>(c->d_tiles, (const cf *)c->d_tdata, x, c->n, c->d_cube_off,
                                                   c->d_nzpart, c->part_len, done);
    else
        k_near_tiles<cd><<<grid, 128, sh, c->st>>>(c->d_tiles, (const cd *)c->d_tdata, x, c->n, c->d_cube_off,
                                                   c->d_nzpart, c->part_len, done);
    c->launches += 1;
}

void launch_gather(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done) {
    (void)x;
    const GridDims G = dims_of(c);
    dim3 grid((c->ncubes + WARPS_PER_CTA - 1) / WARPS_PER_CTA, nrhs);
    k_gather<<<grid, 32 * WARPS_PER_CTA, 0, c->st>>>(c->d_R, c->d_P, c->T, c->d_cube_off, G, c->k * c->k,
                                                     c->d_nzpart, c->part_len, c->d_pslot_base, c->d_pslot_cnt,
                                                     y, c->n, done);
    c->launches += 1;
}

void run_matvec(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done) {
    if (c->timing) cudaEventRecord(c->ev[0], c->st);
    launch_near(c, x, nrhs, done);
    if (c->timing) cudaEventRecord(c->ev[1], c->st);
    launch_fft_chain(c, x, nrhs, done);
    if (c->timing) cudaEventRecord(c->ev[2], c->st);
    launch_gather(c, x, y, nrhs, done);
    if (c->timing) cudaEventRecord(c->ev[3], c->st);
}
