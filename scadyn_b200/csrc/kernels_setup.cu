// Per-wavelength set-up on the device that is not the hot loop: the Green's
// function spectrum (build_G, src/build_G.f90) and the T-matrix assembly
// T(:, c) = mat^H x_c (src/T_matrix.f90:260).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <vector>

#include "ctx.h"

namespace {

constexpr double PI = 3.141592653589793;   // src/common.f90:20

// The zero-padded Green's function of build_G is even in every axis
// (A(P-k) = A(k), src/build_G.f90:34-54), so its DFT is even as well and is
// fully described by the octant 0 <= j <= P/2.  The octant is computed as a
// separable DCT-I of the spatial octant: F(j) = sum_k w_k A(k) cos(2 pi jk/P),
// w_0 = w_{P/2} = 1, otherwise 2.
__global__ void k_green_spatial(cd *A, int Hx, int Hy, int Hz, int Nx, int Ny, int Nz, double delta,
                                double mx, double my, double mz, double k) {
    const long long tot = (long long)Hx * Hy * Hz;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % Hx), y = (int)((i / Hx) % Hy), z = (int)(i / ((long long)Hx * Hy));
        cd v = cmk(0, 0);
        if (x < Nx && y < Ny && z < Nz && (x | y | z)) {
            // R = norm(nodes(:,1), nodes(:,las)) with nodes = min + delta*(k-1)
            const double dx = mx - (mx + delta * (double)x);
            const double dy = my - (my + delta * (double)y);
            const double dz = mz - (mz + delta * (double)z);
            const double R = sqrt(dx * dx + dy * dy + dz * dz);
            if (R > 0.0) {
                const double d = 4 * PI * R;
                double s, c;
                sincos(k * R, &s, &c);
                v = cmk(c / d, s / d);
            }
        }
        A[i] = v;
    }
}

// one DCT-I pass along axis `ax` (0: x, 1: y, 2: z) of an Hx*Hy*Hz octant
__global__ void k_dct1_axis(const cd *in, cd *out, int Hx, int Hy, int Hz, int ax, int P, double scale) {
    const long long tot = (long long)Hx * Hy * Hz;
    const int H = ax == 0 ? Hx : (ax == 1 ? Hy : Hz);
    const long long st = ax == 0 ? 1 : (ax == 1 ? Hx : (long long)Hx * Hy);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % Hx), y = (int)((i / Hx) % Hy), z = (int)(i / ((long long)Hx * Hy));
        const int j = ax == 0 ? x : (ax == 1 ? y : z);
        const long long base = i - (long long)j * st;
        double re = 0, im = 0;
        for (int kk = 0; kk < H; ++kk) {
            const double w = (kk == 0 || kk == H - 1) ? 1.0 : 2.0;
            const long long m = ((long long)j * kk) % P;
            const double cs = cospi(2.0 * (double)m / (double)P) * w;
            const cd a = in[base + (long long)kk * st];
            re += cs * a.x;
            im += cs * a.y;
        }
        out[i] = cmk(re * scale, im * scale);
    }
}

// Tcols(r, c) = sum_i conj(mat(i, r)) X(i, c): 16x16 output tiles, split over
// K into `nsplit` partial sums that a second kernel adds in a fixed order.
constexpr int TB = 16;
__global__ void k_tgemm_partial(const cd *__restrict__ mat, long long n, int ncol, const cd *__restrict__ X,
                                int ncb, long long kchunk, cd *__restrict__ part) {
    __shared__ cd As[TB][TB + 1];
    __shared__ cd Bs[TB][TB + 1];
    const int tr = threadIdx.y, tc = threadIdx.x;
    const int r = blockIdx.y * TB + tr, cc = blockIdx.z * TB + tc;
    const long long k0 = (long long)blockIdx.x * kchunk, k1 = min(n, k0 + kchunk);
    cd acc = cmk(0, 0);
    for (long long kb = k0; kb < k1; kb += TB) {
        // As[kk][rr] = mat(kb+kk, row0+rr); Bs[kk][cc] = X(kb+kk, col0+cc)
        {
            const long long kk = kb + tc;
            const int rr = blockIdx.y * TB + tr;
            As[tc][tr] = (kk < k1 && rr < ncol) ? mat[(long long)rr * n + kk] : cmk(0, 0);
            const int c2 = blockIdx.z * TB + tr;
            Bs[tc][tr] = (kk < k1 && c2 < ncb) ? X[(long long)c2 * n + kk] : cmk(0, 0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < TB; ++kk) cfma_conj(acc, As[kk][tr], Bs[kk][tc]);
        __syncthreads();
    }
    if (r < ncol && cc < ncb) part[((long long)blockIdx.x * ncb + cc) * ncol + r] = acc;
}

__global__ void k_tgemm_reduce(const cd *part, int nsplit, int ncol, int ncb, cd *T, int col0) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ncol * ncb) return;
    cd s = cmk(0, 0);
    for (int p = 0; p < nsplit; ++p) s = cadd(s, part[(long long)p * ncol * ncb + i]);
    const int r = i % ncol, cc = i / ncol;
    T[(long long)(col0 + cc) * ncol + r] = s;
}

}  // namespace

int setup_green(scd_ctx *c, const scd_c128 *Fg) {
    NvtxRange range("Green octant");
    const long long oct = (long long)c->Hx * c->Hy * c->Hz;
    cd *tmp = nullptr;
    if (c->d_Fo) { cudaFree(c->d_Fo); c->d_Fo = nullptr; }
    if (cudaMalloc(&c->d_Fo, sizeof(cd) * oct) != cudaSuccess) return set_error(c, SCD_OOM, "Green octant");
    const double scale = 1.0 / ((double)c->Px * (double)c->Py * (double)c->Pz);
    if (Fg) {
        // host Fg(2Nx,2Ny,2Nz) == (Px,Py,Pz): keep the octant, fold in the
        // 1/(8 Nx Ny Nz) of arr2vec (src/common.f90:436)
        std::vector<cd> h((size_t)oct);
        for (int z = 0; z < c->Hz; ++z)
            for (int y = 0; y < c->Hy; ++y)
                for (int x = 0; x < c->Hx; ++x) {
                    const scd_c128 v = Fg[(size_t)x + (size_t)c->Px * ((size_t)y + (size_t)c->Py * z)];
                    h[(size_t)x + (size_t)c->Hx * ((size_t)y + (size_t)c->Hy * z)] = cmk(v.re * scale, v.im * scale);
                }
        return check_cuda(c, cudaMemcpyAsync(c->d_Fo, h.data(), sizeof(cd) * oct, cudaMemcpyHostToDevice, c->st), "Green octant");
    }
    if (cudaMalloc(&tmp, sizeof(cd) * oct) != cudaSuccess) return set_error(c, SCD_OOM, "Green scratch");
    const int blocks = (int)std::min<long long>((oct + 255) / 256, 65535);
    k_green_spatial<<<blocks, 256, 0, c->st>>>(c->d_Fo, c->Hx, c->Hy, c->Hz, c->Nx, c->Ny, c->Nz, c->d.delta,
                                               c->d.min_coord[0], c->d.min_coord[1], c->d.min_coord[2], c->k);
    k_dct1_axis<<<blocks, 256, 0, c->st>>>(c->d_Fo, tmp, c->Hx, c->Hy, c->Hz, 0, c->Px, 1.0);
    k_dct1_axis<<<blocks, 256, 0, c->st>>>(tmp, c->d_Fo, c->Hx, c->Hy, c->Hz, 1, c->Py, 1.0);
    k_dct1_axis<<<blocks, 256, 0, c->st>>>(c->d_Fo, tmp, c->Hx, c->Hy, c->Hz, 2, c->Pz, scale);
    int rc = check_cuda(c, cudaMemcpyAsync(c->d_Fo, tmp, sizeof(cd) * oct, cudaMemcpyDeviceToDevice, c->st), "Green");
    if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "Green");
    cudaFree(tmp);
    return rc;
}

void launch_T_assemble(scd_ctx *c, const cd *d_mat, int ncol, int col0, int ncb, const cd *d_X, cd *d_T) {
    const long long n = c->n;
    int nsplit = (int)std::min<long long>(64, std::max<long long>(1, n / 4096));
    const long long kchunk = ((n + nsplit - 1) / nsplit + TB - 1) / TB * TB;
    nsplit = (int)((n + kchunk - 1) / kchunk);
    cd *part = nullptr;
    cudaMallocAsync(&part, sizeof(cd) * (size_t)nsplit * ncol * ncb, c->st);
    dim3 grid(nsplit, (ncol + TB - 1) / TB, (ncb + TB - 1) / TB);
    k_tgemm_partial<<<grid, dim3(TB, TB), 0, c->st>>>(d_mat, n, ncol, d_X + (size_t)col0 * n, ncb, kchunk, part);
    k_tgemm_reduce<<<(ncol * ncb + 255) / 256, 256, 0, c->st>>>(part, nsplit, ncol, ncb, d_T, col0);
    cudaFreeAsync(part, c->st);
    c->launches += 2;
}


// ------------------------------------------------------------ no allocation
// scd_T_assemble_noalloc: the same split-K assembly T = mat^H X for callers
// that must not allocate device memory -- e.g. a Fortran host whose device
// arrays all come from its own allocator (CUDA Fortran `device` arrays,
// OpenACC data regions), where a cudaMalloc inside the library would hold
// memory outside that allocator's accounting and synchronise the device.
// The split-K partial sums live in this fixed file-scope array instead of a
// cudaMallocAsync buffer.
#define SCD_NOALLOC_SCRATCH (1 << 18)   // complex doubles: 4 MiB per device
static __device__ __align__(256) cd g_noalloc_scratch[SCD_NOALLOC_SCRATCH];

// device address of g_noalloc_scratch per device; the symbol name in host
// code is only a host-side stand-in, so the address is looked up once per
// device with that device current (first call on the device).  Atomic, as
// host threads may make their first calls at the same time; both store the
// same address.
static std::atomic<cd *> g_noalloc_ptr[128];

extern "C" SCD_API int scd_T_assemble_noalloc(const scd_c128 *mat, int64_t n, int32_t ncol, const scd_c128 *X,
                                              int32_t ncb, scd_c128 *T, void *stream) {
    if (!mat || !X || !T || n < 1 || ncol < 1 || ncb < 1) return SCD_BAD_ARG;
    if ((int64_t)ncol * ncb > SCD_NOALLOC_SCRATCH) return SCD_BAD_ARG;   // one split must fit the scratch
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return SCD_NO_DEVICE;
    // an error left pending by an earlier call of the caller's is not this
    // call's: report it without launching and leave it for the caller to read
    if (cudaPeekAtLastError() != cudaSuccess) return SCD_CUDA_ERROR;
    cd *part = g_noalloc_ptr[dev].load(std::memory_order_acquire);
    if (!part) {
        if (cudaGetSymbolAddress((void **)&part, g_noalloc_scratch) != cudaSuccess || !part) {
            cudaGetLastError();   // this lookup's own error
            return SCD_CUDA_ERROR;
        }
        g_noalloc_ptr[dev].store(part, std::memory_order_release);
    }
    cudaStream_t st = (cudaStream_t)stream;
    // as many K splits as the scratch holds (at most 64); every partial entry
    // is written before it is read, so nothing needs clearing between calls
    long long maxsplit = SCD_NOALLOC_SCRATCH / ((long long)ncol * ncb);
    int nsplit = (int)std::min<long long>(std::min<long long>(64, maxsplit), std::max<long long>(1, n / 4096));
    const long long kchunk = ((n + nsplit - 1) / nsplit + TB - 1) / TB * TB;
    nsplit = (int)((n + kchunk - 1) / kchunk);
    dim3 grid(nsplit, (ncol + TB - 1) / TB, (ncb + TB - 1) / TB);
    k_tgemm_partial<<<grid, dim3(TB, TB), 0, st>>>((const cd *)mat, n, ncol, (const cd *)X, ncb, kchunk, part);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();   // this launch's own error
        return SCD_CUDA_ERROR;
    }
    k_tgemm_reduce<<<(ncol * ncb + 255) / 256, 256, 0, st>>>(part, nsplit, ncol, ncb, (cd *)T, 0);
    if (cudaPeekAtLastError() != cudaSuccess) {
        cudaGetLastError();
        return SCD_CUDA_ERROR;
    }
    return SCD_OK;
}
