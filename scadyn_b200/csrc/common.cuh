// Shared device helpers: complex arithmetic on double2/float2, a bounded
// grid barrier for cooperative launches, error plumbing.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef SCD_HD
#define SCD_HD __host__ __device__ __forceinline__
#endif

typedef double2 cd;     // complex double, (x, y) = (re, im)
typedef float2  cf;     // complex float

// Complex arithmetic with a pinned operation sequence: device code uses
// explicit round-to-nearest intrinsics so that the compiler cannot contract
// or reorder differently in different kernels (results of a column are
// bit-identical whichever kernel variant computes them).
#ifdef __CUDA_ARCH__
#define SCD_FMA(a, b, c) __fma_rn((a), (b), (c))
#define SCD_MUL(a, b) __dmul_rn((a), (b))
#define SCD_ADD(a, b) __dadd_rn((a), (b))
#define SCD_SUB(a, b) __dsub_rn((a), (b))
#else
#define SCD_FMA(a, b, c) fma((a), (b), (c))
#define SCD_MUL(a, b) ((a) * (b))
#define SCD_ADD(a, b) ((a) + (b))
#define SCD_SUB(a, b) ((a) - (b))
#endif

SCD_HD cd  cmk(double r, double i) { return make_double2(r, i); }
SCD_HD cd  cadd(cd a, cd b) { return make_double2(SCD_ADD(a.x, b.x), SCD_ADD(a.y, b.y)); }
SCD_HD cd  csub(cd a, cd b) { return make_double2(SCD_SUB(a.x, b.x), SCD_SUB(a.y, b.y)); }
SCD_HD cd  cmul(cd a, cd b) {
    return make_double2(SCD_FMA(a.x, b.x, SCD_MUL(-a.y, b.y)), SCD_FMA(a.x, b.y, SCD_MUL(a.y, b.x)));
}
SCD_HD cd  cconj(cd a) { return make_double2(a.x, -a.y); }
SCD_HD cd  cscale(cd a, double s) { return make_double2(SCD_MUL(a.x, s), SCD_MUL(a.y, s)); }
// a += b * c
SCD_HD void cfma(cd &a, cd b, cd c) {
    a.x = SCD_FMA(-b.y, c.y, SCD_FMA(b.x, c.x, a.x));
    a.y = SCD_FMA(b.y, c.x, SCD_FMA(b.x, c.y, a.y));
}
// a += conj(b) * c
SCD_HD void cfma_conj(cd &a, cd b, cd c) {
    a.x = SCD_FMA(b.y, c.y, SCD_FMA(b.x, c.x, a.x));
    a.y = SCD_FMA(-b.y, c.x, SCD_FMA(b.x, c.y, a.y));
}
SCD_HD double cabs2(cd a) { return SCD_FMA(a.x, a.x, SCD_MUL(a.y, a.y)); }
// w -= h * p
SCD_HD void csub_mul(cd &w, cd h, cd p) {
    w.x = SCD_FMA(h.y, p.y, SCD_FMA(-h.x, p.x, w.x));
    w.y = SCD_FMA(-h.y, p.x, SCD_FMA(-h.x, p.y, w.y));
}
// (re, im) += conj(z) * w
SCD_HD void cdot_acc(double &re, double &im, cd z, cd w) {
    re = SCD_FMA(z.y, w.y, SCD_FMA(z.x, w.x, re));
    im = SCD_FMA(-z.y, w.x, SCD_FMA(z.x, w.y, im));
}
// a - k2 * b
SCD_HD cd csub_scaled(cd a, double k2, cd b) { return make_double2(SCD_FMA(-k2, b.x, a.x), SCD_FMA(-k2, b.y, a.y)); }
SCD_HD cd cdiv(cd a, cd b) {
    double d = SCD_FMA(b.x, b.x, SCD_MUL(b.y, b.y));
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// complex float with pinned single-precision operations
#ifdef __CUDA_ARCH__
#define SCD_FMAF(a, b, c) __fmaf_rn((a), (b), (c))
#define SCD_MULF(a, b) __fmul_rn((a), (b))
#define SCD_ADDF(a, b) __fadd_rn((a), (b))
#define SCD_SUBF(a, b) __fsub_rn((a), (b))
#else
#define SCD_FMAF(a, b, c) fmaf((a), (b), (c))
#define SCD_MULF(a, b) ((a) * (b))
#define SCD_ADDF(a, b) ((a) + (b))
#define SCD_SUBF(a, b) ((a) - (b))
#endif
SCD_HD cf  fmk(float r, float i) { return make_float2(r, i); }
SCD_HD cf  cadd(cf a, cf b) { return make_float2(SCD_ADDF(a.x, b.x), SCD_ADDF(a.y, b.y)); }
SCD_HD cf  csub(cf a, cf b) { return make_float2(SCD_SUBF(a.x, b.x), SCD_SUBF(a.y, b.y)); }
SCD_HD cf  cmul(cf a, cf b) {
    return make_float2(SCD_FMAF(a.x, b.x, SCD_MULF(-a.y, b.y)), SCD_FMAF(a.x, b.y, SCD_MULF(a.y, b.x)));
}
SCD_HD cf  cconj(cf a) { return make_float2(a.x, -a.y); }
SCD_HD void cfma(cf &a, cf b, cf c) {
    a.x = SCD_FMAF(-b.y, c.y, SCD_FMAF(b.x, c.x, a.x));
    a.y = SCD_FMAF(b.y, c.x, SCD_FMAF(b.x, c.y, a.y));
}
SCD_HD cf csub_scaled(cf a, float k2, cf b) { return make_float2(SCD_FMAF(-k2, b.x, a.x), SCD_FMAF(-k2, b.y, a.y)); }
SCD_HD cf  fadd(cf a, cf b) { return cadd(a, b); }
SCD_HD cf  fsub(cf a, cf b) { return csub(a, b); }
SCD_HD cf  fmul(cf a, cf b) { return cmul(a, b); }

// zero / construction for either complex type
template <typename C> SCD_HD C czero();
template <> SCD_HD cd czero<cd>() { return make_double2(0.0, 0.0); }
template <> SCD_HD cf czero<cf>() { return make_float2(0.f, 0.f); }
template <typename C> struct CReal;
template <> struct CReal<cd> { typedef double type; };
template <> struct CReal<cf> { typedef float type; };
template <typename C> SCD_HD C cmake(double r, double i);
template <> SCD_HD cd cmake<cd>(double r, double i) { return make_double2(r, i); }
template <> SCD_HD cf cmake<cf>(double r, double i) { return make_float2((float)r, (float)i); }

// widen a stored near-zone value to FP64 (dcmplx(val) in src/sparse_mat.f90:113)
SCD_HD cd widen(cf a) { return make_double2((double)a.x, (double)a.y); }
SCD_HD cd widen(cd a) { return a; }
// stored value in the compute precision C
template <typename C> SCD_HD C as_c(cf a);
template <typename C> SCD_HD C as_c(cd a);
template <> SCD_HD cd as_c<cd>(cf a) { return make_double2((double)a.x, (double)a.y); }
template <> SCD_HD cd as_c<cd>(cd a) { return a; }
template <> SCD_HD cf as_c<cf>(cf a) { return a; }
template <> SCD_HD cf as_c<cf>(cd a) { return make_float2((float)a.x, (float)a.y); }

// Grid-wide barrier for kernels launched with cudaLaunchCooperativeKernel
// (all CTAs co-resident).  The spin is bounded: after `limit` polls the CTA
// records a timeout in *err and continues, so a broken launch ends with an
// error status instead of a hung GPU.
struct GridBarrier {
    unsigned int count;
    unsigned int gen;
};

__device__ __forceinline__ void grid_barrier(GridBarrier *b, unsigned int nblocks, int *err,
                                             long long limit = (1LL << 24)) {
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned int *vgen = &b->gen;
        unsigned int g = *vgen;
        __threadfence();
        unsigned int arrived = atomicAdd(&b->count, 1u);
        if (arrived == nblocks - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            long long it = 0;
            while (*vgen == g) {
                if (++it > limit) { atomicExch(err, 1); break; }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// block-wide sum of NV doubles; result valid in all threads.  `sh` needs
// NV * (blockDim.x / 32) doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sh) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
    }
    __syncthreads();
    if (lane == 0) {
#pragma unroll
        for (int q = 0; q < NV; ++q) sh[q * nw + w] = v[q];
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        double s = 0.0;
        for (int i = 0; i < nw; ++i) s += sh[q * nw + i];
        v[q] = s;
    }
    __syncthreads();
}

// ---- asynchronous copies into shared memory ----
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// element copy global -> shared (LDGSTS); src_bytes = 0 fills zeros
template <int BYTES>
__device__ __forceinline__ void cp_async_el(void *dst, const void *src, bool valid) {
    const int n = valid ? BYTES : 0;
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(smem_addr(dst)), "l"(src), "n"(BYTES), "r"(n)
                     : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// mbarrier + one-dimensional bulk copy (TMA engine, no tensor map): the
// copy's completion is counted on the barrier in bytes.
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}
// dst, src 16-byte aligned; bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for phase `parity` of *bar: after `limit` polls the thread
// records a timeout in *err and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err, long long limit = (1LL << 22)) {
    for (long long k = 0; k < limit; ++k) {
        if (mbar_try_wait(bar, parity)) return true;
        if (k > 16) __nanosleep(64);
    }
    atomicExch(err, 1);
    return false;
}
// The same wait, also ended (false, nothing recorded) as soon as another
// thread of the CTA raises *stop: once one wait of a pipeline has given up,
// the others stop waiting for copies that will not be issued.
__device__ __forceinline__ bool mbar_wait_or(uint64_t *bar, uint32_t parity, int *err, const volatile int *stop,
                                             long long limit = (1LL << 22)) {
    for (long long k = 0; k < limit; ++k) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*stop) return false;
        if (k > 16) __nanosleep(64);
    }
    atomicExch(err, 1);
    return false;
}
// arrive on *bar once every cp.async issued so far by this thread has landed
// (the barrier's expected count includes this arrival)
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// acc[a][u] += m[a] * x[u] for a 3 x U register tile.  Per accumulator the
// operation sequence equals cfma (re: fma(m.x, x.x) then fma(-m.y, x.y);
// im: fma(m.x, x.y) then fma(m.y, x.x)); the first halves of all products
// are issued before the second halves so that the dependent pairs are far
// apart in the instruction stream.
template <typename C, int U>
__device__ __forceinline__ void mac3(C (&acc)[3][U], const C (&m)[3], const C (&x)[U]) {
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if constexpr (sizeof(C) == 16) {
                acc[a][u].x = SCD_FMA(m[a].x, x[u].x, acc[a][u].x);
                acc[a][u].y = SCD_FMA(m[a].x, x[u].y, acc[a][u].y);
            } else {
                acc[a][u].x = SCD_FMAF(m[a].x, x[u].x, acc[a][u].x);
                acc[a][u].y = SCD_FMAF(m[a].x, x[u].y, acc[a][u].y);
            }
        }
#pragma unroll
    for (int a = 0; a < 3; ++a)
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if constexpr (sizeof(C) == 16) {
                acc[a][u].x = SCD_FMA(-m[a].y, x[u].y, acc[a][u].x);
                acc[a][u].y = SCD_FMA(m[a].y, x[u].x, acc[a][u].y);
            } else {
                acc[a][u].x = SCD_FMAF(-m[a].y, x[u].y, acc[a][u].x);
                acc[a][u].y = SCD_FMAF(m[a].y, x[u].x, acc[a][u].y);
            }
        }
}

// explicit shared-memory loads at 32-bit shared addresses (ld.shared)
__device__ __forceinline__ cf lds_c(uint32_t addr, cf) {
    cf v;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];\n" : "=f"(v.x), "=f"(v.y) : "r"(addr));
    return v;
}
__device__ __forceinline__ cd lds_c(uint32_t addr, cd) {
    cd v;
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];\n" : "=d"(v.x), "=d"(v.y) : "r"(addr));
    return v;
}
// two consecutive complex64 values (16-byte aligned address)
__device__ __forceinline__ void lds_c2(uint32_t addr, cf &a, cf &b) {
    asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];\n" : "=f"(a.x), "=f"(a.y), "=f"(b.x), "=f"(b.y) : "r"(addr));
}
