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

SCD_HD cd  cmk(double r, double i) { return make_double2(r, i); }
SCD_HD cd  cadd(cd a, cd b) { return make_double2(a.x + b.x, a.y + b.y); }
SCD_HD cd  csub(cd a, cd b) { return make_double2(a.x - b.x, a.y - b.y); }
SCD_HD cd  cmul(cd a, cd b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
SCD_HD cd  cconj(cd a) { return make_double2(a.x, -a.y); }
SCD_HD cd  cscale(cd a, double s) { return make_double2(a.x * s, a.y * s); }
// a += b * c
SCD_HD void cfma(cd &a, cd b, cd c) { a.x += b.x * c.x - b.y * c.y; a.y += b.x * c.y + b.y * c.x; }
// a += conj(b) * c
SCD_HD void cfma_conj(cd &a, cd b, cd c) { a.x += b.x * c.x + b.y * c.y; a.y += b.x * c.y - b.y * c.x; }
SCD_HD double cabs2(cd a) { return a.x * a.x + a.y * a.y; }
SCD_HD cd cdiv(cd a, cd b) {
    double d = b.x * b.x + b.y * b.y;
    return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

SCD_HD cf  fmk(float r, float i) { return make_float2(r, i); }
SCD_HD cf  fadd(cf a, cf b) { return make_float2(a.x + b.x, a.y + b.y); }
SCD_HD cf  fsub(cf a, cf b) { return make_float2(a.x - b.x, a.y - b.y); }
SCD_HD cf  fmul(cf a, cf b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

// widen a stored near-zone value to FP64 (dcmplx(val) in src/sparse_mat.f90:113)
SCD_HD cd widen(cf a) { return make_double2((double)a.x, (double)a.y); }
SCD_HD cd widen(cd a) { return a; }

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
