// Self-test of the bounded device waits: each wait in the library (grid
// barrier of the cooperative kernels, mbarrier phases of the near-zone
// pipeline) gives up after an iteration limit, records an error and returns,
// so a launch that cannot complete ends with a status instead of a hung GPU.
// scd_selftest_waits runs both waits against conditions nothing satisfies,
// with short limits, and reports what the host reads back.
#include <cuda_runtime.h>

#include "ctx.h"

namespace {

__global__ void k_wait_test(GridBarrier *bar, int *err_bar, int *err_mbar, long long limit) {
    // a grid barrier for one block more than the grid has: never completes
    grid_barrier(bar, gridDim.x + 1, err_bar, limit);
    // an mbarrier phase that nothing arrives on
    __shared__ uint64_t mb;
    if (threadIdx.x == 0) {
        mbar_init(&mb, 1);
        mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait(&mb, 0u, err_mbar, limit);
    __syncthreads();
}

}  // namespace

extern "C" int scd_selftest_waits(int32_t device) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return SCD_NO_DEVICE; }
    if (device < 0 || device >= ndev) return SCD_BAD_ARG;
    cudaSetDevice(device);
    GridBarrier *bar = nullptr;
    int *err = nullptr;
    if (cudaMalloc(&bar, sizeof(GridBarrier)) != cudaSuccess) { cudaGetLastError(); return SCD_OOM; }
    if (cudaMalloc(&err, 2 * sizeof(int)) != cudaSuccess) { cudaGetLastError(); cudaFree(bar); return SCD_OOM; }
    cudaMemset(bar, 0, sizeof(GridBarrier));
    cudaMemset(err, 0, 2 * sizeof(int));
    k_wait_test<<<2, 32>>>(bar, err, err + 1, 4096);
    int h[2] = {0, 0};
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpy(h, err, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(bar);
    cudaFree(err);
    if (e != cudaSuccess) return SCD_CUDA_ERROR;
    return (h[0] && h[1]) ? SCD_TIMEOUT : SCD_CUDA_ERROR;
}
