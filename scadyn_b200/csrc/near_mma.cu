// Near-zone tile products of the mixed-precision (complex64) matvec on the
// tensor cores: tcgen05.mma kind::f16 with FP32 accumulators in tensor
// memory, tiles stored as f16 hi/lo planes (layouts and instruction schedule
// in near_mma.cuh).  The sums are those of k_near_groups
// (matmul_Acorr_const, src/sparse_mat.f90:96-123, complex-symmetric: the
// transpose, not the conjugate): per group g the row sums over its tiles go
// to partial slot 0, and each tile (g, g2), g2 != g, writes A^T x(g) to its
// partial slot of g2; k_gather adds the slots in a fixed order.
//
// The default near zone of the complex64 matvec when the blocks are stored
// complex64 (scd_grid_desc.near_kernel: SCD_NEAR_TENSOR_MERGED, 16 right-hand
// sides per pass; SCD_NEAR_TENSOR_WIDE, the same schedule over 32;
// SCD_NEAR_TENSOR_SPLIT for the split instruction schedule; SCD_NEAR_CUDA_CORES
// selects k_near_groups instead).
#include <cuda_fp16.h>

#include <cmath>

#include "ctx.h"
#include "near_mma.cuh"

namespace {

constexpr int NZM_SLOTS = 8;
constexpr int NZM_THREADS = 192;          // warp 0 producer, warp 1 MMA issuer, warps 2-5 epilogue
constexpr uint32_t NZM_META = 256;
// two CTAs per SM (schedules 0, 1): 2 x (dynamic + static + 1 KB reserved per
// CTA) must stay within the SM's 228 KB; 113 KB dynamic plus the kernel's
// static bytes no longer did, and halved the resident CTAs
constexpr size_t NZM_SMEM = 112 * 1024;
constexpr size_t NZM_SMEM_WIDE = NzmSched<2>::CTAS == 2 ? NZM_SMEM : 224 * 1024;   // schedule 2

struct NzmArgs {
    const NearTile *tiles;
    const int *grp_tile, *grp_off;
    const long long *pslot_base;
    const unsigned char *t16;
    const long long *t16_off;
    const unsigned char *xb;
    const long long *xb_off;
    cf *part;
    long long part_len;
    const int *skip;
    int r0, rg;
    const float *xinv;          // per right-hand side of the pass: 1 / (sA sx)
    uint32_t x1_bytes, ring_bytes, slack_bytes;
    int *err;
};

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t da, uint64_t db, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred q;\n setp.ne.b32 q, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, q;\n}\n" ::"r"(d),
        "l"(da), "l"(db), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
        : "memory");
}
// arrive on *bar when every tcgen05.mma issued so far by this thread has completed
__device__ __forceinline__ void tc_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
          "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// issue every instruction of one product (use 0: row, 1: transposed)
template <int S>
__device__ __forceinline__ void issue_product(int use, int n1, int n2, uint32_t tile, uint32_t xblk, uint32_t dcol,
                                              bool overwrite) {
    const int ks = nzm_ksteps(use, n1, n2);
    if constexpr (S == 0) {
        for (int kk = 0; kk < ks; ++kk)
#pragma unroll
            for (int s = 0; s < NZM_SPLITS; ++s)
#pragma unroll
                for (int q = 0; q < NZM_OPS; ++q) {
                    const NzmOp o = nzm_op(use, n1, n2, kk, s, q);
                    const uint64_t da = nzm_sdesc(tile + o.a_off, o.a_lbo, o.a_sbo);
                    const uint64_t db = nzm_sdesc(xblk + o.b_off, o.b_lbo, o.b_sbo);
                    tc_mma(dcol + (uint32_t)o.d_col, da, db, nzm_idesc(o), (overwrite && o.first) ? 0u : 1u);
                }
    } else {
        // descriptors of K step 0, then constant start-address steps (the
        // 14-bit address field cannot carry: shared addresses stay below 2^18)
        constexpr int NOP = NzmSched<S>::PARTS * NZM_OPS;
        uint64_t da[NOP], db[NOP];
        uint32_t id[NOP], dc[NOP];
#pragma unroll
        for (int j = 0; j < NOP; ++j) {
            const NzmOp o = nzm_op_s<S>(use, n1, n2, 0, j / NZM_OPS, j % NZM_OPS);
            da[j] = nzm_sdesc(tile + o.a_off, o.a_lbo, o.a_sbo);
            db[j] = nzm_sdesc(xblk + o.b_off, o.b_lbo, o.b_sbo);
            id[j] = nzm_idesc(o);
            dc[j] = dcol + (uint32_t)o.d_col;
        }
        const uint64_t sa = nzm_a_step(use, n2) >> 4, sb = NZM_B_STEP >> 4;
        for (int kk = 0; kk < ks; ++kk)
#pragma unroll
            for (int j = 0; j < NOP; ++j)
                tc_mma(dc[j], da[j] + (uint64_t)kk * sa, db[j] + (uint64_t)kk * sb, id[j],
                       (overwrite && kk == 0 && j == 0) ? 0u : 1u);
    }
}

// a lane's accumulator row of a product as the complex y_r of the pass's R
// right-hand sides (all lanes of the warp take part).  Schedule 0 holds
// [Re y | Im y]; schedules 1 and 2 hold [Re (x hi) | Re (x lo) | Im (x hi) |
// Im (x lo)], each R columns, added pairwise (hi part first).
template <int S> struct NzmRows { float re[NzmSched<S>::R], im[NzmSched<S>::R]; };

template <int S>
__device__ __forceinline__ void load_rows(uint32_t taddr, NzmRows<S> &y) {
    constexpr int R = NzmSched<S>::R;
    float a[32], b[32];
    if constexpr (S == 0) {
        tc_ld32(taddr, a);
#pragma unroll
        for (int r = 0; r < R; ++r) { y.re[r] = a[r]; y.im[r] = a[R + r]; }
    } else if constexpr (R == 16) {
        tc_ld32(taddr, a);
        tc_ld32(taddr + 32, b);
#pragma unroll
        for (int r = 0; r < R; ++r) { y.re[r] = a[r] + a[R + r]; y.im[r] = b[r] + b[R + r]; }
    } else {
        tc_ld32(taddr, a);
        tc_ld32(taddr + R, b);
#pragma unroll
        for (int r = 0; r < R; ++r) y.re[r] = a[r] + b[r];
        tc_ld32(taddr + 2 * R, a);
        tc_ld32(taddr + 3 * R, b);
#pragma unroll
        for (int r = 0; r < R; ++r) y.im[r] = a[r] + b[r];
    }
}

// that row scaled by xinv (sc, in shared memory), written to
// part[(r0 + r) * part_len + base + row] for the right-hand sides whose bit
// is set in `on` (present and not finished)
template <int S>
__device__ __forceinline__ void store_rows(const NzmArgs &a, const NzmRows<S> &y, int row_ok, int row, long long base,
                                           const float *sc, unsigned on) {
    if (!row_ok) return;
#pragma unroll
    for (int r = 0; r < NzmSched<S>::R; ++r) {
        if (!((on >> r) & 1u)) continue;
        a.part[(long long)(a.r0 + r) * a.part_len + base + row] = make_float2(y.re[r] * sc[r], y.im[r] * sc[r]);
    }
}

// a product's accumulator rows into the partial slots; `release` runs once
// every read of the accumulator is done, so that the buffer can take the
// next product.  Schedule 2 reads its 32 right-hand sides in two halves of
// 16 and stores each half at once, which keeps its registers within two CTAs
// per SM; the sums and stores are those of load_rows / store_rows.
template <int S, typename Rel>
__device__ __forceinline__ void drain_rows(const NzmArgs &a, uint32_t taddr, int row_ok, int row, long long base,
                                           const float *sc, unsigned on, Rel release) {
    if constexpr (S == 2) {
        constexpr int R = NzmSched<S>::R;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float p[16], q[16], re[16], im[16];
            tc_ld16(taddr + 16 * h, p);
            tc_ld16(taddr + R + 16 * h, q);
#pragma unroll
            for (int i = 0; i < 16; ++i) re[i] = p[i] + q[i];
            tc_ld16(taddr + 2 * R + 16 * h, p);
            tc_ld16(taddr + 3 * R + 16 * h, q);
#pragma unroll
            for (int i = 0; i < 16; ++i) im[i] = p[i] + q[i];
            if (h == 1) release();
            if (row_ok) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int r = 16 * h + i;
                    if (!((on >> r) & 1u)) continue;
                    a.part[(long long)(a.r0 + r) * a.part_len + base + row] = make_float2(re[i] * sc[r], im[i] * sc[r]);
                }
            }
        }
    } else {
        NzmRows<S> y;
        load_rows<S>(taddr, y);
        release();
        store_rows<S>(a, y, row_ok, row, base, sc, on);
    }
}

// one CTA per near-zone group, one pass of up to NzmSched<S>::R right-hand sides
template <int S>
__global__ void __launch_bounds__(NZM_THREADS, NzmSched<S>::CTAS) k_near_mma(NzmArgs a) {
    constexpr uint32_t NZM_TMEM_COLS = NzmSched<S>::TMEM;   // row product + two transposed buffers
    constexpr uint32_t DC = NzmSched<S>::DCOLS;
    extern __shared__ unsigned char nzm_raw[];
    // 128-byte aligned base: core matrices and bulk copies start on 16-byte
    // boundaries, slots on 128-byte boundaries
    unsigned char *sh = nzm_raw + ((128u - (smem_addr(nzm_raw) & 127u)) & 127u);
    uint64_t *full = reinterpret_cast<uint64_t *>(sh);
    uint64_t *empty = full + NZM_SLOTS;
    uint64_t *tfull = empty + NZM_SLOTS;
    uint64_t *tempty = tfull + 2;
    uint64_t *rowfull = tempty + 2;
    uint64_t *mmadone = rowfull + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mmadone + 1);
    uint32_t *toff = tslot + 1;                         // [NZM_SLOTS] ring offset of each slot's tile
    unsigned char *X1 = sh + NZM_META;
    unsigned char *ring = X1 + a.x1_bytes;

    const int g = blockIdx.x;
    const int t0 = a.grp_tile[g], t1 = a.grp_tile[g + 1];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // every byte the tensor core may read holds a finite value: zero the ring
    // and its slack once (the data copied in later are finite too)
    {
        uint4 *z = reinterpret_cast<uint4 *>(ring);
        const int nz = (int)((a.ring_bytes + a.slack_bytes) / 16);
        for (int i = threadIdx.x; i < nz; i += NZM_THREADS) z[i] = make_uint4(0, 0, 0, 0);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < NZM_SLOTS; ++k) {
            mbar_init(&full[k], 1);
            mbar_init(&empty[k], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&tfull[b], 1);
            mbar_init(&tempty[b], 4);
        }
        mbar_init(rowfull, 1);
        mbar_init(mmadone, 1);
        mbar_fence_init();
    }
    // the pass's scales and which right-hand sides to write, read once
    __shared__ float s_sc[NzmSched<S>::R];
    __shared__ unsigned s_on;
    if (warp == 2) {
        const int r = lane;
        const bool on = r < NzmSched<S>::R && r < a.rg && !(a.skip && a.skip[a.r0 + r]);
        if (r < NzmSched<S>::R) s_sc[r] = on ? a.xinv[r] : 0.f;
        const unsigned m = __ballot_sync(0xffffffffu, on);
        if (r == 0) s_on = m;
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_addr(tslot)),
                     "r"(NZM_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = *tslot;

    if (warp == 0) {
        // ------------------------------------------------------ producer
        if (lane == 0) {
            const uint32_t R = a.ring_bytes;
            uint32_t head = 0, used = 0;
            uint32_t resv[NZM_SLOTS] = {};
            int oldest = 0, count = 0, ord = 0;
            bool ok = true;
            const int n1 = a.grp_off[g + 1] - a.grp_off[g];
            for (int t = t0; t < t1 && ok; ++t, ++ord) {
                const NearTile &tl = a.tiles[t];
                const uint32_t mb = nzm_tile_bytes(tl.n1, tl.n2);
                const uint32_t xb = nzm_xblock_bytes<S>(tl.n2);
                const uint32_t x1b = t == t0 ? nzm_xblock_bytes<S>(n1) : 0u;
                const uint32_t SZ = mb + xb;
                bool fit = head + SZ <= R;
                uint32_t res = fit ? SZ : (R - head) + SZ;
                while (ok && count > 0 && (count == NZM_SLOTS || used + res > R)) {
                    const int k = oldest % NZM_SLOTS;
                    ok = mbar_wait(&empty[k], (uint32_t)((oldest / NZM_SLOTS) & 1), a.err);
                    used -= resv[k];
                    ++oldest;
                    --count;
                }
                if (!ok) break;
                if (count == 0) { head = 0; used = 0; fit = true; res = SZ; }
                const uint32_t st = fit ? head : 0u;
                const int k = ord % NZM_SLOTS;
                toff[k] = st;
                mbar_expect_tx(&full[k], SZ + x1b);
                bulk_g2s(ring + st, a.t16 + a.t16_off[t], mb, &full[k]);
                bulk_g2s(ring + st + mb, a.xb + a.xb_off[tl.g2], xb, &full[k]);
                if (x1b) bulk_g2s(X1, a.xb + a.xb_off[g], x1b, &full[k]);
                head = st + SZ;
                used += res;
                resv[k] = res;
                ++count;
            }
            // no copy of this CTA may still be in flight when it exits
            for (int o = ord - NZM_SLOTS > 0 ? ord - NZM_SLOTS : 0; o < ord; ++o)
                mbar_wait(&full[o % NZM_SLOTS], (uint32_t)((o / NZM_SLOTS) & 1), a.err);
        }
    } else if (warp == 1) {
        // ---------------------------------------------------- MMA issuer
        if (lane == 0) {
            const int n1 = a.grp_off[g + 1] - a.grp_off[g];
            int tcount = 0, ord = 0;
            bool ok = true;
            for (int t = t0; t < t1 && ok; ++t, ++ord) {
                const NearTile &tl = a.tiles[t];
                const int k = ord % NZM_SLOTS;
                if (!(ok = mbar_wait(&full[k], (uint32_t)((ord / NZM_SLOTS) & 1), a.err))) break;
                tc_fence_after();
                const uint32_t tile = smem_addr(ring + toff[k]);
                const uint32_t xblk = tile + nzm_tile_bytes(n1, tl.n2);
                issue_product<S>(0, n1, tl.n2, tile, xblk, tbase, t == t0);
                if (tl.col_off >= 0) {
                    constexpr int NB = NzmSched<S>::NBUF;
                    const int b = tcount % NB;
                    if (!(ok = mbar_wait(&tempty[b], (uint32_t)(((tcount / NB) & 1) ^ 1), a.err))) break;
                    tc_fence_after();
                    issue_product<S>(1, n1, tl.n2, tile, smem_addr(X1), tbase + DC * (1 + b), true);
                    tc_commit(&tfull[b]);
                    ++tcount;
                }
                tc_commit(&empty[k]);
            }
            tc_commit(rowfull);
            // every issued instruction has finished before tensor memory is released
            tc_commit(mmadone);
            mbar_wait(mmadone, 0u, a.err);
        }
    } else {
        // ------------------------------------------------------- epilogue
        const int quarter = warp & 3;                   // TMEM lanes 32*quarter .. +31
        const int n1 = a.grp_off[g + 1] - a.grp_off[g];
        int tcount = 0;
        bool ok = true;
        for (int t = t0; t < t1 && ok; ++t) {
            const NearTile &tl = a.tiles[t];
            if (tl.col_off < 0) continue;
            constexpr int NB = NzmSched<S>::NBUF;
            const int b = tcount % NB;
            if (!(ok = mbar_wait(&tfull[b], (uint32_t)((tcount / NB) & 1), a.err))) break;
            tc_fence_after();
            const int row = nzm_row_of_lane(nzm_M(1, n1, tl.n2), 32 * quarter + lane);
            drain_rows<S>(a, tbase + ((uint32_t)(32 * quarter) << 16) + DC * (1 + b), row >= 0 && row < 3 * tl.n2, row,
                          tl.col_off, s_sc, s_on, [&]() {
                              tc_fence_before();
                              __syncwarp();
                              if (lane == 0) mbar_arrive(&tempty[b]);
                          });
            ++tcount;
        }
        if (ok && mbar_wait(rowfull, 0u, a.err)) {
            tc_fence_after();
            const int row = nzm_row_of_lane(nzm_M(0, n1, 1), 32 * quarter + lane);
            drain_rows<S>(a, tbase + ((uint32_t)(32 * quarter) << 16), row >= 0 && row < 3 * n1, row, a.pslot_base[g],
                          s_sc, s_on, []() {});
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tbase), "r"(NZM_TMEM_COLS) : "memory");
    }
}

// per right-hand side r < rg: the largest |Re|, |Im| of x_r (float bits; a
// non-negative float orders like its bits)
__global__ void k_xabsmax(const cf *__restrict__ x, long long n, int r0, int rg, unsigned int *__restrict__ xmax) {
    const int r = blockIdx.y;
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const cf v = x[(long long)(r0 + r) * n + i];
        m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(&xmax[r], __float_as_uint(m));
}

// x blocks of one pass for every group: f16 hi/lo of sx * x (zero for
// unknowns beyond the group, absent or skipped right-hand sides); block 0
// also records 1 / (sA sx) per right-hand side
template <int S>
__global__ void k_xblocks(const cf *__restrict__ x, long long n, int r0, int rg, const int *__restrict__ skip,
                          const unsigned int *__restrict__ xmax, float sA, const int *__restrict__ grp_off,
                          const long long *__restrict__ xb_off, unsigned char *__restrict__ xb, float *__restrict__ xinv) {
    constexpr int R = NzmSched<S>::R;
    __shared__ float sx[R];
    if (threadIdx.x < R) sx[threadIdx.x] = nzm_scale_for(__uint_as_float(xmax[threadIdx.x]));
    __syncthreads();
    const int g = blockIdx.x;
    const int s0 = grp_off[g], ng = grp_off[g + 1] - s0;
    const int K = nzm_xk(ng);
    uint16_t *blk = reinterpret_cast<uint16_t *>(xb + xb_off[g]);
    const int total = 4 * R * K;
    for (int e = threadIdx.x; e < total; e += blockDim.x) blk[e] = nzm_xblock_bits<S>(x, n, r0, rg, skip, sx, s0, ng, e);
    if (g == 0 && threadIdx.x < R) {
        const int r = threadIdx.x;
        xinv[r] = r < rg ? 1.f / (sA * sx[r]) : 0.f;
    }
}

// largest |Re|, |Im| over the complex64 tile store
__global__ void k_tabsmax(const float *__restrict__ v, long long nv, unsigned int *__restrict__ out) {
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf(v[i]));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// f16 hi/lo planes of one tile from its complex64 blocks (one CTA per tile)
__global__ void k_tile_planes(const NearTile *__restrict__ tiles, const cf *__restrict__ data, float sA,
                              const long long *__restrict__ t16_off, unsigned char *__restrict__ t16) {
    const NearTile tl = tiles[blockIdx.x];
    const long long P = (long long)nzm_rows8(tl.n1) * nzm_cols8(tl.n2);
    uint16_t *pl = reinterpret_cast<uint16_t *>(t16 + t16_off[blockIdx.x]);
    for (long long e = threadIdx.x; e < P; e += blockDim.x) {
        uint16_t v[4];
        nzm_plane_values(tl, data, sA, e, [](int n1, int i, int j, int el) { return tile_at(n1, i, j, el); }, v);
#pragma unroll
        for (int p = 0; p < 4; ++p) pl[p * P + e] = v[p];
    }
}

}  // namespace

// f16 planes of every tile, x-block offsets and buffers (once per near zone)
int near_mma_prepare(scd_ctx *c) {
    if (c->nzm_ready) return SCD_OK;
    if (c->near_prec != SCD_STORE_C64) return set_error(c, SCD_BAD_ARG, "tensor-core near zone needs complex64 storage");
    auto fr = [](void *&p) { if (p) { cudaFree(p); p = nullptr; } };
    fr((void *&)c->d_t16); fr((void *&)c->d_t16_off); fr((void *&)c->d_xb); fr((void *&)c->d_xb_off);
    fr((void *&)c->d_xmax); fr((void *&)c->d_xinv);
    std::vector<long long> toff(c->ntiles + 1, 0);
    uint32_t slack = 0;
    for (int t = 0; t < c->ntiles; ++t) {
        const NearTile &tl = c->tiles_h[t];
        toff[t + 1] = toff[t] + nzm_tile_bytes(tl.n1, tl.n2);
        slack = std::max({slack, nzm_overrun<0>(tl.n1, tl.n2), nzm_overrun<1>(tl.n1, tl.n2), nzm_overrun<2>(tl.n1, tl.n2)});
    }
    // x blocks sized for the widest pass (schedule 2), so every schedule fits
    std::vector<long long> xoff(c->ngroups + 1, 0);
    for (int g = 0; g < c->ngroups; ++g) xoff[g + 1] = xoff[g] + nzm_xblock_bytes<2>(c->grp_off[g + 1] - c->grp_off[g]);
    auto al = [&](void **p, size_t bytes, const char *what) -> int {
        if (cudaMalloc(p, std::max<size_t>(bytes, 16)) != cudaSuccess) {
            cudaGetLastError();
            return set_error(c, SCD_OOM, "tensor-core near zone: %s (%zu bytes)", what, bytes);
        }
        return SCD_OK;
    };
    int rc;
    if ((rc = al((void **)&c->d_t16, (size_t)toff[c->ntiles], "tile planes")) ||
        (rc = al((void **)&c->d_t16_off, sizeof(long long) * c->ntiles, "tile offsets")) ||
        (rc = al((void **)&c->d_xb, (size_t)xoff[c->ngroups], "x blocks")) ||
        (rc = al((void **)&c->d_xb_off, sizeof(long long) * c->ngroups, "x-block offsets")) ||
        (rc = al((void **)&c->d_xmax, sizeof(unsigned int) * (NZM_RMAX + 1), "x scales")) ||
        (rc = al((void **)&c->d_xinv, sizeof(float) * NZM_RMAX, "x scales")))
        return rc;
    if ((rc = check_cuda(c, cudaMemcpyAsync(c->d_t16_off, toff.data(), sizeof(long long) * c->ntiles, cudaMemcpyHostToDevice, c->st),
                         "tile offsets")) ||
        (rc = check_cuda(c, cudaMemcpyAsync(c->d_xb_off, xoff.data(), sizeof(long long) * c->ngroups, cudaMemcpyHostToDevice, c->st),
                         "x-block offsets")))
        return rc;
    // one power-of-two scale for all tiles
    unsigned int mbits = 0;
    unsigned int *dm = c->d_xmax + NZM_RMAX;
    if ((rc = check_cuda(c, cudaMemsetAsync(dm, 0, sizeof(unsigned int), c->st), "tile scale"))) return rc;
    k_tabsmax<<<4 * c->nsm, 256, 0, c->st>>>((const float *)c->d_tdata, 2 * c->tile_store, dm);
    if ((rc = check_cuda(c, cudaMemcpyAsync(&mbits, dm, sizeof(unsigned int), cudaMemcpyDeviceToHost, c->st), "tile scale")) ||
        (rc = check_cuda(c, cudaStreamSynchronize(c->st), "tile scale")))
        return rc;
    float m;
    memcpy(&m, &mbits, sizeof m);
    if (!std::isfinite(m)) return set_error(c, SCD_NAN, "near-zone tiles hold a non-finite value");
    c->nzm_sA = nzm_scale_for(m);
    if (c->ntiles > 0)
        k_tile_planes<<<c->ntiles, 256, 0, c->st>>>(c->d_tiles, (const cf *)c->d_tdata, c->nzm_sA, c->d_t16_off, c->d_t16);
    if ((rc = check_cuda(c, cudaGetLastError(), "tile planes")) ||
        (rc = check_cuda(c, cudaStreamSynchronize(c->st), "tile planes")))
        return rc;
    // shared memory per pass width (16: schedules 0 and 1, 32: schedule 2):
    // meta, the row group's x block, the ring, its slack
    c->nzm_slack = (slack + 127u) & ~127u;
    for (int w = 0; w < 2; ++w) {
        auto xbytes = [w](int n) { return w ? nzm_xblock_bytes<2>(n) : nzm_xblock_bytes<1>(n); };
        const uint32_t x1 = xbytes(c->max_per_group);
        uint32_t max_slot = 0;
        for (int t = 0; t < c->ntiles; ++t) {
            const NearTile &tl = c->tiles_h[t];
            max_slot = std::max(max_slot, nzm_tile_bytes(tl.n1, tl.n2) + xbytes(tl.n2));
        }
        size_t budget = w ? NZM_SMEM_WIDE : NZM_SMEM;
        {
            // what the SM holds for this many CTAs: per CTA its static bytes
            // and the reserved kilobyte come out of the SM's shared memory
            int per_sm = 0, reserved = 0, optin = 0;
            cudaFuncAttributes fa{};
            const cudaError_t e1 = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, c->dev);
            const cudaError_t e2 = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, c->dev);
            const cudaError_t e3 = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->dev);
            const cudaError_t e4 = w ? cudaFuncGetAttributes(&fa, k_near_mma<2>) : cudaFuncGetAttributes(&fa, k_near_mma<1>);
            if (e1 == cudaSuccess && e2 == cudaSuccess && e3 == cudaSuccess && e4 == cudaSuccess) {
                const int ctas = w ? NzmSched<2>::CTAS : NzmSched<1>::CTAS;
                const long long fit = (long long)per_sm / ctas - reserved - (long long)fa.sharedSizeBytes;
                budget = (size_t)std::max<long long>(0, std::min<long long>(fit, optin - (long long)fa.sharedSizeBytes));
                budget = budget / 1024 * 1024;
            } else {
                cudaGetLastError();
            }
        }
        const size_t fixed = 128 + NZM_META + x1 + c->nzm_slack;
        size_t ring = budget > fixed ? (budget - fixed) / 128 * 128 : 0;
        if (ring < max_slot) ring = (size_t)max_slot;   // one slot at least (then one CTA per SM)
        if (fixed + ring > 227 * 1024) return set_error(c, SCD_BAD_ARG, "tensor-core near zone: a tile does not fit");
        c->nzm_x1[w] = x1;
        c->nzm_ring[w] = (uint32_t)ring;
    }
    c->nzm_ready = true;
    return SCD_OK;
}

// one pass of schedule S over right-hand sides r0 .. r0 + rg - 1
template <int S>
static void near_mma_pass(scd_ctx *c, const cf *x, int r0, int rg, const int *done) {
    constexpr int R = NzmSched<S>::R;
    const int w = R == NZM_RMAX ? 1 : 0;
    const size_t sh = 128 + NZM_META + c->nzm_x1[w] + c->nzm_ring[w] + c->nzm_slack;
    cudaFuncSetAttribute(k_near_mma<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh);
    cudaMemsetAsync(c->d_xmax, 0, sizeof(unsigned int) * R, c->st);
    k_xabsmax<<<dim3((unsigned)c->nsm, (unsigned)rg), 256, 0, c->st>>>(x, c->n, r0, rg, c->d_xmax);
    k_xblocks<S><<<c->ngroups, 256, 0, c->st>>>(x, c->n, r0, rg, done, c->d_xmax, c->nzm_sA, c->d_grp_off,
                                               c->d_xb_off, c->d_xb, c->d_xinv);
    NzmArgs a;
    a.tiles = c->d_tiles; a.grp_tile = c->d_grp_tile; a.grp_off = c->d_grp_off; a.pslot_base = c->d_pslot_base;
    a.t16 = c->d_t16; a.t16_off = c->d_t16_off; a.xb = c->d_xb; a.xb_off = c->d_xb_off;
    a.part = c->f_nzpart; a.part_len = c->part_len; a.skip = done; a.r0 = r0; a.rg = rg; a.xinv = c->d_xinv;
    a.x1_bytes = c->nzm_x1[w]; a.ring_bytes = c->nzm_ring[w]; a.slack_bytes = c->nzm_slack; a.err = c->d_kerr;
    if (c->timing) cudaEventRecord(c->ev[6], c->st);
    k_near_mma<S><<<c->ngroups, NZM_THREADS, sh, c->st>>>(a);
    if (c->timing) cudaEventRecord(c->ev[7], c->st);
    c->launches += 3;
}

// near-zone partial slots of nrhs complex64 right-hand sides (columns of
// stride n): passes of 16 (schedules 0, 1); with schedule 2, passes of 32
// while more than 16 remain and a last pass of schedule 1 (a 32-wide pass
// costs twice the tensor work of a 16-wide one).  Schedules 1 and 2 form
// every output element from the same K = 16 products in the same order (hi
// part, then lo part, added pairwise) and differ only in how many columns
// one instruction covers, so a column gets the same bits from either;
// tests/test_gpu_near_mma.py checks that on the device.
void near_mma_run(scd_ctx *c, const cf *x, int nrhs, const int *done) {
    for (int r0 = 0; r0 < nrhs;) {
        const int left = nrhs - r0;
        if (c->nzm_sched == 2 && left > NZM_R) {
            const int rg = std::min(NZM_RMAX, left);
            near_mma_pass<2>(c, x, r0, rg, done);
            r0 += rg;
        } else {
            const int rg = std::min(NZM_R, left);
            if (c->nzm_sched == 0) near_mma_pass<0>(c, x, r0, rg, done);
            else near_mma_pass<1>(c, x, r0, rg, done);
            r0 += rg;
        }
    }
}
