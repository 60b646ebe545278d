// Batched T-matrix column solves: `nslots` GMRES solves advance together,
// one Arnoldi step per tick, sharing every read of the operator (projectors,
// Green octant, near-zone tiles) and every grid barrier.  Each slot runs its
// own restarted GMRES exactly as gmres (src/gmres_module.f90:180-325): x0 =
// rhs, MGS with the conditional re-orthogonalisation, complex Givens, y =
// H^-1 g, x += V y.  A slot's arithmetic does not depend on what the other slots hold
// (per-slot reductions over fixed chunks, summed in a fixed order), so a
// column's result is bit-identical whether it is solved alone (scd_gmres
// runs one slot) or in a batch.  A slot whose column converged (or ran out
// of cycles) is refilled with the next column on the following tick
// (continuous batching).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "ctx.h"

namespace {

constexpr int BT = 256;             // threads per CTA of the tick kernel
constexpr int NSMAX = 64;           // slot limit (partial buffer sizing)
constexpr int BW = BT / 32;         // warps per CTA
// resident CTAs per SM the complex64 tick is compiled for (its register cap;
// the cooperative grid follows the occupancy this gives)
#ifndef SCD_TICK_MINB
#define SCD_TICK_MINB 2
#endif

enum { SLOT_FREE = 0, SLOT_START = 1, SLOT_ARNOLDI = 2, SLOT_DONE = 3, SLOT_RESID = 4, SLOT_INNER_DONE = 5 };

// One column in flight.  Plain form: START/ARNOLDI until DONE.  Mixed form:
// RESID (FP64 residual of the FP64 iterate) -> inner complex64 GMRES on the
// normalised residual (START/ARNOLDI, zero initial guess) -> INNER_DONE
// (x += rho d) -> RESID ... until the FP64 residual meets the tolerance.
struct Slot {
    int mode, col, cycle, step, iters, conv, status, reorth, finish, zero_x;
    int outer, upd;    // mixed: outer steps taken; x += rho d pending
    int mpos, rpos;    // column of this slot in the tick's compacted matvec input (inner, FP64 residual), -1: none
    double b_norm, beta, error;
    double rho;        // mixed: ||r|| of the residual the inner solve corrects
    double b64;        // mixed: ||rhs|| in FP64
    double relres;     // mixed: last FP64 relative residual
};

template <typename C>
struct TickArgs {
    Slot *slots;
    int ns;
    C *V;           // [slot][m+1][n]
    cd *H;          // [slot][(m+1) m]
    cd *cs, *sn, *g, *y;   // [slot][m+1]
    C *x, *rhs, *w; // [slot][n]
    double *red;    // [2][grid][NSMAX*4]
    double *cpart;  // [NSMAX][NCH][4] chunk partials
    double *ctot;   // [2][NSMAX][4] slot totals
    int *ccnt;      // [NSMAX] chunks published in the current reduction
    int *qctr;      // [QMAX] work-queue counters, one per phase of the tick
    GridBarrier *bar;
    int *err;
    long long n;
    int m, max_cycles;
    double tol;
    int mixed;      // inner solve of the mixed form: finish -> INNER_DONE
    int cgs;        // classical Gram-Schmidt for the Arnoldi steps (complex64 inner solves, opt-in)
    double *cpm;    // cgs: [slot][NCH][CGS_NV] chunk partials of the dots
    double *ctm;    // cgs: [slot][CGS_NV] slot totals
};

// vector elements in FP64 for arithmetic, rounded back on store
__device__ __forceinline__ cd to_cd(cd a) { return a; }
__device__ __forceinline__ cd to_cd(cf a) { return widen(a); }
__device__ __forceinline__ void store_c(cd &d, cd v) { d = v; }
__device__ __forceinline__ void store_c(cf &d, cd v) { d = make_float2((float)v.x, (float)v.y); }
// v rounded to the storage precision C, back in FP64
template <typename C> __device__ __forceinline__ cd rounded(cd v);
template <> __device__ __forceinline__ cd rounded<cd>(cd v) { return v; }
template <> __device__ __forceinline__ cd rounded<cf>(cd v) { return widen(make_float2((float)v.x, (float)v.y)); }

// Streaming loops take a lane's elements of a chunk TU at a time: the loads
// of TU elements are issued together (memory-level parallelism), the
// arithmetic runs in the same element order as a plain loop.
constexpr int TU = 4;

// ---- reductions over fixed chunks
// Every slot vector is cut into NCH fixed chunks; chunk c of slot s is
// always handled by global warp (s*NCH + c) mod (warps in the grid), its
// lanes take elements q = c*L + lane + 32t in order (TU at a time, loads
// first), the lanes' sums meet in an xor tree, and the last warp to finish a
// slot adds its NCH chunk partials (lane l: chunks l, l+32, ..., then an xor
// tree) into the slot's total.  The arithmetic of a slot therefore depends
// on n and the grid only -- never on which other slots are active -- and
// each warp streams long contiguous runs (deep memory-level parallelism).
constexpr int NCH = 512;
// values per slot of the classical Gram-Schmidt reduction: <v_k, w> for k <=
// SCD_M_MAX (two doubles each) and ||w||^2
constexpr int CGS_NV = 2 * SCD_M_MAX + 2;

struct Chunks {
    long long L;    // chunk length
    int gw, nw;     // this warp, warps in the grid
    int lane;
    __device__ Chunks(long long n, int nch) {
        L = (n + nch - 1) / nch;
        gw = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
        nw = (int)(((long long)gridDim.x * blockDim.x) >> 5);
        lane = threadIdx.x & 31;
    }
};

// Work items (slot, chunk) of a phase.  With at least two items per warp
// they are handed out in runs of QG by an atomic counter, the slots with the
// most Krylov vectors first, so that warps finish a phase together instead of
// waiting at the next grid barrier for the one whose fixed share held the
// long slots; with fewer, warp w takes items w, w + warps, ... (a counter
// that every warp polls would cost more than the imbalance).  Which warp
// takes an item does not change any result: every item publishes its partial
// sums to a fixed place, summed in chunk order.
constexpr int QG = 4;                          // items per grab
constexpr int QMAX = 256;                      // phases (counters) per tick
static_assert(QMAX >= 8 + 3 * (SCD_M_MAX + 1), "one counter per phase of a tick");
struct WorkQueue {
    int *ctr;
    int n, lane, it, end, step;
    bool dyn;
    __device__ WorkQueue(int *c, int nitems, const Chunks &ch)
        : ctr(c), n(nitems), lane(ch.lane), it(0), end(0), step(ch.nw), dyn(nitems >= 2 * ch.nw) {
        if (!dyn) it = ch.gw - ch.nw;
    }
    __device__ bool next() {
        if (!dyn) {
            it += step;
            return it < n;
        }
        if (++it < end) return true;
        int base = 0;
        if (lane == 0) base = atomicAdd(ctr, QG);
        base = __shfl_sync(0xffffffffu, base, 0);
        it = base;
        end = min(n, base + QG);
        return base < n;
    }
};

// the per-lane sums v of chunk c of slot s: fold, publish, and let the
// slot's last warp form the total
template <int NV, typename C>
__device__ __forceinline__ void chunk_done(const TickArgs<C> &a, int s, int c, double (&v)[NV], int parity, int lane) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
    int last = 0;
    if (lane == 0) {
        double *p = a.cpart + ((size_t)s * NCH + c) * 4;
#pragma unroll
        for (int k = 0; k < NV; ++k) p[k] = v[k];
        __threadfence();
        last = atomicAdd(&a.ccnt[s], 1) == NCH - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
        __threadfence();
        // all loads first (they are independent), then the sums in chunk order
        double pv[NCH / 32][NV];
#pragma unroll
        for (int j = 0; j < NCH / 32; ++j) {
            const double *p = a.cpart + ((size_t)s * NCH + lane + 32 * j) * 4;
#pragma unroll
            for (int k = 0; k < NV; ++k) pv[j][k] = __ldcg(p + k);
        }
        double t[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) t[k] = 0.0;
#pragma unroll
        for (int j = 0; j < NCH / 32; ++j)
#pragma unroll
            for (int k = 0; k < NV; ++k) t[k] += pv[j][k];
#pragma unroll
        for (int k = 0; k < NV; ++k) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
        }
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NV; ++k) a.ctot[((size_t)parity * NSMAX + s) * 4 + k] = t[k];
            a.ccnt[s] = 0;
        }
    }
}

// after the grid barrier: the totals of the flagged slots into shared memory
template <typename C>
__device__ __forceinline__ void load_totals(const TickArgs<C> &a, int parity, int nv, const int *act, double (*tot)[4]) {
    for (int e = threadIdx.x; e < a.ns * 4; e += blockDim.x) {
        const int s = e >> 2, k = e & 3;
        if (k < nv && act[s]) tot[s][k] = __ldcg(a.ctot + ((size_t)parity * NSMAX + s) * 4 + k);
    }
    __syncthreads();
}

// Givens update of the new H column, residual estimate and, when a cycle
// ends, y = H^-1 g (back substitution) for every Arnoldi slot: CTA 0, one
// warp per slot.  H column i-1 is complete except H(i, i-1) = shn[s];
// sreo[s] flags a re-orthogonalised step (counted).  The warp stages the
// column in shared memory (hw) so that lane 0 applies the rotations in their
// order without a global-memory round trip per step; the back substitution
// runs column by column over the warp, lane r holding rows r and r + 32.
template <typename C>
__device__ void givens_step(const TickArgs<C> &a, const int *smode, const int *sstep, const double *shn, const int *sreo,
                            cd (*hws)[SCD_M_MAX + 1]) {
    const int ldh = a.m + 1;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    cd *hw = hws[warp];
    for (int s = warp; s < a.ns; s += BW) {
        if (smode[s] != SLOT_ARNOLDI) continue;   // uniform across the warp
        Slot &sl = a.slots[s];
        const int i = sstep[s] + 1;
        cd *Hc = a.H + (size_t)s * ldh * a.m + (size_t)ldh * (i - 1);
        cd *cs = a.cs + (size_t)s * (a.m + 1), *sn = a.sn + (size_t)s * (a.m + 1), *g = a.g + (size_t)s * (a.m + 1);
        __syncwarp();
        for (int k = lane; k < i; k += 32) hw[k] = Hc[k];
        if (lane == 0) hw[i] = cmk(shn[s], 0.0);
        // the rotations so far, two per lane (k = lane, lane + 32)
        cd c0 = cmk(0, 0), s0 = cmk(0, 0), c1 = cmk(0, 0), s1 = cmk(0, 0);
        if (lane < i - 1) { c0 = cs[lane]; s0 = sn[lane]; }
        if (lane + 32 < i - 1) { c1 = cs[lane + 32]; s1 = sn[lane + 32]; }
        __syncwarp();
        int fin = 0;
        for (int k = 1; k <= i - 1; ++k) {
            const int src = (k - 1) & 31;
            const bool hi = k - 1 >= 32;
            cd c, sv;
            c.x = __shfl_sync(0xffffffffu, hi ? c1.x : c0.x, src);
            c.y = __shfl_sync(0xffffffffu, hi ? c1.y : c0.y, src);
            sv.x = __shfl_sync(0xffffffffu, hi ? s1.x : s0.x, src);
            sv.y = __shfl_sync(0xffffffffu, hi ? s1.y : s0.y, src);
            if (lane == 0) {
                const cd tmp = csub(cmul(c, hw[k - 1]), cmul(sv, hw[k]));
                hw[k] = cadd(cmul(sv, hw[k - 1]), cmul(cconj(c), hw[k]));
                hw[k - 1] = tmp;
            }
        }
        if (lane == 0) {
            const double nu = sqrt(cabs2(hw[i - 1]) + cabs2(hw[i]));
            if (nu != 0.0) {
                const cd c = cconj(cmk(hw[i - 1].x / nu, hw[i - 1].y / nu));
                const cd sv = cmk(-hw[i].x / nu, -hw[i].y / nu);
                cs[i - 1] = c;
                sn[i - 1] = sv;
                hw[i - 1] = csub(cmul(c, hw[i - 1]), cmul(sv, hw[i]));
                hw[i] = cmk(0, 0);
                const cd t1 = g[i - 1], t2 = g[i];
                g[i - 1] = csub(cmul(c, t1), cmul(sv, t2));
                g[i] = cadd(cmul(sv, t1), cmul(cconj(c), t2));
            }
            const double error = sqrt(cabs2(g[i])) / sl.b_norm;
            sl.error = error;
            sl.step = i;
            sl.iters += 1;
            if (sreo[s]) sl.reorth += 1;
            sl.finish = 0;
            if (error < a.tol) { sl.conv = 1; sl.finish = 1; }
            else if (i == a.m) sl.finish = 1;
            if (!(error == error)) { sl.status = SCD_NAN; sl.finish = 0; sl.mode = SLOT_DONE; }
            if (*a.err) { sl.status = SCD_TIMEOUT; sl.finish = 0; sl.mode = SLOT_DONE; }
            fin = sl.finish;
        }
        __syncwarp();
        for (int k = lane; k <= i; k += 32) Hc[k] = hw[k];
        fin = __shfl_sync(0xffffffffu, fin, 0);
        if (fin) {
            // y = H(1:i,1:i)^-1 g(1:i): column cc gives y_cc on the lane of row
            // cc, then every row above subtracts H(r, cc) y_cc
            __syncwarp();   // g and column i-1 of H as written by lane 0
            const cd *Hs = a.H + (size_t)s * ldh * a.m;
            cd *ys = a.y + (size_t)s * (a.m + 1);
            const cd *gv = g;
            cd b0 = lane < i ? gv[lane] : cmk(0, 0), b1 = lane + 32 < i ? gv[lane + 32] : cmk(0, 0);
            for (int cc = i - 1; cc >= 0; --cc) {
                const cd *col = Hs + (size_t)ldh * cc;
                const cd h0 = lane <= cc ? col[lane] : cmk(0, 0);
                const cd h1 = lane + 32 <= cc ? col[lane + 32] : cmk(0, 0);
                const int own = cc & 31;
                const bool hi = cc >= 32;
                cd yc = cmk(0, 0);
                if (lane == own) yc = cdiv(hi ? b1 : b0, hi ? h1 : h0);
                yc.x = __shfl_sync(0xffffffffu, yc.x, own);
                yc.y = __shfl_sync(0xffffffffu, yc.y, own);
                if (lane == own) ys[cc] = yc;
                if (lane < cc) b0 = csub(b0, cmul(h0, yc));
                if (lane + 32 < cc) b1 = csub(b1, cmul(h1, yc));
            }
        }
    }
}

// Cycle ends (x += V(:,1:i) y, chunks handled like the streaming phases)
// and the slots' next modes.  Call after the grid barrier that follows
// givens_step.
template <typename C>
__device__ void cycle_end(const TickArgs<C> &a, const Chunks &ch, int nch, const int *smode, cd (*ysm)[SCD_M_MAX + 1],
                          const int *sorder, int *qctr) {
    const long long n = a.n;
    constexpr int TUC = sizeof(C) == 8 ? 2 * TU : TU;
    const int lane = ch.lane;
    const int nitems = a.ns * nch;
    {
        cd *yw = ysm[threadIdx.x >> 5];
        for (WorkQueue q(qctr, nitems, ch); q.next();) {
            const int s = sorder[q.it / nch], c = q.it % nch;
            if (smode[s] != SLOT_ARNOLDI) continue;
            const Slot *sl = a.slots + s;
            if (!__ldcg(&sl->finish)) continue;      // uniform across the warp (L2 read after the barrier)
            const int kd = __ldcg(&sl->step);
            const cd *ys = a.y + (size_t)s * (a.m + 1);
            for (int cc = lane; cc < kd; cc += 32) yw[cc] = make_double2(__ldcg(&ys[cc].x), __ldcg(&ys[cc].y));
            __syncwarp();
            const long long qa = c * ch.L, qb = min(n, qa + ch.L);
            const C *Vs = a.V + (size_t)s * (a.m + 1) * n;
            C *xs = a.x + (size_t)s * n;
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd acc[TUC];
#pragma unroll
                for (int e = 0; e < TUC; ++e) acc[e] = cmk(0, 0);
                for (int cc = 0; cc < kd; ++cc) {
                    const cd yc = yw[cc];
                    const C *vc = Vs + (size_t)cc * n;
#pragma unroll
                    for (int e = 0; e < TUC; ++e) {
                        const long long qq = q + 32 * e;
                        if (qq < qb) cfma(acc[e], to_cd(vc[qq]), yc);
                    }
                }
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    if (qq < qb) store_c(xs[qq], cadd(to_cd(xs[qq]), acc[e]));
                }
            }
            __syncwarp();
        }
    }
    if (blockIdx.x == 0) {
        // `finish` stays set: other CTAs may still be reading it; the next
        // Givens update of the slot overwrites it
        for (int s = threadIdx.x; s < a.ns; s += blockDim.x) {
            if (smode[s] != SLOT_ARNOLDI) continue;
            Slot &sl = a.slots[s];
            if (!sl.finish) continue;
            if (sl.conv) sl.mode = a.mixed ? SLOT_INNER_DONE : SLOT_DONE;
            else if (sl.cycle < a.max_cycles) { sl.mode = SLOT_START; sl.zero_x = 0; }
            else sl.mode = a.mixed ? SLOT_INNER_DONE : SLOT_DONE;
        }
    }
}

// Classical Gram-Schmidt, first pass, chunk c of slot s: the dots <v_k, w>,
// k = 1..i, and ||w||^2 in one sweep over the chunk (w is re-read from cache
// for each k), published per chunk; the slot's last warp sums the NCH chunk
// partials of every value in chunk order into ctm.
template <typename C, int TUC>
__device__ __forceinline__ void cgs_dots(const TickArgs<C> &a, int s, int c, int i, const C *Vs, const C *ws,
                                         long long qa, long long qb, int lane) {
    const long long n = a.n;
    double *pp = a.cpm + ((size_t)s * NCH + c) * CGS_NV;
    double nw = 0.0;
    for (int k = 1; k <= i; ++k) {
        const C *vk = Vs + (size_t)(k - 1) * n;
        double d[2] = {0.0, 0.0};
        for (long long q = qa + lane; q < qb; q += 32 * TUC) {
            C w[TUC], z[TUC];
#pragma unroll
            for (int e = 0; e < TUC; ++e) {
                const long long qq = q + 32 * e;
                w[e] = z[e] = C{};
                if (qq < qb) { w[e] = ws[qq]; z[e] = vk[qq]; }
            }
#pragma unroll
            for (int e = 0; e < TUC; ++e) {
                if (q + 32 * e >= qb) break;
                const cd wv = to_cd(w[e]);
                cdot_acc(d[0], d[1], to_cd(z[e]), wv);
                if (k == 1) nw += cabs2(wv);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) d[h] += __shfl_xor_sync(0xffffffffu, d[h], o);
        if (lane == 0) { pp[2 * (k - 1)] = d[0]; pp[2 * (k - 1) + 1] = d[1]; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nw += __shfl_xor_sync(0xffffffffu, nw, o);
    int last = 0;
    if (lane == 0) {
        pp[CGS_NV - 1] = nw;
        __threadfence();
        last = atomicAdd(&a.ccnt[s], 1) == NCH - 1;
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (!last) return;
    __threadfence();
    double *tt = a.ctm + (size_t)s * CGS_NV;
    for (int v = 0; v < CGS_NV; ++v) {
        if (v >= 2 * i && v != CGS_NV - 1) continue;
        double t = 0.0;
#pragma unroll
        for (int j = 0; j < NCH / 32; ++j) t += __ldcg(a.cpm + ((size_t)s * NCH + lane + 32 * j) * CGS_NV + v);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if (lane == 0) tt[v] = t;
    }
    if (lane == 0) a.ccnt[s] = 0;
}

// One tick: cycle starts (r = rhs - A x, V0 = r/||r||) and Arnoldi steps
// (MGS, normalisation, Givens) for every active slot; cycle ends update x.
template <typename C>
__global__ void __launch_bounds__(BT, sizeof(C) == 8 ? SCD_TICK_MINB : 2) k_tick(TickArgs<C> a) {
    __shared__ double tot[NSMAX][4];
    __shared__ int smode[NSMAX], sstep[NSMAX], szero[NSMAX], swpos[NSMAX], sact[NSMAX], sro[NSMAX];
    __shared__ double snormav[NSMAX], shn[NSMAX];
    __shared__ cd sh_h[NSMAX];
    __shared__ cd ysm[BW][SCD_M_MAX + 1];    // per warp: y of the slot being updated
    const long long n = a.n;
    constexpr int TUC = sizeof(C) == 8 ? 2 * TU : TU;   // complex64: twice the elements in flight
    const int ldh = a.m + 1;
    const Chunks ch(n, NCH);
    const int lane = ch.lane;
    const int nitems = a.ns * NCH;
    for (int s = threadIdx.x; s < a.ns; s += blockDim.x) {
        smode[s] = a.slots[s].mode;
        sstep[s] = a.slots[s].step;
        szero[s] = a.slots[s].zero_x;
        swpos[s] = max(a.slots[s].mpos, 0);   // A v of the slot sits in column mpos of w
    }
    __syncthreads();
    // slots by cost (Krylov vectors a step reads), largest first, ties by index
    __shared__ int sorder[NSMAX];
    if (threadIdx.x == 0) {
        auto cost = [&](int s) { return smode[s] == SLOT_ARNOLDI ? sstep[s] + 2 : smode[s] == SLOT_START ? 1 : 0; };
        for (int s = 0; s < a.ns; ++s) {
            const int cs = cost(s);
            int j = s - 1;
            while (j >= 0 && cost(sorder[j]) < cs) { sorder[j + 1] = sorder[j]; --j; }
            sorder[j + 1] = s;
        }
    }
    __syncthreads();
    int ph = 0;        // phases so far: each takes the next work-queue counter
    int parity = 0;
    // ---- phase A: first reduction of every active slot
    for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
        const int s = sorder[q.it / NCH], c = q.it % NCH;
        const int md = smode[s];
        if (md != SLOT_START && md != SLOT_ARNOLDI) continue;
        const long long qa = c * ch.L, qb = min(n, qa + ch.L);
        double v[3] = {0, 0, 0};
        const C *ws = a.w + (size_t)swpos[s] * n;
        C *V0 = a.V + (size_t)s * (a.m + 1) * n;
        if (md == SLOT_START) {
            const C *bs = a.rhs + (size_t)s * n;
            const bool zx = szero[s] != 0;
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd b[TUC], w[TUC];
#pragma unroll
                for (int u = 0; u < TUC; ++u) {
                    const long long qq = q + 32 * u;
                    b[u] = w[u] = cmk(0, 0);
                    if (qq < qb) {
                        b[u] = to_cd(bs[qq]);
                        if (!zx) w[u] = to_cd(ws[qq]);
                    }
                }
#pragma unroll
                for (int u = 0; u < TUC; ++u) {
                    const long long qq = q + 32 * u;
                    if (qq >= qb) break;
                    const cd r = zx ? b[u] : csub(b[u], w[u]);
                    store_c(V0[qq], r);
                    v[0] += cabs2(r);
                    v[1] += cabs2(b[u]);
                }
            }
        } else if (a.cgs) {
            cgs_dots<C, TUC>(a, s, c, sstep[s] + 1, V0, ws, qa, qb, lane);
            continue;
        } else {
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd w[TUC], z[TUC];
#pragma unroll
                for (int u = 0; u < TUC; ++u) {
                    const long long qq = q + 32 * u;
                    w[u] = z[u] = cmk(0, 0);
                    if (qq < qb) { w[u] = to_cd(ws[qq]); z[u] = to_cd(V0[qq]); }
                }
#pragma unroll
                for (int u = 0; u < TUC; ++u) {
                    if (q + 32 * u >= qb) break;
                    v[0] += cabs2(w[u]);
                    cdot_acc(v[1], v[2], z[u], w[u]);
                }
            }
        }
        chunk_done<3>(a, s, c, v, parity, lane);
    }
    for (int s = threadIdx.x; s < a.ns; s += blockDim.x)
        sact[s] = smode[s] == SLOT_START || (smode[s] == SLOT_ARNOLDI && !a.cgs);
    grid_barrier(a.bar, gridDim.x, a.err);
    load_totals(a, parity, 3, sact, tot);
    int kmax = 0;
    for (int s = 0; s < a.ns; ++s) {
        if (smode[s] == SLOT_ARNOLDI && !a.cgs) kmax = max(kmax, sstep[s] + 1);
        if (threadIdx.x == 0) {
            if (smode[s] == SLOT_ARNOLDI && a.cgs) {
                snormav[s] = sqrt(__ldcg(a.ctm + (size_t)s * CGS_NV + CGS_NV - 1));
            } else {
                snormav[s] = sqrt(tot[s][0]);
                sh_h[s] = cmk(tot[s][1], tot[s][2]);
            }
        }
    }
    __syncthreads();
    // cycle starts: normalise V0, set g, b_norm
    for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
        const int s = sorder[q.it / NCH], c = q.it % NCH;
        if (smode[s] != SLOT_START) continue;
        const double beta = sqrt(tot[s][0]);
        const long long qa = c * ch.L, qb = min(n, qa + ch.L);
        C *V0 = a.V + (size_t)s * (a.m + 1) * n;
        for (long long q = qa + lane; q < qb; q += 32 * TUC) {
            cd r[TUC];
#pragma unroll
            for (int u = 0; u < TUC; ++u) {
                const long long qq = q + 32 * u;
                r[u] = qq < qb ? to_cd(V0[qq]) : cmk(0, 0);
            }
#pragma unroll
            for (int u = 0; u < TUC; ++u) {
                const long long qq = q + 32 * u;
                if (qq < qb) store_c(V0[qq], cmk(r[u].x / beta, r[u].y / beta));
            }
        }
    }
    if (blockIdx.x == 0 && threadIdx.x < a.ns) {
        const int s = threadIdx.x;
        if (smode[s] == SLOT_START) {
            const double beta = sqrt(tot[s][0]);
            Slot &sl = a.slots[s];
            cd *gs = a.g + (size_t)s * (a.m + 1);
            for (int i = 0; i <= a.m; ++i) gs[i] = cmk(0, 0);
            gs[0] = cmk(beta, 0.0);
            sl.beta = beta;
            if (sl.cycle == 0) sl.b_norm = sqrt(tot[s][1]);
            sl.cycle += 1;
            sl.step = 0;
            sl.mode = SLOT_ARNOLDI;
            if (sl.cycle == 1 && sl.b_norm == 0.0) { sl.error = 0.0; sl.conv = 1; sl.mode = SLOT_DONE; }
            else if (!(beta == beta)) { sl.status = SCD_NAN; sl.mode = SLOT_DONE; }
        }
    }
    // ---- MGS for the Arnoldi slots: one barrier per term
    for (int k = 1; k <= kmax; ++k) {
        for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
            const int s = sorder[q.it / NCH], c = q.it % NCH;
            if (smode[s] != SLOT_ARNOLDI) continue;
            const int i = sstep[s] + 1;
            if (k > i) continue;
            const cd h = sh_h[s];
            if (c == 0 && lane == 0) a.H[(size_t)s * ldh * a.m + (size_t)ldh * (i - 1) + (k - 1)] = h;
            const long long qa = c * ch.L, qb = min(n, qa + ch.L);
            C *ws = a.w + (size_t)swpos[s] * n;
            const C *Vs = a.V + (size_t)s * (a.m + 1) * n;
            const C *vk = Vs + (size_t)(k - 1) * n;
            const C *vn = (k < i) ? Vs + (size_t)k * n : nullptr;
            double u[2] = {0, 0};
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                C w[TUC], p[TUC], z[TUC];      // raw elements, widened at use
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    w[e] = p[e] = z[e] = C{};
                    if (qq < qb) {
                        w[e] = ws[qq];
                        p[e] = vk[qq];
                        if (vn) z[e] = vn[qq];
                    }
                }
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    if (qq >= qb) break;
                    cd wv = to_cd(w[e]);
                    csub_mul(wv, h, to_cd(p[e]));
                    store_c(ws[qq], wv);
                    const cd wr = rounded<C>(wv);
                    if (vn) cdot_acc(u[0], u[1], to_cd(z[e]), wr);
                    else u[0] += cabs2(wr);
                }
            }
            chunk_done<2>(a, s, c, u, parity ^ 1, lane);
        }
        for (int s = threadIdx.x; s < a.ns; s += blockDim.x) sact[s] = smode[s] == SLOT_ARNOLDI && k <= sstep[s] + 1;
        parity ^= 1;
        grid_barrier(a.bar, gridDim.x, a.err);
        load_totals(a, parity, 2, sact, tot);
        if (threadIdx.x < a.ns) {
            const int s = threadIdx.x;
            if (sact[s]) {
                sh_h[s] = cmk(tot[s][0], tot[s][1]);
                if (k == sstep[s] + 1) shn[s] = sqrt(tot[s][0]);
            }
        }
        __syncthreads();
    }
    // ---- classical Gram-Schmidt update: w -= sum_k h_k v_k (k ascending,
    // FP64 per element, one rounding to the storage precision), ||w||^2
    if (a.cgs) {
        cd *hs = ysm[threadIdx.x >> 5];
        for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
            const int s = sorder[q.it / NCH], c = q.it % NCH;
            if (smode[s] != SLOT_ARNOLDI) continue;
            const int i = sstep[s] + 1;
            const double *tt = a.ctm + (size_t)s * CGS_NV;
            __syncwarp();   // every lane is done with the previous item's coefficients
            for (int k = lane; k < i; k += 32) hs[k] = cmk(__ldcg(tt + 2 * k), __ldcg(tt + 2 * k + 1));
            __syncwarp();
            if (c == 0 && lane == 0)
                for (int k = 0; k < i; ++k) a.H[(size_t)s * ldh * a.m + (size_t)ldh * (i - 1) + k] = hs[k];
            const long long qa = c * ch.L, qb = min(n, qa + ch.L);
            C *ws = a.w + (size_t)swpos[s] * n;
            const C *Vs = a.V + (size_t)s * (a.m + 1) * n;
            double u[1] = {0.0};
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd acc[TUC];
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    acc[e] = qq < qb ? to_cd(ws[qq]) : cmk(0, 0);
                }
                for (int k = 0; k < i; ++k) {
                    const cd hk = hs[k];
                    const C *vk = Vs + (size_t)k * n;
                    C p[TUC];
#pragma unroll
                    for (int e = 0; e < TUC; ++e) {
                        const long long qq = q + 32 * e;
                        p[e] = qq < qb ? vk[qq] : C{};
                    }
#pragma unroll
                    for (int e = 0; e < TUC; ++e) csub_mul(acc[e], hk, to_cd(p[e]));
                }
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    if (qq >= qb) break;
                    store_c(ws[qq], acc[e]);
                    u[0] += cabs2(rounded<C>(acc[e]));
                }
            }
            __syncwarp();
            chunk_done<1>(a, s, c, u, parity ^ 1, lane);
        }
        for (int s = threadIdx.x; s < a.ns; s += blockDim.x) sact[s] = smode[s] == SLOT_ARNOLDI;
        parity ^= 1;
        grid_barrier(a.bar, gridDim.x, a.err);
        load_totals(a, parity, 1, sact, tot);
        if (threadIdx.x < a.ns && sact[threadIdx.x]) shn[threadIdx.x] = sqrt(tot[threadIdx.x][0]);
        __syncthreads();
    }
    // ---- conditional re-orthogonalisation (src/gmres_module.f90:251-258)
    for (int s = threadIdx.x; s < a.ns; s += blockDim.x)
        sro[s] = smode[s] == SLOT_ARNOLDI && snormav[s] + (double)0.001f * shn[s] == snormav[s];
    __syncthreads();
    int jmax = 0;
    for (int s = 0; s < a.ns; ++s)
        if (sro[s]) jmax = max(jmax, sstep[s] + 1);
    for (int j = 1; j <= jmax; ++j) {
        for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
            const int s = sorder[q.it / NCH], c = q.it % NCH;
            if (!sro[s] || j > sstep[s] + 1) continue;
            const long long qa = c * ch.L, qb = min(n, qa + ch.L);
            const C *vj = a.V + (size_t)s * (a.m + 1) * n + (size_t)(j - 1) * n;
            const C *ws = a.w + (size_t)swpos[s] * n;
            double u[2] = {0, 0};
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd z[TUC], w[TUC];
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    z[e] = w[e] = cmk(0, 0);
                    if (qq < qb) { z[e] = to_cd(vj[qq]); w[e] = to_cd(ws[qq]); }
                }
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    if (q + 32 * e >= qb) break;
                    cdot_acc(u[0], u[1], z[e], w[e]);
                }
            }
            chunk_done<2>(a, s, c, u, parity ^ 1, lane);
        }
        for (int s = threadIdx.x; s < a.ns; s += blockDim.x) sact[s] = sro[s] && j <= sstep[s] + 1;
        parity ^= 1;
        grid_barrier(a.bar, gridDim.x, a.err);
        load_totals(a, parity, 2, sact, tot);
        if (blockIdx.x == 0 && threadIdx.x < a.ns) {
            const int s = threadIdx.x;
            if (sact[s]) {
                const int i = sstep[s] + 1;
                cd *Hc = a.H + (size_t)s * ldh * a.m + (size_t)ldh * (i - 1);
                Hc[j - 1] = cadd(Hc[j - 1], cmk(tot[s][0], tot[s][1]));
            }
        }
        for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
            const int s = sorder[q.it / NCH], c = q.it % NCH;
            if (!sact[s]) continue;
            const cd hr = cmk(tot[s][0], tot[s][1]);
            const long long qa = c * ch.L, qb = min(n, qa + ch.L);
            const C *vj = a.V + (size_t)s * (a.m + 1) * n + (size_t)(j - 1) * n;
            C *ws = a.w + (size_t)swpos[s] * n;
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd w[TUC], p[TUC];
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    w[e] = p[e] = cmk(0, 0);
                    if (qq < qb) { w[e] = to_cd(ws[qq]); p[e] = to_cd(vj[qq]); }
                }
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    if (qq >= qb) break;
                    csub_mul(w[e], hr, p[e]);
                    store_c(ws[qq], w[e]);
                }
            }
        }
        __syncthreads();   // sact / tot are rewritten by the next round
    }
    if (jmax > 0) {
        for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
            const int s = sorder[q.it / NCH], c = q.it % NCH;
            if (!sro[s]) continue;
            const long long qa = c * ch.L, qb = min(n, qa + ch.L);
            const C *ws = a.w + (size_t)swpos[s] * n;
            double u[1] = {0};
            for (long long q = qa + lane; q < qb; q += 32 * TUC) {
                cd w[TUC];
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    const long long qq = q + 32 * e;
                    w[e] = qq < qb ? to_cd(ws[qq]) : cmk(0, 0);
                }
#pragma unroll
                for (int e = 0; e < TUC; ++e) {
                    if (q + 32 * e >= qb) break;
                    u[0] += cabs2(w[e]);
                }
            }
            chunk_done<1>(a, s, c, u, parity ^ 1, lane);
        }
        parity ^= 1;
        grid_barrier(a.bar, gridDim.x, a.err);
        load_totals(a, parity, 1, sro, tot);
        if (threadIdx.x < a.ns && sro[threadIdx.x]) shn[threadIdx.x] = sqrt(tot[threadIdx.x][0]);
        __syncthreads();
    }
    // ---- v_i = w / h(i+1,i) and the Givens update
    for (WorkQueue q(a.qctr + ph++, nitems, ch); q.next();) {
        const int s = sorder[q.it / NCH], c = q.it % NCH;
        if (smode[s] != SLOT_ARNOLDI) continue;
        const int i = sstep[s] + 1;
        const double hn = shn[s];
        const long long qa = c * ch.L, qb = min(n, qa + ch.L);
        const C *ws = a.w + (size_t)swpos[s] * n;
        C *vi = a.V + (size_t)s * (a.m + 1) * n + (size_t)i * n;
        for (long long q = qa + lane; q < qb; q += 32 * TUC) {
            cd w[TUC];
#pragma unroll
            for (int e = 0; e < TUC; ++e) {
                const long long qq = q + 32 * e;
                w[e] = qq < qb ? to_cd(ws[qq]) : cmk(0, 0);
            }
#pragma unroll
            for (int e = 0; e < TUC; ++e) {
                const long long qq = q + 32 * e;
                if (qq < qb) store_c(vi[qq], (hn != 0.0) ? cmk(w[e].x / hn, w[e].y / hn) : w[e]);
            }
        }
    }
    if (blockIdx.x == 0) {
        if (threadIdx.x < a.ns) sact[threadIdx.x] = snormav[threadIdx.x] + (double)0.001f * shn[threadIdx.x] == snormav[threadIdx.x];
        __syncthreads();
        givens_step(a, smode, sstep, shn, sact, ysm);
    }
    grid_barrier(a.bar, gridDim.x, a.err);
    cycle_end(a, ch, NCH, smode, ysm, sorder, a.qctr + ph);
}

// matvec input per slot, compacted: x at a cycle start, v_step during
// Arnoldi, into column mpos; slots without a matvec this tick have mpos < 0
template <typename C>
__global__ void k_stage(const Slot *slots, int ns, const C *V, const C *x, C *Xin, long long n, int m) {
    const int s = blockIdx.y;
    const int md = slots[s].mode, pos = slots[s].mpos;
    if (pos < 0) return;
    const C *src = md == SLOT_START ? x + (size_t)s * n : V + ((size_t)s * (m + 1) + slots[s].step) * n;
    C *dst = Xin + (size_t)pos * n;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        dst[q] = src[q];
}

// ---- mixed form: the FP64 outer refinement
// x64 += rho * d (the inner complex64 correction), for slots flagged upd
__global__ void k_outer_update(const Slot *slots, cd *x64, const cf *d32, long long n) {
    const int s = blockIdx.y;
    if (!slots[s].upd) return;
    const double rho = slots[s].rho;
    cd *xs = x64 + (size_t)s * n;
    const cf *ds = d32 + (size_t)s * n;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x) {
        const cd d = widen(ds[q]);
        xs[q] = cadd(xs[q], cmk(rho * d.x, rho * d.y));
    }
}

__global__ void k_stage_resid(const Slot *slots, const cd *x64, cd *Xin, long long n) {
    const int s = blockIdx.y;
    const int pos = slots[s].rpos;
    if (slots[s].mode != SLOT_RESID || pos < 0) return;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
        Xin[(size_t)pos * n + q] = x64[(size_t)s * n + q];
}

struct ResidArgs {
    Slot *slots;
    int ns;
    const cd *b64, *w64;   // rhs and A x, FP64
    cf *rhs32, *x32;       // inner right-hand side (r / rho) and initial guess (0)
    double *red;
    GridBarrier *bar;
    int *err;
    long long n;
    double tol;
    int max_outer;
};

// r = b - A x in FP64; stop when ||r||/||b|| < tol, else hand r/||r|| to an
// inner complex64 solve with a zero initial guess
__global__ void __launch_bounds__(BT) k_resid(ResidArgs a) {
    __shared__ double bsh[64];
    __shared__ double tot[NSMAX][4];
    __shared__ int smode[NSMAX];
    const long long n = a.n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long q0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    for (int s = threadIdx.x; s < a.ns; s += blockDim.x) smode[s] = a.slots[s].mode;
    __syncthreads();
    for (int s = 0; s < a.ns; ++s) {
        if (smode[s] != SLOT_RESID) continue;
        double v[2] = {0, 0};
        const cd *bs = a.b64 + (size_t)s * n, *ws = a.w64 + (size_t)max(a.slots[s].rpos, 0) * n;
        for (long long q = q0; q < n; q += stride) {
            const cd b = bs[q], r = csub(b, ws[q]);
            v[0] += cabs2(r);
            v[1] += cabs2(b);
        }
        block_sum<2>(v, bsh);
        if (threadIdx.x == 0) {
            double *p = a.red + (size_t)blockIdx.x * (NSMAX * 4) + s * 4;
            p[0] = v[0];
            p[1] = v[1];
        }
    }
    grid_barrier(a.bar, gridDim.x, a.err);
    {
        const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        for (int s = wp; s < a.ns; s += nw) {
            double acc[2] = {0, 0};
            for (int b = lane; b < (int)gridDim.x; b += 32) {
                const double *p = a.red + (size_t)b * (NSMAX * 4) + s * 4;
                acc[0] += __ldcg(p);
                acc[1] += __ldcg(p + 1);
            }
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
            if (lane == 0) { tot[s][0] = acc[0]; tot[s][1] = acc[1]; }
        }
        __syncthreads();
    }
    for (int s = 0; s < a.ns; ++s) {
        if (smode[s] != SLOT_RESID) continue;
        const double rho = sqrt(tot[s][0]);
        const double bn = a.slots[s].outer == 0 ? sqrt(tot[s][1]) : a.slots[s].b64;
        const double rel = bn > 0.0 ? rho / bn : 0.0;
        const bool stop = !(rel >= a.tol) || a.slots[s].outer >= a.max_outer;   // NaN stops too
        if (!stop) {
            const cd *bs = a.b64 + (size_t)s * n, *ws = a.w64 + (size_t)max(a.slots[s].rpos, 0) * n;
            cf *rs = a.rhs32 + (size_t)s * n, *xs = a.x32 + (size_t)s * n;
            for (long long q = q0; q < n; q += stride) {
                const cd r = csub(bs[q], ws[q]);
                rs[q] = make_float2((float)(r.x / rho), (float)(r.y / rho));
                xs[q] = make_float2(0.f, 0.f);
            }
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            Slot &sl = a.slots[s];
            if (sl.outer == 0) sl.b64 = bn;
            sl.relres = rel;
            sl.upd = 0;
            if (stop) {
                sl.mode = SLOT_DONE;
                sl.conv = rel < a.tol;
                sl.error = rel;
                if (!(rel == rel)) sl.status = SCD_NAN;
            } else {
                sl.rho = rho;
                sl.outer += 1;
                sl.mode = SLOT_START;
                sl.zero_x = 1;
                sl.cycle = 0;
                sl.step = 0;
                sl.conv = 0;
                sl.finish = 0;
            }
            if (*a.err) { sl.status = SCD_TIMEOUT; sl.mode = SLOT_DONE; }
        }
    }
}

}  // namespace

struct BatchBuffers {
    int ns = 0, m = 0, mixed = 0;
    long long n = 0;
    void *V = nullptr;                       // cd or cf bases
    cd *H = nullptr, *cs = nullptr, *sn = nullptr, *g = nullptr, *y = nullptr;
    void *x = nullptr, *rhs = nullptr, *Xin = nullptr, *W = nullptr;   // GMRES precision
    cd *x64 = nullptr, *b64 = nullptr, *Xin64 = nullptr, *W64 = nullptr;   // mixed: FP64 outer vectors
    Slot *slots = nullptr;
    Slot *h_slots = nullptr;
    double *red = nullptr;
    double *cpart = nullptr, *ctot = nullptr;
    double *cpm = nullptr, *ctm = nullptr;   // classical Gram-Schmidt reductions (opt-in)
    int *ccnt = nullptr;
    int grid = 0;                        // CTAs of the cooperative FP64 tick and residual kernels
    int grid_f = 0;                      // CTAs of the complex64 tick
};

static void free_bb(BatchBuffers &b) {
    void *p[] = {b.V, b.H, b.cs, b.sn, b.g, b.y, b.x, b.rhs, b.Xin, b.W, b.x64, b.b64, b.Xin64, b.W64,
                 b.slots, b.red, b.cpart, b.ctot, b.ccnt, b.cpm, b.ctm};
    for (void *q : p) if (q) cudaFree(q);
    if (b.h_slots) cudaFreeHost(b.h_slots);
    b = BatchBuffers();
}

void batch_free(scd_ctx *c) {
    if (!c->batch) return;
    free_bb(*(BatchBuffers *)c->batch);
    delete (BatchBuffers *)c->batch;
    c->batch = nullptr;
}

int batch_prepare(scd_ctx *c, int ns, int m, int mixed, BatchBuffers &b) {
    if (b.ns >= ns && b.m >= m && b.n == c->n && b.mixed == mixed && b.V && (!(mixed && c->cgs_on) || b.cpm))
        return SCD_OK;
    free_bb(b);
    const long long n = c->n;
    const size_t es = mixed ? sizeof(cf) : sizeof(cd);
    auto al = [&](void **p, size_t bytes, const char *what) -> int {
        if (cudaMalloc(p, bytes) != cudaSuccess) { cudaGetLastError(); return set_error(c, SCD_OOM, "batch %s (%zu bytes)", what, bytes); }
        return SCD_OK;
    };
    int rc;
    if ((rc = al(&b.V, es * (size_t)ns * (m + 1) * n, "Krylov bases"))) return rc;
    if ((rc = al((void **)&b.H, sizeof(cd) * (size_t)ns * (m + 1) * m, "H"))) return rc;
    if ((rc = al((void **)&b.cs, sizeof(cd) * (size_t)ns * (m + 1), "cs"))) return rc;
    if ((rc = al((void **)&b.sn, sizeof(cd) * (size_t)ns * (m + 1), "sn"))) return rc;
    if ((rc = al((void **)&b.g, sizeof(cd) * (size_t)ns * (m + 1), "g"))) return rc;
    if ((rc = al((void **)&b.y, sizeof(cd) * (size_t)ns * (m + 1), "y"))) return rc;
    if ((rc = al(&b.x, es * (size_t)ns * n, "x"))) return rc;
    if ((rc = al(&b.rhs, es * (size_t)ns * n, "rhs"))) return rc;
    if ((rc = al(&b.Xin, es * (size_t)ns * n, "Xin"))) return rc;
    if ((rc = al(&b.W, es * (size_t)ns * n, "W"))) return rc;
    if (mixed) {
        if ((rc = al((void **)&b.x64, sizeof(cd) * (size_t)ns * n, "x64"))) return rc;
        if ((rc = al((void **)&b.b64, sizeof(cd) * (size_t)ns * n, "b64"))) return rc;
        if ((rc = al((void **)&b.Xin64, sizeof(cd) * (size_t)ns * n, "Xin64"))) return rc;
        if ((rc = al((void **)&b.W64, sizeof(cd) * (size_t)ns * n, "W64"))) return rc;
    }
    if ((rc = al((void **)&b.slots, sizeof(Slot) * ns, "slots"))) return rc;
    if ((rc = al((void **)&b.cpart, sizeof(double) * (size_t)NSMAX * NCH * 4, "chunk partials"))) return rc;
    if ((rc = al((void **)&b.ctot, sizeof(double) * 2 * NSMAX * 4, "slot totals"))) return rc;
    if ((rc = al((void **)&b.ccnt, sizeof(int) * (NSMAX + QMAX), "chunk and work-queue counters"))) return rc;
    if (mixed && c->cgs_on) {
        if ((rc = al((void **)&b.cpm, sizeof(double) * (size_t)ns * NCH * CGS_NV, "Gram-Schmidt partials"))) return rc;
        if ((rc = al((void **)&b.ctm, sizeof(double) * (size_t)ns * CGS_NV, "Gram-Schmidt totals"))) return rc;
    }

    if (cudaMallocHost((void **)&b.h_slots, sizeof(Slot) * ns) != cudaSuccess) return set_error(c, SCD_OOM, "pinned slots");
    int per_sm = 0, per_sm2 = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tick<cd>, BT, 0);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_tick<cf>, BT, 0);
    per_sm = std::min(per_sm, per_sm2);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_resid, BT, 0);
    per_sm = std::min(per_sm, per_sm2);
    if (per_sm < 1) return set_error(c, SCD_CUDA_ERROR, "tick kernel cannot be resident");
    per_sm = std::min(per_sm, 2);
    b.grid = per_sm * c->nsm;
    {
        int per_f = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_f, k_tick<cf>, BT, 0);
        b.grid_f = std::max(1, std::min(per_f, SCD_TICK_MINB)) * c->nsm;
    }
    if ((rc = al((void **)&b.red, sizeof(double) * 2 * (size_t)b.grid * NSMAX * 4, "partials"))) return rc;
    b.ns = ns;
    b.m = m;
    b.n = n;
    b.mixed = mixed;
    return SCD_OK;
}

// The matvecs of one tick: columns [off_w, off_w + cnt[w]) of in/out (stride
// n) with operator ops[w].  The other contexts' matvecs run on their own
// streams, forked from and joined back to c's stream, so the operators of a
// sweep work concurrently.
template <typename C>
static void multi_matvec(scd_ctx *c, const std::vector<scd_ctx *> &ops, const C *in, C *out, const std::vector<int> &cnt) {
    const long long n = c->n;
    if (ops.size() == 1) {
        if (cnt[0] > 0) run_matvec(ops[0], in, out, cnt[0], nullptr);
        return;
    }
    if (!c->ev_fork) cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    cudaEventRecord(c->ev_fork, c->st);
    long long off = 0;
    for (size_t w = 0; w < ops.size(); ++w) {
        if (cnt[w] == 0) continue;
        scd_ctx *o = ops[w];
        if (o == c) {
            run_matvec(o, in + off * n, out + off * n, cnt[w], nullptr);
        } else {
            if (!o->ev_join) cudaEventCreateWithFlags(&o->ev_join, cudaEventDisableTiming);
            cudaStreamWaitEvent(o->st, c->ev_fork, 0);
            run_matvec(o, in + off * n, out + off * n, cnt[w], nullptr);
            cudaEventRecord(o->ev_join, o->st);
            cudaStreamWaitEvent(c->st, o->ev_join, 0);
        }
        off += cnt[w];
    }
}

template <typename C>
static int launch_tick(scd_ctx *c, BatchBuffers &bb, int ns, int nact, int m, int cycles, double tol, int mixed,
                       const std::vector<scd_ctx *> &ops, const std::vector<int> &cnt) {
    TickArgs<C> a;
    a.slots = bb.slots; a.ns = ns; a.V = (C *)bb.V; a.H = bb.H; a.cs = bb.cs; a.sn = bb.sn; a.g = bb.g; a.y = bb.y;
    a.x = (C *)bb.x; a.rhs = (C *)bb.rhs; a.w = (C *)bb.W; a.red = bb.red; a.bar = c->d_bar; a.err = c->d_err;
    a.cpart = bb.cpart; a.ctot = bb.ctot; a.ccnt = bb.ccnt; a.qctr = bb.ccnt + NSMAX;
    a.n = c->n; a.m = m; a.max_cycles = cycles; a.tol = tol; a.mixed = mixed;
    a.cgs = (mixed && c->cgs_on && bb.cpm) ? 1 : 0;
    a.cpm = bb.cpm; a.ctm = bb.ctm;
    const long long n = c->n;
    if (nact > 0) {
        k_stage<C><<<dim3(std::min<long long>((n + 255) / 256, 1024), ns), 256, 0, c->st>>>(bb.slots, ns, (C *)bb.V,
                                                                                           (C *)bb.x, (C *)bb.Xin, n, m);
        multi_matvec<C>(c, ops, (const C *)bb.Xin, (C *)bb.W, cnt);
    }
    NvtxRange r("arnoldi tick");
    void *args[] = {&a};
    cudaMemsetAsync(bb.ccnt, 0, sizeof(int) * (NSMAX + QMAX), c->st);
    const int grid = std::is_same<C, cf>::value ? bb.grid_f : bb.grid;
    cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_tick<C>, dim3(grid), dim3(BT), args, 0, c->st);
    c->launches += 2;
    return check_cuda(c, e, "tick launch");
}

// Solve columns `rhs_cols` (device pointers to slot-ordered right-hand
// sides) with up to `ns` slots; FP64 solutions go to X[j] (stride n).
// precision 0: restarted GMRES(m) in complex128 to `tol` (the reference's
// algorithm); 1: FP64 iterative refinement to `tol` around complex64
// GMRES(m) inner solves to `inner_tol`, at most `max_outer` outer steps.
int batch_run(scd_ctx *c, ColumnSource &src, double tol, int m, int cycles, int ns, int precision, double inner_tol,
              int max_outer, const std::vector<scd_ctx *> *ops_in) {
    NvtxRange range(precision == SCD_PREC_MIXED ? "batch solve (mixed)" : "batch solve (fp64)");
    if (!c->batch) c->batch = new BatchBuffers();
    BatchBuffers &bb = *(BatchBuffers *)c->batch;
    const int mixed = precision == SCD_PREC_MIXED ? 1 : 0;
    if (m < 1 || m > SCD_M_MAX) return set_error(c, SCD_BAD_ARG, "m = %d outside 1..%d", m, SCD_M_MAX);
    if (ns > NSMAX) ns = NSMAX;
    if (ns < 1) ns = 1;
    const std::vector<scd_ctx *> ops = ops_in && !ops_in->empty() ? *ops_in : std::vector<scd_ctx *>{c};
    const int nops = (int)ops.size();
    for (scd_ctx *o : ops)
        if (o->n != c->n || o->dev != c->dev)
            return set_error(c, SCD_BAD_ARG, "operators of one batch need the same device and unknowns");
    int rc = batch_prepare(c, ns, m, mixed, bb);
    if (rc) return rc;
    // work buffers of operator w for nm complex64 and nr FP64 right-hand
    // sides (mixed), or nr FP64 ones: one operator is sized for every slot up
    // front; several grow to the next power of two of their columns in flight
    auto prepare = [&](int w, int nm, int nr) -> int {
        scd_ctx *o = ops[w];
        int r;
        if (mixed) {
            r = ensure_single(o);
            if (!r && nm > 0) r = ensure_work_single(o, nm);
            if (!r) r = ensure_work(o, std::max(nr, 1));
        } else {
            r = ensure_work(o, std::max(nr, 1));
        }
        return r == SCD_OK || o == c ? r : set_error(c, r, "operator of the batch: %s", o->err.c_str());
    };
    auto grown = [ns](int v) { int p = 1; while (p < v) p <<= 1; return std::min(p, ns); };
    if (nops == 1 && (rc = prepare(0, ns, ns))) return rc;
    if (mixed && (rc = ensure_work(c, ns))) return rc;
    std::vector<char> live(nops, nops == 1 ? 1 : 0);   // operators holding work buffers
    std::vector<int> sop(ns, 0), cnt_m(nops, 0), cnt_r(nops, 0);   // slot operators, columns per operator
    if (!c->d_bar) {
        if (cudaMalloc(&c->d_bar, sizeof(GridBarrier)) != cudaSuccess || cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess)
            return set_error(c, SCD_OOM, "barrier");
    }
    cudaMemsetAsync(c->d_bar, 0, sizeof(GridBarrier), c->st);
    cudaMemsetAsync(c->d_err, 0, sizeof(int), c->st);
    const long long n = c->n;
    Slot *hs = bb.h_slots;
    std::memset(hs, 0, sizeof(Slot) * ns);
    for (int s = 0; s < ns; ++s) { hs[s].mode = SLOT_FREE; hs[s].col = -1; }
    std::vector<cd *> xout(ns, nullptr);        // where each slot's solution goes
    const double gm_tol = mixed ? inner_tol : tol;
    while (true) {
        bool inner = false, resid = false, upd = false;
        int busy = 0;
        for (int s = 0; s < ns; ++s) {
            if (hs[s].mode == SLOT_DONE) {
                const cd *xs = mixed ? bb.x64 + (size_t)s * n : (const cd *)bb.x + (size_t)s * n;
                cudaMemcpyAsync(xout[s], xs, sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->st);
                c->n_arn += hs[s].iters;
                c->n_matvec += hs[s].iters + hs[s].cycle;
                src.finished(hs[s].col, hs[s].iters, hs[s].conv, hs[s].status, mixed ? hs[s].relres : hs[s].error);
                std::memset(&hs[s], 0, sizeof(Slot));
                hs[s].mode = SLOT_FREE;
                hs[s].col = -1;
                xout[s] = nullptr;
            }
            const cd *rhs = nullptr;
            int tag = -1;
            if (hs[s].mode == SLOT_FREE && src.next(&rhs, &xout[s], &tag)) {
                std::memset(&hs[s], 0, sizeof(Slot));
                if (mixed) {
                    cudaMemcpyAsync(bb.b64 + (size_t)s * n, rhs, sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->st);
                    cudaMemcpyAsync(bb.x64 + (size_t)s * n, rhs, sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->st);
                    hs[s].mode = SLOT_RESID;
                } else {
                    cudaMemcpyAsync((cd *)bb.rhs + (size_t)s * n, rhs, sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->st);
                    cudaMemcpyAsync((cd *)bb.x + (size_t)s * n, rhs, sizeof(cd) * n, cudaMemcpyDeviceToDevice, c->st);
                    hs[s].mode = SLOT_START;
                }
                hs[s].col = tag;
                sop[s] = nops > 1 ? src.op_of(tag) : 0;
                if (sop[s] < 0 || sop[s] >= nops) return set_error(c, SCD_BAD_ARG, "column %d: operator %d", tag, sop[s]);
            }
            if (hs[s].mode == SLOT_INNER_DONE) { hs[s].mode = SLOT_RESID; hs[s].upd = 1; upd = true; }
            if (hs[s].mode == SLOT_RESID) resid = true;
            if (hs[s].mode == SLOT_START || hs[s].mode == SLOT_ARNOLDI) inner = true;
            if (hs[s].mode != SLOT_FREE) ++busy;
        }
        if (busy == 0) {
            // every slot idle: the source may still bring columns (a served pool)
            if ((rc = check_cuda(c, cudaStreamSynchronize(c->st), "batch idle"))) return rc;
            if (!src.wait_more()) break;
            continue;
        }
        if (!inner && !resid) return set_error(c, SCD_CUDA_ERROR, "batch solver stalled");
        // compacted matvec columns: only slots that need A x this tick, grouped
        // by operator
        int nact = 0, nres = 0;
        for (int s = 0; s < ns; ++s) hs[s].mpos = hs[s].rpos = -1;
        for (int w = 0; w < nops; ++w) {
            cnt_m[w] = cnt_r[w] = 0;
            for (int s = 0; s < ns; ++s) {
                if (sop[s] != w) continue;
                if (hs[s].mode == SLOT_RESID) { hs[s].rpos = nres++; ++cnt_r[w]; }
                if ((hs[s].mode == SLOT_START && !hs[s].zero_x) || hs[s].mode == SLOT_ARNOLDI) {
                    hs[s].mpos = nact++;
                    ++cnt_m[w];
                }
            }
        }
        if (nops > 1) {
            for (int w = 0; w < nops; ++w) {
                const int nm = mixed ? cnt_m[w] : 0, nr = mixed ? cnt_r[w] : cnt_m[w];
                if (nm == 0 && nr == 0) continue;
                if ((rc = prepare(w, nm ? grown(nm) : 0, nr ? grown(nr) : 0))) return rc;
                live[w] = 1;
            }
        }
        cudaMemcpyAsync(bb.slots, hs, sizeof(Slot) * ns, cudaMemcpyHostToDevice, c->st);
        if (mixed) {
            const dim3 g2(std::min<long long>((n + 255) / 256, 1024), ns);
            if (upd) k_outer_update<<<g2, 256, 0, c->st>>>(bb.slots, bb.x64, (const cf *)bb.x, n);
            if (resid) {
                k_stage_resid<<<g2, 256, 0, c->st>>>(bb.slots, bb.x64, bb.Xin64, n);
                multi_matvec<cd>(c, ops, (const cd *)bb.Xin64, bb.W64, cnt_r);
                ResidArgs ra;
                ra.slots = bb.slots; ra.ns = ns; ra.b64 = bb.b64; ra.w64 = bb.W64; ra.rhs32 = (cf *)bb.rhs;
                ra.x32 = (cf *)bb.x; ra.red = bb.red; ra.bar = c->d_bar; ra.err = c->d_err; ra.n = n; ra.tol = tol;
                ra.max_outer = max_outer;
                void *args[] = {&ra};
                cudaError_t e = cudaLaunchCooperativeKernel((const void *)k_resid, dim3(bb.grid), dim3(BT), args, 0, c->st);
                c->launches += 3 + (upd ? 1 : 0);
                if ((rc = check_cuda(c, e, "residual launch"))) return rc;
            }
            if ((rc = launch_tick<cf>(c, bb, ns, nact, m, cycles, gm_tol, 1, ops, cnt_m))) return rc;
        } else {
            if ((rc = launch_tick<cd>(c, bb, ns, nact, m, cycles, gm_tol, 0, ops, cnt_m))) return rc;
        }
        cudaMemcpyAsync(hs, bb.slots, sizeof(Slot) * ns, cudaMemcpyDeviceToHost, c->st);
        if ((rc = check_cuda(c, cudaStreamSynchronize(c->st), "tick"))) return rc;
        for (int s = 0; s < ns; ++s)
            if (hs[s].status == SCD_TIMEOUT) return set_error(c, SCD_TIMEOUT, "grid barrier wait expired in the batch solver");
        // operators with no column in a slot and none left to hand out give
        // their work buffers back (every kernel of theirs has finished: the
        // stream synchronisation above follows the join of their streams)
        for (int w = 0; w < nops && nops > 1; ++w) {
            if (!live[w] || ops[w] == c || src.op_pending(w)) continue;
            bool used = false;
            for (int s = 0; s < ns && !used; ++s) used = hs[s].mode != SLOT_FREE && sop[s] == w;
            if (!used) {
                release_work(ops[w]);
                live[w] = 0;
            }
        }
    }
    return check_cuda(c, cudaStreamSynchronize(c->st), "batch end");
}

namespace {
// the columns of one call, in order
struct ArraySource final : ColumnSource {
    scd_ctx *c;
    int ncol, next_col = 0;
    const cd *const *rhs;
    cd *X;
    int *iters, *conv, *status;
    double *relres;
    int worst = SCD_OK;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::vector<double> t_in;
    double now_ms() const {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    bool next(const cd **r, cd **xout, int *tag) override {
        if (next_col >= ncol) return false;
        *r = rhs[next_col];
        *xout = X + (size_t)next_col * c->n;
        *tag = next_col;
        t_in[next_col] = now_ms();
        ++next_col;
        return true;
    }
    void finished(int col, int it, int cv, int st, double rr) override {
        if (iters) iters[col] = it;
        if (conv) conv[col] = cv;
        if (status) status[col] = st;
        if (relres) relres[col] = rr;
        c->col_latency_ms[col] = now_ms() - t_in[col];
        if (st != SCD_OK) worst = st;
        else if (!cv && worst == SCD_OK) worst = SCD_NOT_CONVERGED;
    }
};
}  // namespace

int batch_solve(scd_ctx *c, int ncol, const cd *const *rhs_cols, cd *X, double tol, int m, int cycles, int ns,
                int *iters, int *conv_out, int *status_out, double *relres_out, int precision, double inner_tol,
                int max_outer) {
    ArraySource src;
    src.c = c;
    src.ncol = ncol;
    src.rhs = rhs_cols;
    src.X = X;
    src.iters = iters;
    src.conv = conv_out;
    src.status = status_out;
    src.relres = relres_out;
    src.t_in.assign(ncol, 0.0);
    c->col_latency_ms.assign(ncol, 0.0);
    const int rc = batch_run(c, src, tol, m, cycles, std::min(ns, ncol), precision, inner_tol, max_outer);
    if (rc) return rc;
    return src.worst;
}
