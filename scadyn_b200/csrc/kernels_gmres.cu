// Restarted GMRES on the device, restating gmres (src/gmres_module.f90:180-325):
// x0 = rhs, modified Gram-Schmidt with the conditional re-orthogonalisation
// test `normav + 0.001*normav2 == normav`, complex Givens rotations, stop on
// |g(i+1)|/||rhs|| < tol, y = H(1:i,1:i)^-1 g(1:i) and x += V y.
//
// Each Arnoldi step is one cooperative kernel: the i dot products of MGS are
// sequential (each needs the updated w), so every one is a grid-wide
// reduction.  Partial sums are written per CTA, a bounded grid barrier is
// crossed, and every CTA adds the partials in the same fixed order, so all
// CTAs hold bit-identical coefficients and the run is deterministic.  The
// next dot product is fused into the axpy of the current one, giving one
// barrier per MGS term.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "ctx.h"

namespace {

constexpr int GT = 256;   // threads per CTA of the cooperative kernels

struct GmArgs {
    cd *V;            // (m+1) columns of length n
    cd *H;            // (m+1) x m, column-major
    cd *cs, *sn, *g;  // m+1
    cd *w;            // A v
    cd *x;            // iterate
    const cd *rhs;
    double *red;      // [2][grid][4]
    GridBarrier *bar;
    int *err;
    GmresState *st;
    long long n;
    int m;
    double tol;
};

__device__ __forceinline__ void write_partial(double *red, int parity, int nv, const double *v) {
    if (threadIdx.x == 0) {
        double *p = red + ((size_t)parity * gridDim.x + blockIdx.x) * 4;
        for (int q = 0; q < nv; ++q) p[q] = v[q];
    }
}

// every CTA sums the per-CTA partials in CTA order (deterministic); L2 reads
__device__ __forceinline__ void read_total(const double *red, int parity, int nv, double *out, double *sh) {
    // warp 0 reduces with a fixed tree: lane l sums CTAs l, l+32, ... in order
    if (threadIdx.x < 32) {
        double acc[4] = {0, 0, 0, 0};
        for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) {
            const double *p = red + ((size_t)parity * gridDim.x + b) * 4;
            for (int q = 0; q < nv; ++q) acc[q] += __ldcg(p + q);
        }
        for (int q = 0; q < nv; ++q) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
        }
        if (threadIdx.x == 0)
            for (int q = 0; q < nv; ++q) sh[q] = acc[q];
    }
    __syncthreads();
    for (int q = 0; q < nv; ++q) out[q] = sh[q];
    __syncthreads();
}

// r = rhs - w; beta = ||r||; V0 = r / beta; g = (beta, 0, ...); first cycle: b_norm
__global__ void __launch_bounds__(GT) k_cycle_init(GmArgs a, int first) {
    __shared__ double sh[64];
    __shared__ double tot[4];
    GmresState *st = a.st;
    if (st->done) return;
    const long long stride = (long long)gridDim.x * blockDim.x;
    double v[2] = {0.0, 0.0};
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.n; q += stride) {
        cd b = a.rhs[q];
        cd r = csub(b, a.w[q]);
        a.V[q] = r;
        v[0] += cabs2(r);
        v[1] += cabs2(b);
    }
    block_sum<2>(v, sh);
    write_partial(a.red, 0, 2, v);
    grid_barrier(a.bar, gridDim.x, a.err);
    double t[2];
    read_total(a.red, 0, 2, t, tot);
    const double beta = sqrt(t[0]);
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.n; q += stride) {
        cd r = a.V[q];
        a.V[q] = cmk(r.x / beta, r.y / beta);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int i = 0; i <= a.m; ++i) a.g[i] = cmk(0, 0);
        a.g[0] = cmk(beta, 0.0);
        st->beta = beta;
        if (first) st->b_norm = sqrt(t[1]);
        st->step = 0;
        if (first && st->b_norm == 0.0) { st->error = 0.0; st->done = 1; }   // rhs = 0: x0 = 0 is exact
        else if (!(beta == beta)) { st->status = SCD_NAN; st->done = 1; }
    }
}

// One Arnoldi step i (1-based): MGS of w = A v_{i-1} against v_0..v_{i-1},
// optional re-orthogonalisation, v_i = w / h(i+1,i), Givens update.
__global__ void __launch_bounds__(GT) k_arnoldi(GmArgs a, int i) {
    __shared__ double sh[64];
    __shared__ double tot[4];
    GmresState *st = a.st;
    if (st->done) return;
    const long long n = a.n;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long q0 = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int ldh = a.m + 1;
    cd *Hc = a.H + (size_t)ldh * (i - 1);
    int parity = 0;

    // ||w|| and <v_0, w>
    double v[3] = {0, 0, 0};
    for (long long q = q0; q < n; q += stride) {
        cd w = a.w[q], z = a.V[q];
        v[0] += cabs2(w);
        cdot_acc(v[1], v[2], z, w);
    }
    block_sum<3>(v, sh);
    write_partial(a.red, parity, 3, v);
    grid_barrier(a.bar, gridDim.x, a.err);
    double t[3];
    read_total(a.red, parity, 3, t, tot);
    const double normav = sqrt(t[0]);
    cd h = cmk(t[1], t[2]);
    // modified Gram-Schmidt: subtract h_k v_{k-1}, fused with the next dot
    for (int k = 1; k <= i; ++k) {
        if (blockIdx.x == 0 && threadIdx.x == 0) Hc[k - 1] = h;
        const cd *vk = a.V + (size_t)(k - 1) * n;
        const cd *vn = (k < i) ? a.V + (size_t)k * n : nullptr;
        double u[2] = {0, 0};
        for (long long q = q0; q < n; q += stride) {
            cd w = a.w[q];
            cd p = vk[q];
            csub_mul(w, h, p);
            a.w[q] = w;
            if (vn) {
                cd z = vn[q];
                cdot_acc(u[0], u[1], z, w);
            } else {
                u[0] += cabs2(w);
            }
        }
        parity ^= 1;
        block_sum<2>(u, sh);
        write_partial(a.red, parity, 2, u);
        grid_barrier(a.bar, gridDim.x, a.err);
        double tt[2];
        read_total(a.red, parity, 2, tt, tot);
        h = cmk(tt[0], tt[1]);   // last iteration: (||w||^2, 0)
    }
    double hn = sqrt(h.x);
    const double normav2 = hn;
    if (normav + (double)0.001f * normav2 == normav) {
        // re-orthogonalise against v_0 .. v_{i-1} (src/gmres_module.f90:251-258)
        for (int j = 1; j <= i; ++j) {
            const cd *vj = a.V + (size_t)(j - 1) * n;
            double u[2] = {0, 0};
            for (long long q = q0; q < n; q += stride) {
                cd z = vj[q], w = a.w[q];
                cdot_acc(u[0], u[1], z, w);
            }
            parity ^= 1;
            block_sum<2>(u, sh);
            write_partial(a.red, parity, 2, u);
            grid_barrier(a.bar, gridDim.x, a.err);
            double tt[2];
            read_total(a.red, parity, 2, tt, tot);
            const cd hr = cmk(tt[0], tt[1]);
            if (blockIdx.x == 0 && threadIdx.x == 0) Hc[j - 1] = cadd(Hc[j - 1], hr);
            for (long long q = q0; q < n; q += stride) {
                cd w = a.w[q], p = vj[q];
                csub_mul(w, hr, p);
                a.w[q] = w;
            }
        }
        double u[1] = {0};
        for (long long q = q0; q < n; q += stride) u[0] += cabs2(a.w[q]);
        parity ^= 1;
        block_sum<1>(u, sh);
        write_partial(a.red, parity, 1, u);
        grid_barrier(a.bar, gridDim.x, a.err);
        double tt[1];
        read_total(a.red, parity, 1, tt, tot);
        hn = sqrt(tt[0]);
        if (blockIdx.x == 0 && threadIdx.x == 0) st->reorth += 1;
    }
    cd *vi = a.V + (size_t)i * n;
    for (long long q = q0; q < n; q += stride) {
        cd w = a.w[q];
        vi[q] = (hn != 0.0) ? cmk(w.x / hn, w.y / hn) : w;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Hc[i] = cmk(hn, 0.0);
        // previous rotations (src/gmres_module.f90:266-272)
        for (int k = 1; k <= i - 1; ++k) {
            cd c = a.cs[k - 1], s = a.sn[k - 1];
            cd tmp = csub(cmul(c, Hc[k - 1]), cmul(s, Hc[k]));
            Hc[k] = cadd(cmul(s, Hc[k - 1]), cmul(cconj(c), Hc[k]));
            Hc[k - 1] = tmp;
        }
        const double nu = sqrt(cabs2(Hc[i - 1]) + cabs2(Hc[i]));
        if (nu != 0.0) {
            cd c = cconj(cmk(Hc[i - 1].x / nu, Hc[i - 1].y / nu));
            cd s = cmk(-Hc[i].x / nu, -Hc[i].y / nu);
            a.cs[i - 1] = c;
            a.sn[i - 1] = s;
            Hc[i - 1] = csub(cmul(c, Hc[i - 1]), cmul(s, Hc[i]));
            Hc[i] = cmk(0, 0);
            cd t1 = a.g[i - 1], t2 = a.g[i];
            a.g[i - 1] = csub(cmul(c, t1), cmul(s, t2));
            a.g[i] = cadd(cmul(s, t1), cmul(cconj(c), t2));
        }
        const double error = sqrt(cabs2(a.g[i])) / st->b_norm;
        st->error = error;
        st->step = i;
        st->iters += 1;
        if (error < a.tol) { st->conv_step = i; st->done = 1; }
        if (!(error == error)) { st->status = SCD_NAN; st->done = 1; }
        if (*a.err) { st->status = SCD_TIMEOUT; st->done = 1; }
    }
}

// y = H(1:k,1:k)^-1 g(1:k) by back substitution on the rotated (upper
// triangular) H, then x += V(:,1:k) y.  k = the converged step, or the
// steps of the cycle.
__global__ void __launch_bounds__(GT) k_update(GmArgs a) {
    extern __shared__ cd ysh[];
    GmresState *st = a.st;
    const int kdim = st->conv_step ? st->conv_step : st->step;
    if (kdim == 0 || st->status != SCD_OK) return;
    const int ldh = a.m + 1;
    if (threadIdx.x == 0) {
        for (int r = kdim - 1; r >= 0; --r) {
            cd s = a.g[r];
            for (int c = r + 1; c < kdim; ++c) s = csub(s, cmul(a.H[r + (size_t)ldh * c], ysh[c]));
            ysh[r] = cdiv(s, a.H[r + (size_t)ldh * r]);
        }
    }
    __syncthreads();
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < a.n; q += stride) {
        cd s = cmk(0, 0);
        for (int c = 0; c < kdim; ++c) cfma(s, a.V[(size_t)c * a.n + q], ysh[c]);
        a.x[q] = cadd(a.x[q], s);
    }
}

__global__ void k_state_init(GmresState *st, GridBarrier *bar, int *err) {
    memset(st, 0, sizeof(GmresState));
    bar->count = 0;
    bar->gen = 0;
    *err = 0;
}

__global__ void k_state_cycle(GmresState *st) {
    if (!st->done) { st->step = 0; }
}

GmArgs make_args(scd_ctx *c, const cd *rhs, cd *x, double tol) {
    GmArgs a;
    a.V = c->d_V; a.H = c->d_H; a.cs = c->d_cs; a.sn = c->d_sn; a.g = c->d_g;
    a.w = c->d_w; a.x = x; a.rhs = rhs; a.red = c->d_red; a.bar = c->d_bar; a.err = c->d_err;
    a.st = c->d_state; a.n = c->n; a.m = c->gm_m; a.tol = tol;
    return a;
}

}  // namespace

int gmres_prepare(scd_ctx *c, int m) {
    if (c->gm_m >= m && c->d_V) return SCD_OK;
    cudaFree(c->d_V); cudaFree(c->d_H); cudaFree(c->d_cs); cudaFree(c->d_sn); cudaFree(c->d_g);
    c->d_V = c->d_H = c->d_cs = c->d_sn = c->d_g = nullptr;
    c->gm_m = m;
    cudaError_t e = cudaMalloc(&c->d_V, sizeof(cd) * (size_t)(m + 1) * c->n);
    if (e != cudaSuccess) { c->gm_m = 0; return set_error(c, SCD_OOM, "GMRES basis (%d x %lld)", m + 1, c->n); }
    if (cudaMalloc(&c->d_H, sizeof(cd) * (size_t)(m + 1) * m) != cudaSuccess ||
        cudaMalloc(&c->d_cs, sizeof(cd) * (m + 1)) != cudaSuccess ||
        cudaMalloc(&c->d_sn, sizeof(cd) * (m + 1)) != cudaSuccess ||
        cudaMalloc(&c->d_g, sizeof(cd) * (m + 1)) != cudaSuccess)
        return set_error(c, SCD_OOM, "GMRES small buffers");
    if (!c->d_w && cudaMalloc(&c->d_w, sizeof(cd) * c->n) != cudaSuccess) return set_error(c, SCD_OOM, "GMRES w");
    if (!c->d_state) {
        if (cudaMalloc(&c->d_state, sizeof(GmresState)) != cudaSuccess ||
            cudaMalloc(&c->d_bar, sizeof(GridBarrier)) != cudaSuccess ||
            cudaMalloc(&c->d_err, sizeof(int)) != cudaSuccess ||
            cudaMallocHost(&c->h_state, sizeof(GmresState)) != cudaSuccess)
            return set_error(c, SCD_OOM, "GMRES state");
    }
    if (!c->coop_grid) {
        int per_sm = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_arnoldi, GT, 0);
        int per_sm2 = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, k_cycle_init, GT, 0);
        per_sm = per_sm < per_sm2 ? per_sm : per_sm2;
        if (per_sm < 1) return set_error(c, SCD_CUDA_ERROR, "cooperative GMRES kernels cannot be resident");
        per_sm = per_sm > 2 ? 2 : per_sm;
        c->coop_grid = per_sm * c->nsm;
        if (cudaMalloc(&c->d_red, sizeof(double) * 2 * 4 * (size_t)c->coop_grid) != cudaSuccess)
            return set_error(c, SCD_OOM, "GMRES reduction buffer");
    }
    return check_cuda(c, cudaGetLastError(), "gmres_prepare");
}

static int launch_coop(scd_ctx *c, const void *fn, void **args) {
    cudaError_t e = cudaLaunchCooperativeKernel(fn, dim3(c->coop_grid), dim3(GT), args, 0, c->st);
    c->launches += 1;
    return check_cuda(c, e, "cooperative launch");
}

int gmres_solve(scd_ctx *c, const cd *d_rhs, cd *d_x, double tol, int m, int cycles, int *iters, double *relres) {
    int rc = gmres_prepare(c, m);
    if (rc) return rc;
    GmArgs a = make_args(c, d_rhs, d_x, tol);
    a.m = m;
    k_state_init<<<1, 1, 0, c->st>>>(c->d_state, c->d_bar, c->d_err);
    cudaMemcpyAsync(d_x, d_rhs, sizeof(cd) * c->n, cudaMemcpyDeviceToDevice, c->st);   // x0 = rhs
    const int check_every = 4;
    bool done = false;
    int cycles_run = 0;
    for (int cyc = 0; cyc < cycles && !done; ++cyc) {
        ++cycles_run;
        run_matvec(c, d_x, c->d_w, 1, nullptr);
        int first = cyc == 0;
        void *args_init[] = {&a, &first};
        if ((rc = launch_coop(c, (const void *)k_cycle_init, args_init))) return rc;
        for (int i = 1; i <= m; ++i) {
            run_matvec(c, c->d_V + (size_t)(i - 1) * c->n, c->d_w, 1, &c->d_state->done);
            void *args_arn[] = {&a, &i};
            if ((rc = launch_coop(c, (const void *)k_arnoldi, args_arn))) return rc;
            if (i % check_every == 0 || i == m) {
                cudaMemcpyAsync(c->h_state, c->d_state, sizeof(GmresState), cudaMemcpyDeviceToHost, c->st);
                if ((rc = check_cuda(c, cudaStreamSynchronize(c->st), "gmres step"))) return rc;
                if (c->h_state->done) break;
            }
        }
        k_update<<<c->nsm * 4, GT, sizeof(cd) * m, c->st>>>(a);
        k_state_cycle<<<1, 1, 0, c->st>>>(c->d_state);
        c->launches += 2;
        cudaMemcpyAsync(c->h_state, c->d_state, sizeof(GmresState), cudaMemcpyDeviceToHost, c->st);
        if ((rc = check_cuda(c, cudaStreamSynchronize(c->st), "gmres cycle"))) return rc;
        done = c->h_state->done != 0;
    }
    if (iters) *iters = c->h_state->iters;
    if (relres) *relres = c->h_state->error;
    c->n_arn += c->h_state->iters;
    c->n_matvec += c->h_state->iters + cycles_run;
    if (c->h_state->status == SCD_TIMEOUT) return set_error(c, SCD_TIMEOUT, "grid barrier wait expired in GMRES");
    if (c->h_state->status == SCD_NAN) return set_error(c, SCD_NAN, "non-finite residual in GMRES");
    if (!(c->h_state->error < tol)) return SCD_NOT_CONVERGED;
    return SCD_OK;
}
