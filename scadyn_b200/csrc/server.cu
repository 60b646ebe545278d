// Request loop (include/scadyn_server.h) over resident operator pools.
//
// A pool is one device context (scd_ctx: grid, Green octant, projectors,
// near-zone tiles, batched-solver workspace) for one operator key -- the
// mesh and its permittivities, the wavenumber, the cell size, the near-zone
// storage and the solve options -- with its own worker thread and CUDA
// stream.  Its worker builds the operator once and then runs the batched
// solver on a queue of columns that every request of that key feeds: a
// request that arrives while the pool is solving has its incident columns
// built on the device and queued at once, and they take slots as the
// running columns finish (continuous batching across requests).  When its
// requests are done the pool stays resident, so a later request of the same
// key starts solving without a rebuild; idle pools are evicted, least
// recently used first, when a new pool needs their memory.
//
// Admission is by the HBM budget: a new pool needs its estimated operator
// and workspace bytes, every request its incident columns and solutions
// (2 x 3T x 2nm complex128); max_running (0 = no limit but the budget)
// bounds the pools solving at once.  Kernels of different pools overlap on
// the GPU.  A column's arithmetic does not depend on its batch, so a
// request's T is bit-identical alone, in a mix, and in a shared pool.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/scadyn_server.h"
#include "ctx.h"

namespace {

using clk = std::chrono::steady_clock;

int ncols_of(int Nmax) { return 2 * ((Nmax + 1) * (Nmax + 1) - 1); }

// FNV-1a over the mesh arrays: the pool key's fingerprint of a geometry
uint64_t fnv(uint64_t h, const void *p, size_t bytes) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < bytes; ++i) {
        h ^= b[i];
        h *= 1099511628211ull;
    }
    return h;
}

struct PoolKey {
    uint64_t mesh = 0;
    int32_t Nv = 0, T = 0, storage_prec = 0;
    double k = 0, grid_size = 0;
    scd_solve_opts opts{};
    bool operator==(const PoolKey &o) const {
        return mesh == o.mesh && Nv == o.Nv && T == o.T && storage_prec == o.storage_prec && k == o.k &&
               grid_size == o.grid_size && std::memcmp(&opts, &o.opts, sizeof opts) == 0;
    }
};

struct Pool;

struct Req {
    int64_t id = 0;
    int32_t Nv = 0, T = 0;
    std::vector<double> coord;
    std::vector<int32_t> etopol;
    std::vector<scd_c128> param;
    double k = 0, grid_size = 0;
    int32_t Nmax = 0, storage_prec = SCD_STORE_C64;
    scd_solve_opts opts{};
    PoolKey key;
    int64_t est_req = 0;          // the request's own device bytes
    int64_t est_pool = 0;         // a new pool's bytes for it
    int32_t state = SCD_REQ_QUEUED, status = SCD_OK;
    bool consumed = false;        // the result has been read
    std::string err;
    clk::time_point t_submit, t_done;
    std::vector<scd_c128> Tm;
    std::vector<int32_t> iters;
    // while solving (owned by the pool's worker)
    std::shared_ptr<Pool> pool;
    cd *d_mat = nullptr, *d_X = nullptr;
    int cols_done = 0;
    int worst = SCD_OK;
};

struct Pool {
    PoolKey key;
    int64_t est = 0;                       // operator and workspace bytes
    scd_ctx *ctx = nullptr;
    std::thread worker;
    std::deque<int64_t> joining;           // admitted requests the worker has not set up yet
    std::deque<std::pair<int64_t, int>> cols;   // queued columns (request, column)
    int active = 0;                        // admitted requests not finished
    bool stop = false, dead = false;
    clk::time_point last_used;
};

// Device bytes of a request's pool: near-zone tiles (about 250 blocks per
// tet in the 27-box neighbourhood), projectors, Green octant, FFT grids and
// partial sums for the slots, Krylov bases and vectors of the batched
// solver, the mesh; plus a fixed 10% and 64 MiB margin.  And the request's
// own incident columns and solutions.
void estimate(const scd_request *r, const scd_grid_desc &d, int64_t *pool_bytes, int64_t *req_bytes) {
    const double T = r->T, n = 3.0 * T;
    const int ncol = ncols_of(r->Nmax);
    const int ns = 64;   // a pool's slots: `block` columns in flight per request it serves
    const bool mixed = r->opts.precision == SCD_PREC_MIXED;
    auto p2 = [](int v) { int p = 8; while (p < 2 * v) p <<= 1; return (double)p; };
    const double Px = p2(d.Nx), Py = p2(d.Ny);
    const double es = mixed ? 8.0 : 16.0;
    double b = 0;
    b += T * 250.0 * 9.0 * (r->storage_prec == SCD_STORE_C128 ? 16.0 : 8.0);   // near zone
    b += 4.0 * 27.0 * T * (16.0 + 8.0);                                           // projectors
    b += (Px / 2 + 1) * (Py / 2 + 1) * (p2(d.Nz) / 2 + 1) * 48.0;                 // Green octant (and its transpose)
    b += ns * 4.0 * Px * Py * d.Nz * (16.0 + (mixed ? 8.0 : 0.0));               // FFT work grids
    b += ns * 4.0 * (double)d.Nx * d.Ny * d.Nz * (16.0 + (mixed ? 8.0 : 0.0));   // result grids
    b += ns * n * 15.0 * (16.0 + (mixed ? 8.0 : 0.0));                            // near-zone partial sums
    b += ns * (r->opts.m + 1.0) * n * es;                                         // Krylov bases
    b += ns * n * (4.0 * es + 6.0 * 16.0 + (mixed ? 4.0 * 16.0 : 0.0));           // solver and work vectors
    b += 12.0 * T * 8.0 + T * 16.0;                                               // mesh on the device
    // tensor-core near zone (the default of the mixed form with complex64
    // storage): f16 hi/lo planes of every tile (8 B per complex plus
    // padding) and a pass of x blocks
    if (d.near_kernel != SCD_NEAR_CUDA_CORES && mixed && r->storage_prec != SCD_STORE_C128)
        b += T * 250.0 * 9.0 * 8.0 * 1.3 + n * 128.0 * 1.3;
    *pool_bytes = (int64_t)(b * 1.1) + (64LL << 20);
    // incident columns, solutions, T and the T assembly's partial sums
    *req_bytes = (int64_t)(2.0 * n * ncol * 16.0 + 70.0 * (double)ncol * ncol * 16.0);
}

}  // namespace

struct scd_server {
    int dev = 0;
    int64_t budget = 0;
    int max_running = 0;                   // pools solving at once (0 = the budget decides)
    std::mutex m;
    std::condition_variable cv;
    std::deque<int64_t> queue;
    std::map<int64_t, Req> reqs;
    std::vector<std::shared_ptr<Pool>> pools;
    int64_t next_id = 1;
    int64_t in_use = 0, peak_bytes = 0;
    int running = 0, peak_running = 0;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, columns = 0;
    int64_t pools_built = 0, pool_reuses = 0;
    std::vector<double> lat_ms;
    double busy_s = 0;
    clk::time_point busy_since;
    bool stop = false;
    std::thread dispatcher;
    std::vector<std::shared_ptr<Pool>> retired;   // pools whose worker returned, to be joined
};

namespace {

// a request left the running set (under the lock)
void finish_request(scd_server *s, Req &r, int rc, const std::string &err) {
    r.status = rc;
    r.err = err;
    r.t_done = clk::now();
    if (rc == SCD_OK || rc == SCD_NOT_CONVERGED) {
        r.state = SCD_REQ_DONE;
        s->completed += 1;
        s->columns += ncols_of(r.Nmax);
        s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count());
    } else {
        r.state = SCD_REQ_FAILED;
        s->failed += 1;
    }
    s->in_use -= r.est_req;
    s->running -= 1;
    if (s->running == 0) s->busy_s += std::chrono::duration<double>(clk::now() - s->busy_since).count();
    if (r.pool) {
        r.pool->active -= 1;
        r.pool->last_used = clk::now();
        r.pool.reset();
    }
}

// The pool's column queue as the batched solver's source.  Runs on the
// pool's worker thread, which owns the context.
struct PoolSource final : ColumnSource {
    scd_server *s;
    std::shared_ptr<Pool> P;
    std::map<int, std::pair<int64_t, int>> inflight;   // tag -> (request, column)
    int next_tag = 0;
    int block = 64;                                    // columns in flight per request

    // set up newly admitted requests: incident columns on the device, room for
    // their solutions, their columns queued
    void take_joining() {
        while (true) {
            int64_t id;
            Req *r;
            {
                std::lock_guard<std::mutex> g(s->m);
                if (P->joining.empty()) return;
                id = P->joining.front();
                P->joining.pop_front();
                r = &s->reqs[id];
            }
            scd_ctx *c = P->ctx;
            const int ncol = ncols_of(r->Nmax);
            const size_t bytes = sizeof(cd) * (size_t)c->n * ncol;
            int rc = SCD_OK;
            if (cudaMalloc(&r->d_mat, bytes) != cudaSuccess || cudaMalloc(&r->d_X, bytes) != cudaSuccess) {
                cudaGetLastError();
                rc = set_error(c, SCD_OOM, "request columns (%zu bytes)", 2 * bytes);
            }
            if (!rc) rc = setup_vswf(c, r->Nmax, r->d_mat);
            if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "request columns");
            std::lock_guard<std::mutex> g(s->m);
            if (rc) {
                cudaFree(r->d_mat); cudaFree(r->d_X);
                r->d_mat = r->d_X = nullptr;
                finish_request(s, *r, rc, c->err);
                s->cv.notify_all();
                continue;
            }
            r->iters.assign(ncol, 0);
            r->cols_done = 0;
            r->worst = SCD_OK;
            for (int j = 0; j < ncol; ++j) P->cols.emplace_back(id, j);
        }
    }

    bool next(const cd **rhs, cd **xout, int *tag) override {
        take_joining();
        std::lock_guard<std::mutex> g(s->m);
        if (P->cols.empty()) return false;
        // `block` columns in flight per unfinished request of the pool: the
        // parallelism separate pools would give them, on one operator
        if ((int)inflight.size() >= block * std::max(1, P->active)) return false;
        const auto job = P->cols.front();
        P->cols.pop_front();
        Req &r = s->reqs[job.first];
        const long long n = P->ctx->n;
        *rhs = r.d_mat + (size_t)job.second * n;
        *xout = r.d_X + (size_t)job.second * n;
        *tag = next_tag;
        inflight[next_tag++] = job;
        return true;
    }

    void finished(int tag, int it, int cv, int st, double) override {
        const auto job = inflight[tag];
        inflight.erase(tag);
        Req *r;
        {
            std::lock_guard<std::mutex> g(s->m);
            r = &s->reqs[job.first];
        }
        r->iters[job.second] = it;
        if (st != SCD_OK) r->worst = st;
        else if (!cv && r->worst == SCD_OK) r->worst = SCD_NOT_CONVERGED;
        if (++r->cols_done < ncols_of(r->Nmax)) return;
        // the request's last column: T = i k^3 mat^H X (src/T_matrix.f90:260,
        // 271-275) on the stream, after the solution copies
        scd_ctx *c = P->ctx;
        const int ncol = ncols_of(r->Nmax);
        int rc = r->worst == SCD_NOT_CONVERGED ? SCD_OK : r->worst;
        std::vector<cd> h((size_t)ncol * ncol);
        cd *d_T = nullptr;
        if (!rc) {
            if (cudaMalloc(&d_T, sizeof(cd) * h.size()) != cudaSuccess) {
                cudaGetLastError();
                rc = set_error(c, SCD_OOM, "T");
            }
        }
        if (!rc) {
            launch_T_assemble(c, r->d_mat, ncol, 0, ncol, r->d_X, d_T);
            rc = check_cuda(c, cudaMemcpyAsync(h.data(), d_T, sizeof(cd) * h.size(), cudaMemcpyDeviceToHost, c->st), "T");
            if (!rc) rc = check_cuda(c, cudaStreamSynchronize(c->st), "T");
        }
        cudaFree(d_T);
        cudaFree(r->d_mat);
        cudaFree(r->d_X);
        r->d_mat = r->d_X = nullptr;
        std::vector<scd_c128> Tm;
        if (!rc) {
            const double k3 = std::pow(c->k, 3.0);
            Tm.resize(h.size());
            for (size_t i = 0; i < h.size(); ++i) Tm[i] = scd_c128{-k3 * h[i].y, k3 * h[i].x};
            if (r->worst == SCD_NOT_CONVERGED) rc = SCD_NOT_CONVERGED;
        }
        std::lock_guard<std::mutex> g(s->m);
        r->Tm.swap(Tm);
        finish_request(s, *r, rc, rc && rc != SCD_NOT_CONVERGED ? c->err : std::string());
        s->cv.notify_all();
    }

    bool wait_more() override {
        std::unique_lock<std::mutex> lk(s->m);
        while (P->joining.empty() && P->cols.empty() && !P->stop) s->cv.wait(lk);
        return !(P->stop && P->joining.empty() && P->cols.empty());
    }
};

// a pool's worker: build the operator, then solve whatever its requests queue
void pool_worker(scd_server *s, std::shared_ptr<Pool> P, Req seed) {
    cudaSetDevice(s->dev);
    scd_grid_desc d{};
    scd_ctx *ctx = nullptr;
    int rc = scd_grid_from_mesh(seed.Nv, seed.coord.data(), seed.T, seed.etopol.data(), seed.grid_size, 2, &d);
    if (!rc) {
        d.device = s->dev;
        rc = scd_create(&ctx, &d);
    }
    if (!rc) rc = scd_set_wavenumber(ctx, seed.k);
    if (!rc) rc = scd_set_mesh(ctx, seed.Nv, seed.coord.data(), seed.etopol.data(), seed.param.data());
    if (!rc) rc = scd_set_green(ctx, nullptr);
    if (!rc) rc = scd_build_projectors(ctx);
    if (!rc) rc = scd_build_nearzone(ctx, seed.storage_prec);
    std::string err = rc ? (ctx ? scd_last_error(ctx) : "context creation failed") : "";
    if (!rc) {
        P->ctx = ctx;
        ctx->cgs_on = seed.opts.gram_schmidt != SCD_GS_MODIFIED;
        PoolSource src;
        src.s = s;
        src.P = P;
        const scd_solve_opts &o = seed.opts;
        src.block = o.block > 0 ? std::min(o.block, 64) : 64;
        rc = batch_run(ctx, src, o.tol, o.m, o.cycles, 64, o.precision, o.inner_tol, o.max_outer);
        if (rc) err = scd_last_error(ctx);
        // a solver error fails whatever is still in flight or queued
        std::lock_guard<std::mutex> g(s->m);
        for (auto &kv : src.inflight) P->cols.emplace_front(kv.second);
    }
    std::vector<int64_t> orphans;
    {
        std::lock_guard<std::mutex> g(s->m);
        P->dead = true;
        for (int64_t id : P->joining) orphans.push_back(id);
        for (auto &job : P->cols)
            if (std::find(orphans.begin(), orphans.end(), job.first) == orphans.end()) orphans.push_back(job.first);
        P->joining.clear();
        P->cols.clear();
        for (int64_t id : orphans) {
            Req &r = s->reqs[id];
            if (r.state != SCD_REQ_RUNNING) continue;
            cudaFree(r.d_mat); cudaFree(r.d_X);
            r.d_mat = r.d_X = nullptr;
            finish_request(s, r, rc ? rc : SCD_CUDA_ERROR, err.empty() ? "pool stopped" : err);
        }
    }
    if (ctx) scd_destroy(ctx);
    {
        std::lock_guard<std::mutex> g(s->m);
        P->ctx = nullptr;
        s->in_use -= P->est;
        s->pools.erase(std::remove(s->pools.begin(), s->pools.end(), P), s->pools.end());
        s->retired.push_back(P);
    }
    s->cv.notify_all();
}

int solving_pools(const scd_server *s) {
    int k = 0;
    for (auto &p : s->pools)
        if (!p->dead && !p->stop && p->active > 0) ++k;
    return k;
}

void dispatch_loop(scd_server *s) {
    std::unique_lock<std::mutex> lk(s->m);
    while (true) {
        // join the workers of retired pools: take the list first, since
        // workers that retire meanwhile append to it (only this thread
        // creates and joins the worker threads)
        if (!s->retired.empty()) {
            std::vector<std::shared_ptr<Pool>> done;
            done.swap(s->retired);
            lk.unlock();
            for (auto &p : done)
                if (p->worker.joinable()) p->worker.join();
            lk.lock();
            continue;   // re-check: more may have retired, and memory came back
        }
        // admit, in arrival order, every queued request that fits now: into
        // the resident pool of its key, or into a new pool (evicting idle
        // pools, least recently used first, when their memory is needed)
        bool admitted = false;
        for (auto q = s->queue.begin(); q != s->queue.end();) {
            Req &r = s->reqs[*q];
            std::shared_ptr<Pool> pool;
            for (auto &p : s->pools)
                if (!p->dead && !p->stop && p->key == r.key) pool = p;
            int64_t need = r.est_req + (pool ? 0 : r.est_pool);
            if (!pool && s->max_running > 0 && solving_pools(s) >= s->max_running) { ++q; continue; }
            if (s->in_use + need > s->budget) {
                // free idle pools of other keys, oldest first
                std::vector<std::shared_ptr<Pool>> idle;
                for (auto &p : s->pools)
                    if (!p->dead && !p->stop && p->active == 0 && p != pool) idle.push_back(p);
                std::sort(idle.begin(), idle.end(), [](auto &a, auto &b) { return a->last_used < b->last_used; });
                int64_t freeable = 0;
                for (auto &p : idle) freeable += p->est;
                if (s->in_use - freeable + need <= s->budget) {
                    int64_t over = s->in_use + need - s->budget;
                    for (auto &p : idle) {
                        if (over <= 0) break;
                        p->stop = true;   // its worker returns and releases p->est
                        over -= p->est;
                    }
                    s->cv.notify_all();
                }
                ++q;   // admitted once the memory is back
                continue;
            }
            if (!pool) {
                pool = std::make_shared<Pool>();
                pool->key = r.key;
                pool->est = r.est_pool;
                pool->last_used = clk::now();
                s->in_use += pool->est;
                s->pools.push_back(pool);
                s->pools_built += 1;
                pool->worker = std::thread(pool_worker, s, pool, r);
            } else {
                s->pool_reuses += 1;
            }
            r.state = SCD_REQ_RUNNING;
            r.pool = pool;
            pool->active += 1;
            pool->joining.push_back(*q);
            if (s->running == 0) s->busy_since = clk::now();
            s->running += 1;
            s->in_use += r.est_req;
            s->peak_running = std::max(s->peak_running, s->running);
            s->peak_bytes = std::max(s->peak_bytes, s->in_use);
            q = s->queue.erase(q);
            admitted = true;
        }
        if (admitted) s->cv.notify_all();
        if (s->stop && s->queue.empty() && s->running == 0) {
            // shut the resident pools down
            for (auto &p : s->pools) p->stop = true;
            s->cv.notify_all();
            if (s->pools.empty() && s->retired.empty()) break;
        }
        if (!admitted) s->cv.wait(lk);
    }
}

double pct(std::vector<double> v, double p) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double x = p / 100.0 * (double)(v.size() - 1);
    const size_t i = (size_t)x;
    const double f = x - (double)i;
    return i + 1 < v.size() ? v[i] * (1 - f) + v[i + 1] * f : v[i];
}

int request_estimate(const scd_request *req, int64_t *pool_bytes, int64_t *req_bytes) {
    if (!req || req->T <= 0 || req->Nv < 4 || !req->coord || !req->etopol || req->Nmax < 1) return SCD_BAD_ARG;
    scd_grid_desc d{};
    const int rc = scd_grid_from_mesh(req->Nv, req->coord, req->T, req->etopol, req->grid_size, 2, &d);
    if (rc) return rc;
    estimate(req, d, pool_bytes, req_bytes);
    return SCD_OK;
}

}  // namespace

extern "C" {

int scd_server_create(scd_server **out, int32_t device, int64_t hbm_budget, int32_t max_running) {
    if (!out || hbm_budget <= 0 || max_running < 0) return SCD_BAD_ARG;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { cudaGetLastError(); return SCD_NO_DEVICE; }
    if (device < 0 || device >= ndev) return SCD_BAD_ARG;
    scd_server *s = new scd_server();
    s->dev = device;
    s->budget = hbm_budget;
    s->max_running = max_running;
    s->dispatcher = std::thread(dispatch_loop, s);
    *out = s;
    return SCD_OK;
}

int scd_server_estimate(const scd_request *req, int64_t *bytes) {
    if (!bytes) return SCD_BAD_ARG;
    int64_t pb = 0, rb = 0;
    const int rc = request_estimate(req, &pb, &rb);
    if (rc) return rc;
    *bytes = pb + rb;
    return SCD_OK;
}

int scd_server_submit(scd_server *s, const scd_request *req, int64_t *id) {
    if (!s || !req || !id || !req->param) return SCD_BAD_ARG;
    if (!(req->k > 0) || req->opts.m < 1 || req->opts.m > SCD_M_MAX || req->opts.cycles < 1 || !(req->opts.tol > 0))
        return SCD_BAD_ARG;
    if (req->opts.precision != SCD_PREC_FP64 && req->opts.precision != SCD_PREC_MIXED) return SCD_BAD_ARG;
    if (req->opts.gram_schmidt < SCD_GS_DEFAULT || req->opts.gram_schmidt > SCD_GS_CLASSICAL) return SCD_BAD_ARG;
    if (req->opts.block < 0) return SCD_BAD_ARG;
    int64_t pb = 0, rb = 0;
    int rc = request_estimate(req, &pb, &rb);
    if (rc) return rc;
    if (pb + rb > s->budget) return SCD_OOM;
    Req r;
    r.Nv = req->Nv;
    r.T = req->T;
    r.coord.assign(req->coord, req->coord + 3LL * req->Nv);
    r.etopol.assign(req->etopol, req->etopol + 4LL * req->T);
    r.param.assign(req->param, req->param + req->T);
    r.k = req->k;
    r.grid_size = req->grid_size;
    r.Nmax = req->Nmax;
    r.storage_prec = req->storage_prec;
    r.opts = req->opts;
    r.est_pool = pb;
    r.est_req = rb;
    uint64_t h = 1469598103934665603ull;
    h = fnv(h, r.coord.data(), sizeof(double) * r.coord.size());
    h = fnv(h, r.etopol.data(), sizeof(int32_t) * r.etopol.size());
    h = fnv(h, r.param.data(), sizeof(scd_c128) * r.param.size());
    r.key.mesh = h;
    r.key.Nv = r.Nv;
    r.key.T = r.T;
    r.key.storage_prec = r.storage_prec;
    r.key.k = r.k;
    r.key.grid_size = r.grid_size;
    r.key.opts = r.opts;
    r.t_submit = clk::now();
    {
        std::lock_guard<std::mutex> g(s->m);
        if (s->stop) return SCD_NOT_READY;
        r.id = s->next_id++;
        *id = r.id;
        s->reqs.emplace(r.id, std::move(r));
        s->queue.push_back(*id);
        s->submitted += 1;
    }
    s->cv.notify_all();
    return SCD_OK;
}

int scd_server_poll(scd_server *s, int64_t id, int32_t *state, int32_t *status, double *latency_ms) {
    if (!s) return SCD_BAD_ARG;
    std::lock_guard<std::mutex> g(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return SCD_BAD_ARG;
    const Req &r = it->second;
    if (state) *state = r.state;
    if (status) *status = r.status;
    if (latency_ms)
        *latency_ms = (r.state == SCD_REQ_DONE || r.state == SCD_REQ_FAILED)
                          ? std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count()
                          : 0.0;
    return SCD_OK;
}

int scd_server_wait(scd_server *s, int64_t id, double timeout_s) {
    if (!s) return SCD_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return SCD_BAD_ARG;
    const auto deadline = clk::now() + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(timeout_s));
    while (it->second.state == SCD_REQ_QUEUED || it->second.state == SCD_REQ_RUNNING) {
        if (s->cv.wait_until(lk, deadline) == std::cv_status::timeout) return SCD_TIMEOUT;
    }
    return SCD_OK;
}

int scd_server_result(scd_server *s, int64_t id, scd_c128 *T, int32_t *iters) {
    if (!s || !T) return SCD_BAD_ARG;
    std::lock_guard<std::mutex> g(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return SCD_BAD_ARG;
    Req &r = it->second;
    if (r.state == SCD_REQ_FAILED) return r.status;
    if (r.state != SCD_REQ_DONE) return SCD_NOT_READY;
    if (r.consumed) return SCD_NOT_READY;   // read once: the result was released by the first read
    std::memcpy(T, r.Tm.data(), sizeof(scd_c128) * r.Tm.size());
    if (iters) std::memcpy(iters, r.iters.data(), sizeof(int32_t) * r.iters.size());
    const int rc = r.status;
    std::vector<scd_c128>().swap(r.Tm);
    r.consumed = true;
    return rc;
}

int scd_server_cancel(scd_server *s, int64_t id) {
    if (!s) return SCD_BAD_ARG;
    std::lock_guard<std::mutex> g(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return SCD_BAD_ARG;
    if (it->second.state != SCD_REQ_QUEUED) return SCD_NOT_READY;
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), id), s->queue.end());
    it->second.state = SCD_REQ_CANCELLED;
    s->cancelled += 1;
    s->cv.notify_all();
    return SCD_OK;
}

int scd_server_stats_get(scd_server *s, scd_server_stats *st) {
    if (!s || !st) return SCD_BAD_ARG;
    std::lock_guard<std::mutex> g(s->m);
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->failed = s->failed;
    st->cancelled = s->cancelled;
    st->columns = s->columns;
    st->queued = (int32_t)s->queue.size();
    st->running = s->running;
    st->peak_running = s->peak_running;
    st->bytes_in_use = s->in_use;
    st->peak_bytes = s->peak_bytes;
    st->p50_ms = pct(s->lat_ms, 50);
    st->p99_ms = pct(s->lat_ms, 99);
    st->busy_s = s->busy_s + (s->running ? std::chrono::duration<double>(clk::now() - s->busy_since).count() : 0.0);
    st->pools_built = s->pools_built;
    st->pool_reuses = s->pool_reuses;
    int res = 0;
    for (auto &p : s->pools)
        if (!p->dead) ++res;
    st->pools_resident = res;
    return SCD_OK;
}

const char *scd_server_error(scd_server *s, int64_t id) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> g(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return "unknown request";
    // a copy per calling thread: valid until this thread's next call, and
    // not overwritten by another thread's
    static thread_local std::string text;
    text = it->second.err;
    return text.c_str();
}

int scd_server_destroy(scd_server *s) {
    if (!s) return SCD_OK;
    {
        std::lock_guard<std::mutex> g(s->m);
        s->stop = true;
        for (int64_t id : s->queue) {
            s->reqs[id].state = SCD_REQ_CANCELLED;
            s->cancelled += 1;
        }
        s->queue.clear();
    }
    s->cv.notify_all();
    if (s->dispatcher.joinable()) s->dispatcher.join();
    delete s;
    return SCD_OK;
}

}  // extern "C"
