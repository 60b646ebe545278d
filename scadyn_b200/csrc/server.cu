// Request loop (include/scadyn_server.h): HBM-budget admission, one worker
// thread, context and CUDA stream per running request.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/scadyn_server.h"

namespace {

using clk = std::chrono::steady_clock;

struct Req {
    int64_t id = 0;
    int32_t Nv = 0, T = 0;
    std::vector<double> coord;
    std::vector<int32_t> etopol;
    std::vector<scd_c128> param;
    double k = 0, grid_size = 0;
    int32_t Nmax = 0, storage_prec = SCD_STORE_C64;
    scd_solve_opts opts{};
    int64_t est = 0;
    int32_t state = SCD_REQ_QUEUED, status = SCD_OK;
    std::string err;
    clk::time_point t_submit, t_done;
    std::vector<scd_c128> Tm;
    std::vector<int32_t> iters;
};

int ncols_of(int Nmax) { return 2 * ((Nmax + 1) * (Nmax + 1) - 1); }

// Device bytes of one request: near-zone tiles (about 250 blocks per tet in
// the 27-box neighbourhood), projectors, Green octant, FFT grids and
// partial sums for the slots, Krylov bases and vectors of the batched
// solver, resident incident columns; plus a fixed 10% and 64 MiB margin.
int64_t estimate(const scd_request *r, const scd_grid_desc &d) {
    const double T = r->T, n = 3.0 * T;
    const int ncol = ncols_of(r->Nmax);
    const int ns = std::max(1, std::min(r->opts.block > 0 ? r->opts.block : ncol, std::min(ncol, 64)));
    const bool mixed = r->opts.precision == SCD_PREC_MIXED;
    auto p2 = [](int v) { int p = 8; while (p < 2 * v) p <<= 1; return (double)p; };
    const double Px = p2(d.Nx), Py = p2(d.Ny);
    const double es = mixed ? 8.0 : 16.0;
    double b = 0;
    b += T * 250.0 * 9.0 * (r->storage_prec == SCD_STORE_C128 ? 16.0 : 8.0);   // near zone
    b += 4.0 * 27.0 * T * (16.0 + 8.0);                                           // projectors
    b += (Px / 2 + 1) * (Py / 2 + 1) * (p2(d.Nz) / 2 + 1) * 24.0;                 // Green octant
    b += ns * 4.0 * Px * Py * d.Nz * (16.0 + (mixed ? 8.0 : 0.0));               // FFT work grids
    b += ns * 4.0 * (double)d.Nx * d.Ny * d.Nz * (16.0 + (mixed ? 8.0 : 0.0));   // result grids
    b += ns * n * 15.0 * (16.0 + (mixed ? 8.0 : 0.0));                            // near-zone partial sums
    b += ns * (r->opts.m + 1.0) * n * es;                                         // Krylov bases
    b += ns * n * (4.0 * es + 6.0 * 16.0 + (mixed ? 4.0 * 16.0 : 0.0));           // solver and work vectors
    b += n * ncol * 16.0;                                                         // incident columns
    b += 12.0 * T * 8.0 + T * 16.0;                                               // mesh on the device
    // tensor-core near zone (the default of the mixed form with complex64
    // storage): f16 hi/lo planes of every tile (8 B per complex plus
    // padding) and a pass of x blocks
    if (d.near_kernel != SCD_NEAR_CUDA_CORES && mixed && r->storage_prec != SCD_STORE_C128)
        b += T * 250.0 * 9.0 * 8.0 * 1.3 + n * 128.0 * 1.3;   // x block: 32 rows x 2 B x hi/lo per unknown
    return (int64_t)(b * 1.1) + (64LL << 20);
}

}  // namespace

struct scd_server {
    int dev = 0;
    int64_t budget = 0;
    int max_running = 1;
    std::mutex m;
    std::condition_variable cv;
    std::deque<int64_t> queue;
    std::map<int64_t, Req> reqs;
    int64_t next_id = 1;
    int64_t in_use = 0, peak_bytes = 0;
    int running = 0, peak_running = 0;
    int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, columns = 0;
    std::vector<double> lat_ms;
    double busy_s = 0;
    clk::time_point busy_since;
    bool stop = false;
    std::thread dispatcher;
    std::map<int64_t, std::thread> workers;   // running (or just finished) request threads
    std::vector<int64_t> finished;            // workers done with the lock, to be joined
    std::string scratch_err;
};

namespace {

void run_request(scd_server *s, int64_t id) {
    Req *r;
    {
        std::lock_guard<std::mutex> g(s->m);
        r = &s->reqs[id];   // map nodes are stable; the worker owns the request while running
    }
    cudaSetDevice(s->dev);
    int rc = SCD_OK;
    std::string err;
    scd_ctx *ctx = nullptr;
    scd_grid_desc d{};
    const int ncol = ncols_of(r->Nmax);
    std::vector<scd_c128> Tm((size_t)ncol * ncol);
    std::vector<int32_t> it(ncol, 0);
    rc = scd_grid_from_mesh(r->Nv, r->coord.data(), r->T, r->etopol.data(), r->grid_size, 2, &d);
    if (!rc) {
        d.device = s->dev;
        rc = scd_create(&ctx, &d);
    }
    if (!rc) rc = scd_set_wavenumber(ctx, r->k);
    if (!rc) rc = scd_set_mesh(ctx, r->Nv, r->coord.data(), r->etopol.data(), r->param.data());
    if (!rc) rc = scd_set_green(ctx, nullptr);
    if (!rc) rc = scd_build_projectors(ctx);
    if (!rc) rc = scd_build_nearzone(ctx, r->storage_prec);
    if (!rc || rc == SCD_NOT_CONVERGED) {
        if (!rc) rc = scd_compute_T_matrix(ctx, r->Nmax, &r->opts, 0, ncol, Tm.data(), it.data());
    }
    if (rc && rc != SCD_NOT_CONVERGED) err = ctx ? scd_last_error(ctx) : "context creation failed";
    if (ctx) scd_destroy(ctx);
    {
        std::lock_guard<std::mutex> g(s->m);
        r->status = rc;
        r->err = err;
        r->t_done = clk::now();
        if (rc == SCD_OK || rc == SCD_NOT_CONVERGED) {
            r->state = SCD_REQ_DONE;
            r->Tm.swap(Tm);
            r->iters.swap(it);
            s->completed += 1;
            s->columns += ncol;
            s->lat_ms.push_back(std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count());
        } else {
            r->state = SCD_REQ_FAILED;
            s->failed += 1;
        }
        s->in_use -= r->est;
        s->running -= 1;
        s->finished.push_back(id);   // after this the worker takes the lock no more
        if (s->running == 0) s->busy_s += std::chrono::duration<double>(clk::now() - s->busy_since).count();
    }
    s->cv.notify_all();
}

void dispatch_loop(scd_server *s) {
    std::unique_lock<std::mutex> lk(s->m);
    while (true) {
        // join the workers that finished (they no longer take the lock)
        for (int64_t id : s->finished) {
            auto w = s->workers.find(id);
            if (w != s->workers.end()) {
                if (w->second.joinable()) w->second.join();
                s->workers.erase(w);
            }
        }
        s->finished.clear();
        // admit, in arrival order, every queued request that fits now
        bool admitted = false;
        for (auto q = s->queue.begin(); q != s->queue.end();) {
            if (s->running >= s->max_running) break;
            Req &r = s->reqs[*q];
            if (s->in_use + r.est > s->budget) { ++q; continue; }
            r.state = SCD_REQ_RUNNING;
            if (s->running == 0) s->busy_since = clk::now();
            s->running += 1;
            s->in_use += r.est;
            s->peak_running = std::max(s->peak_running, s->running);
            s->peak_bytes = std::max(s->peak_bytes, s->in_use);
            s->workers.emplace(*q, std::thread(run_request, s, *q));
            q = s->queue.erase(q);
            admitted = true;
        }
        if (s->stop && s->queue.empty()) break;
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

}  // namespace

extern "C" {

int scd_server_create(scd_server **out, int32_t device, int64_t hbm_budget, int32_t max_running) {
    if (!out || hbm_budget <= 0 || max_running < 1) return SCD_BAD_ARG;
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
    if (!req || !bytes || req->T <= 0 || req->Nv < 4 || !req->coord || !req->etopol || req->Nmax < 1) return SCD_BAD_ARG;
    scd_grid_desc d{};
    const int rc = scd_grid_from_mesh(req->Nv, req->coord, req->T, req->etopol, req->grid_size, 2, &d);
    if (rc) return rc;
    *bytes = estimate(req, d);
    return SCD_OK;
}

int scd_server_submit(scd_server *s, const scd_request *req, int64_t *id) {
    if (!s || !req || !id || !req->param) return SCD_BAD_ARG;
    if (!(req->k > 0) || req->opts.m < 1 || req->opts.m > SCD_M_MAX) return SCD_BAD_ARG;
    int64_t est = 0;
    int rc = scd_server_estimate(req, &est);
    if (rc) return rc;
    if (est > s->budget) return SCD_OOM;
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
    r.est = est;
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
    std::memcpy(T, r.Tm.data(), sizeof(scd_c128) * r.Tm.size());
    if (iters) std::memcpy(iters, r.iters.data(), sizeof(int32_t) * r.iters.size());
    const int rc = r.status;
    std::vector<scd_c128>().swap(r.Tm);
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
    return SCD_OK;
}

const char *scd_server_error(scd_server *s, int64_t id) {
    if (!s) return "null server";
    std::lock_guard<std::mutex> g(s->m);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return "unknown request";
    s->scratch_err = it->second.err;
    return s->scratch_err.c_str();
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
    for (auto &w : s->workers)
        if (w.second.joinable()) w.second.join();
    delete s;
    return SCD_OK;
}

}  // extern "C"
