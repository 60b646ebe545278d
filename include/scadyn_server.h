/* scadyn_server: a request loop for T-matrix solves on one GPU.
 *
 * Requests (a tetrahedral mesh with per-tet permittivity, a wavenumber, a
 * VSWF order and solve options) arrive at any time through
 * scd_server_submit.  Requests with the same operator key (mesh,
 * permittivities, wavenumber, cell size, near-zone storage and solve
 * options) share one resident pool: a device context with the operator
 * built once (Green octant, projectors, near zone) and the batched solver's
 * slots, on its own worker thread and CUDA stream.  A request joining a
 * pool that is solving has its incident columns queued at once; they take
 * slots as running columns finish, beside the columns of the other requests
 * (continuous batching across requests).  A pool has 64 slots and keeps
 * opts.block columns in flight per unfinished request (all 64 for block 0),
 * the parallelism separate pools would give.  Pools stay resident when idle, so
 * a later request of the same key skips the operator build; idle pools are
 * evicted, least recently used first, when a new pool needs the memory.  A
 * dispatcher admits queued requests in arrival order whenever the estimated
 * memory fits the HBM budget (a request that fits may pass one that does
 * not).  Pools solve concurrently, so their kernels overlap on the GPU.  A
 * column's arithmetic does not depend on its batch: a request's T-matrix is
 * bit-identical alone, in a mix, or sharing a pool.
 *
 * This layer has no counterpart in the reference (a batch program that
 * solves one geometry per run); it serves the per-request entry points of
 * scadyn_gpu.h (compute_T_matrix, src/T_matrix.f90:240-277, and its set-up).
 */
#ifndef SCADYN_SERVER_H
#define SCADYN_SERVER_H

#include "scadyn_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct scd_server scd_server;

/* request states */
#define SCD_REQ_QUEUED     0
#define SCD_REQ_RUNNING    1
#define SCD_REQ_DONE       2
#define SCD_REQ_FAILED     3
#define SCD_REQ_CANCELLED  4

typedef struct scd_request {
    int32_t Nv, T;
    const double *coord;        /* (3, Nv); copied by scd_server_submit */
    const int32_t *etopol;      /* (4, T), 1-based; copied */
    const scd_c128 *param;      /* (T) permittivity per tet; copied */
    double k;                   /* wavenumber */
    double grid_size;           /* build_grid cell_size (mesh%grid_size) */
    int32_t Nmax;               /* VSWF order: 2((Nmax+1)^2 - 1) columns */
    int32_t storage_prec;       /* near-zone storage: SCD_STORE_C64 or SCD_STORE_C128 */
    scd_solve_opts opts;        /* tolerances, precision form, slots (opts.block) */
} scd_request;

typedef struct scd_server_stats {
    int64_t submitted, completed, failed, cancelled;
    int64_t columns;            /* T-matrix columns of the completed requests */
    int32_t queued, running;
    int32_t peak_running;       /* most requests ever running at once */
    int64_t bytes_in_use;       /* estimated device bytes of the running requests */
    int64_t peak_bytes;
    double p50_ms, p99_ms;      /* submit -> done latency over the completed requests */
    double busy_s;              /* wall time with at least one request running */
    int64_t pools_built;        /* operator pools built (one per distinct operator key) */
    int64_t pool_reuses;        /* requests that joined a resident pool instead of building one */
    int32_t pools_resident;     /* pools on the device now, solving or idle */
} scd_server_stats;

/* Start a server on `device` with an HBM budget (bytes) for the resident
 * pools and the running requests; max_running bounds the pools solving at
 * once (0: only the budget bounds them). */
SCD_API int scd_server_create(scd_server **srv, int32_t device, int64_t hbm_budget, int32_t max_running);

/* Queue a request; its arrays are copied.  *id identifies it.  A request
 * whose estimate alone exceeds the budget is refused with SCD_OOM. */
SCD_API int scd_server_submit(scd_server *srv, const scd_request *req, int64_t *id);

/* Estimated device bytes of a request (the admission figure). */
SCD_API int scd_server_estimate(const scd_request *req, int64_t *bytes);

/* State of a request; for a finished one also its status code (SCD_OK,
 * SCD_NOT_CONVERGED, an error) and its submit -> done latency. */
SCD_API int scd_server_poll(scd_server *srv, int64_t id, int32_t *state, int32_t *status, double *latency_ms);

/* Block until the request leaves the queue and finishes, or timeout_s
 * elapses (SCD_TIMEOUT). */
SCD_API int scd_server_wait(scd_server *srv, int64_t id, double timeout_s);

/* T (ncol x ncol, column-major, ncol = 2((Nmax+1)^2 - 1)) and per-column
 * iteration counts (may be NULL) of a finished request; the request's
 * result is released afterwards, and a second call returns SCD_NOT_READY. */
SCD_API int scd_server_result(scd_server *srv, int64_t id, scd_c128 *T, int32_t *iters);

/* Drop a queued request (a running one finishes). */
SCD_API int scd_server_cancel(scd_server *srv, int64_t id);

SCD_API int scd_server_stats_get(scd_server *srv, scd_server_stats *st);

/* Text of the last error of a request (empty when none).  The text stays
 * valid until the calling thread's next scd_server_error call. */
SCD_API const char *scd_server_error(scd_server *srv, int64_t id);

/* Stop admitting, let the running requests finish, free everything. */
SCD_API int scd_server_destroy(scd_server *srv);

#ifdef __cplusplus
}
#endif
#endif
