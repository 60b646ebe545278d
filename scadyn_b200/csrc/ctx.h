// Internal context of the scadyn_gpu library and the launch wrappers of its
// kernels.  Device data are kept in "slot order": tetrahedra sorted by the
// projection box (cube) that holds them, so that every cube's tets, projector
// columns and unknowns are contiguous.  The public entry points permute at the
// boundary.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/scadyn_gpu.h"
#include "common.cuh"

// NVTX range for the lifetime of a scope (host side; a no-op unless a
// profiler is attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Near-zone groups: runs of consecutive slots of one projection box (cube)
// holding at most SCD_GROUP_MAX tets; a box with more tets is split into
// near-equal groups.  Tiles couple groups, so a tile's blocks, its two x
// segments and its partial sums fit a CTA's shared memory together.
#define SCD_GROUP_MAX 24

// One dense tile of near-zone blocks coupling the tets of group g1 (rows) to
// the tets of group g2 (columns), g1 <= g2.  Block (i, j) is the 3x3 matrix
// that maps the unknowns of slot s2+j onto the equations of slot s1+i; its
// element e = r + 3c is stored at data[data_off + tile_at(n1, i, j, e)]:
// planes over the row index i with the odd stride n1|1, so that lanes over i
// and lanes over j both read shared memory without bank conflicts.  A tile
// takes tile_elems(n1, n2) elements, an even count, so that tiles of
// complex64 start on 16-byte boundaries.  Diagonal tiles (g1 == g2) hold the
// full symmetric n1 x n1 pattern.
struct NearTile {
    int g1, g2;           // groups
    int c1, c2;           // projection boxes of the two groups
    int s1, s2;           // first slot of each group
    int n1, n2;           // tets of each group
    long long data_off;   // first element
    long long col_off;    // partial slot of g2 that receives M^T x (complex elements), -1 on diagonal tiles
};
SCD_HD long long tile_elems(int n1, int n2) { return ((long long)9 * n2 * (n1 | 1) + 1) & ~1LL; }
SCD_HD long long tile_at(int n1, int i, int j, int e) { return (long long)(9 * j + e) * (n1 | 1) + i; }

struct scd_ctx {
    int dev = 0;
    int nsm = 148;
    cudaStream_t st = nullptr;
    scd_grid_desc d{};
    int Nx = 0, Ny = 0, Nz = 0;          // grid nodes
    int Px = 0, Py = 0, Pz = 0;          // padded FFT lengths >= 2N (powers of two; 80, 96, 192 opt-in)
    int Hx = 0, Hy = 0, Hz = 0;          // P/2 + 1 (independent octant of Fg)
    int ncx = 0, ncy = 0, ncz = 0, ncubes = 0;
    int nb = 1;                          // basis functions per tet: 1 (constant), 4 (linear, as pseudo-tets)
    int T = 0;                           // tets, or pseudo-tets (4 per tet) for the linear basis
    long long n = 0;                     // 3T unknowns
    double k = 0.0;
    bool have_k = false;

    // tet order
    bool have_order = false;
    std::vector<int> perm;               // slot -> original tet (0-based)
    std::vector<int> slot_of;            // original tet -> slot
    std::vector<int> cube_of_slot;       // slot -> cube
    std::vector<int> cube_off;           // ncubes + 1
    int max_per_cube = 0;
    int *d_perm = nullptr, *d_cube_off = nullptr;
    // near-zone groups (see SCD_GROUP_MAX), numbered in slot order
    int ngroups = 0, max_per_group = 0;
    std::vector<int> grp_off;            // ngroups + 1 slot offsets
    std::vector<int> grp_cube;           // projection box of each group
    std::vector<int> grp_of_slot;
    int *d_grp_off = nullptr, *d_grp_cube = nullptr;

    // projectors: d_P[(g*27 + j)*T + slot], g = S, Sx, Sy, Sz
    bool have_proj = false;
    cd *d_P = nullptr;

    cd *d_tw[3] = {nullptr, nullptr, nullptr};   // twiddles for Px, Py, Pz

    // Green octant (Hx*Hy*Hz), pre-scaled by 1/(Px*Py*Pz)
    bool have_green = false;
    cd *d_Fo = nullptr;
    // the octant transposed for the fused y-z FFT pass (fft_yz.cuh), FP64 and
    // complex64, rebuilt after every new Green spectrum
    bool yz_on = true;                   // take the fused y-z pass where its lengths allow
    // right-hand sides per warp of the anterpolation and interpolation
    // kernels (0 = all of a call's; smaller spans give more warps in flight,
    // larger ones reuse the projector rows from L1)
    int scatter_span = 0, gather_span = 0;
    bool fyz_ready = false, fyz_ready_f = false;
    cd *d_Fyz = nullptr;
    cf *f_Fyz = nullptr;

    // near zone
    bool have_near = false;
    int near_prec = SCD_STORE_C64;
    void *d_tdata = nullptr;
    NearTile *d_tiles = nullptr;
    int ntiles = 0;
    long long tile_blocks = 0;           // n1*n2 summed over the tiles
    long long tile_store = 0;            // stored elements (tile_elems summed)
    long long max_tile_store = 0;        // largest tile_elems
    long long B_ref = 0;                 // blocks in the reference layout
    int near_split = 2;                  // partial sums per near-zone row/column sum (scd_grid_desc.near_split)
    int near_cfg_err = 0;                // a near-zone launch was skipped: a tile outgrew the shared-memory ring
    // partial-sum slots per group: slot 0 holds the group's row sums over
    // all its tiles, slots 1.. the M^T x products of the tiles (g', g),
    // g' < g, in tile order
    std::vector<long long> pslot_base;   // per group, complex offset of its first slot
    std::vector<int> pslot_cnt;          // per group, number of slots
    std::vector<int> grp_tile;           // ngroups + 1: first tile whose g1 is the group
    int *d_grp_tile = nullptr;
    int *d_kerr = nullptr;               // near-zone kernel error word (bounded waits)
    long long *d_pslot_base = nullptr;
    int *d_pslot_cnt = nullptr;
    long long part_len = 0;
    std::vector<NearTile> tiles_h;

    // mesh (device-side setup)
    bool have_mesh = false;
    int Nv = 0;
    std::vector<double> coord;           // (3, Nv)
    std::vector<int> etopol;             // (4, T) 1-based
    std::vector<cd> param;               // (T)
    double *d_tc = nullptr;              // slot-ordered tet vertex coords (12 per slot)
    double *d_tvol = nullptr;            // slot-ordered tet volumes
    cd *d_eps = nullptr;                 // slot-ordered eps

    // work buffers (sized for nrhs_cap right-hand sides)
    int nrhs_cap = 0;
    cd *d_bpart = nullptr;               // nrhs * ncubes * 4 * 27
    cd *d_W = nullptr;                   // nrhs * 4 * Px*Py*Nz
    cd *d_R = nullptr;                   // nrhs * 4 * Nx*Ny*Nz
    cd *d_nzpart = nullptr;              // nrhs * part_len
    cd *d_x = nullptr, *d_y = nullptr, *d_io = nullptr;   // n each (nrhs_cap)
    cd *d_xT = nullptr;                  // matvec input, right-hand sides interleaved per unknown

    // GMRES (batch.cu): single right-hand side of scd_gmres, grid barrier
    cd *d_rhs = nullptr;
    GridBarrier *d_bar = nullptr;
    int *d_err = nullptr;

    // timing
    cudaEvent_t ev[8] = {};
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;   // ordering against another context's stream
    double t_matvec = 0, t_near = 0, t_fft = 0, t_gather = 0, t_arn = 0, t_near_k = 0;
    double last_call_ms = 0, accum_ms = 0;
    long long n_matvec = 0, n_arn = 0, launches = 0;
    bool timing = false;

    // complex64 operator copies and work buffers (mixed-precision inner solves)
    bool f_ready = false;
    cf *f_P = nullptr, *f_Fo = nullptr, *f_tw[3] = {nullptr, nullptr, nullptr};
    cf *f_bpart = nullptr, *f_W = nullptr, *f_R = nullptr, *f_nzpart = nullptr, *f_xT = nullptr;
    int f_cap = 0;

    // classical Gram-Schmidt for the complex64 inner solves of the current
    // solve (batch.cu; scd_solve_opts.gram_schmidt)
    bool cgs_on = false;
    // tensor-core near zone of the complex64 matvec (near_mma.cu;
    // scd_grid_desc.near_kernel at context creation, scd_apply_tuning later)
    bool nzm_on = false, nzm_ready = false;
    int nzm_sched = 1;                   // instruction schedule (near_mma.cuh): 0 split, 1 merged, 2 wide
    unsigned char *d_t16 = nullptr;      // f16 hi/lo planes of every tile
    long long *d_t16_off = nullptr;      // per tile byte offset
    unsigned char *d_xb = nullptr;       // x blocks of one pass
    long long *d_xb_off = nullptr;       // per group byte offset
    unsigned int *d_xmax = nullptr;      // per right-hand side largest |x| (float bits), then the tiles'
    float *d_xinv = nullptr;             // per right-hand side 1 / (sA sx)
    float nzm_sA = 1.f;
    uint32_t nzm_x1[2] = {0, 0}, nzm_ring[2] = {0, 0};   // per pass width (16, 32): row x block, ring bytes
    uint32_t nzm_slack = 0;

    void *batch = nullptr;               // batch-solver buffers (batch.cu)
    std::vector<double> col_latency_ms;  // admission -> completion, last batch solve

    // resident incident matrix (3T, mat_cols), slot order: vswf2constant
    // built on the device for (mat_Nmax, mat_k), or the host's matrix
    // (mat_Nmax = 0, scd_set_rhs_matrix / scd_solve_columns); -1 = stale
    cd *d_mat = nullptr;
    int mat_cols = 0;
    int mat_Nmax = -1;
    double mat_k = 0.0;

    std::string err;
};

// ---- launch wrappers (kernels_matvec.cu) ----
void launch_permute_in(scd_ctx *c, const cd *x_orig, cd *x_slot, int nrhs, long long ld);
void launch_permute_out(scd_ctx *c, const cd *x_slot, cd *x_orig, int nrhs, long long ld);
// full matvec y = A x on slot-ordered vectors (nrhs columns, stride n)
void run_matvec(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done);
void run_matvec(scd_ctx *c, const cf *x, cf *y, int nrhs, const int *done);
int ensure_single(scd_ctx *c);
int ensure_work_single(scd_ctx *c, int nrhs);
void launch_near(scd_ctx *c, const cd *x, int nrhs, const int *done);
void launch_fft_chain(scd_ctx *c, const cd *x, int nrhs, const int *done);
void launch_gather(scd_ctx *c, const cd *x, cd *y, int nrhs, const int *done);
int build_twiddles(scd_ctx *c, int P, cd **out);
// tensor-core near zone (near_mma.cu)
int near_mma_prepare(scd_ctx *c);
void near_mma_run(scd_ctx *c, const cf *x, int nrhs, const int *done);

// ---- batched column solves (batch.cu) ----
// Where the batched solver's columns come from: the array of one call, or
// the queue of a served operator pool that arriving requests keep filling.
// All calls come from the thread that runs the solver.
struct ColumnSource {
    virtual ~ColumnSource() = default;
    // the next column to admit into a free slot: its right-hand side (device,
    // slot order), where its solution goes, and a tag; false if none is ready
    virtual bool next(const cd **rhs, cd **xout, int *tag) = 0;
    // the column `tag` left its slot; its solution copy is queued on the
    // context's stream
    virtual void finished(int tag, int iters, int conv, int status, double relres) = 0;
    // every slot is idle and the stream drained: block until columns may be
    // ready (true) or no more will come (false, the solver returns)
    virtual bool wait_more() { return false; }
    // the operator (index into batch_run's ops) that column `tag` is solved with
    virtual int op_of(int tag) { (void)tag; return 0; }
    // false once operator `op` has no column left to hand out
    virtual bool op_pending(int op) { (void)op; return true; }
};
// Batched solves on context c's slots and stream.  With ops (contexts of
// the same device and the same unknowns n, e.g. one per wavelength of one
// mesh), every column is solved with its own operator ops[op_of(tag)]: the
// matvecs of a tick run per operator (each on its context's stream, joined
// back), the Arnoldi steps of all slots in one launch.  An operator's work
// buffers then grow with the columns it has in flight, and are released
// (release_work) once it has none left to solve.
int batch_run(scd_ctx *c, ColumnSource &src, double tol, int m, int cycles, int ns, int precision, double inner_tol,
              int max_outer, const std::vector<scd_ctx *> *ops = nullptr);
void batch_free(scd_ctx *c);
int batch_solve(scd_ctx *c, int ncol, const cd *const *rhs_cols, cd *X, double tol, int m, int cycles, int ns,
                int *iters, int *conv, int *status, double *relres, int precision, double inner_tol, int max_outer);

// ---- setup (kernels_setup.cu) ----
int setup_green(scd_ctx *c, const scd_c128 *Fg_host);
int setup_projectors_device(scd_ctx *c);
int setup_nearzone_device(scd_ctx *c, int prec);
// slot-ordered (n, 2nm), or columns c0 .. c0 + cw - 1 of it (n, cw)
int setup_vswf(scd_ctx *c, int Nmax, cd *d_mat, int c0 = 0, int cw = -1);
void launch_T_assemble(scd_ctx *c, const cd *d_mat, int ncol_total, int col0, int ncb,
                       const cd *d_X, cd *d_T);

// ---- helpers (api.cu) ----
int set_error(scd_ctx *c, int code, const char *fmt, ...);
int check_cuda(scd_ctx *c, cudaError_t e, const char *what);
int ensure_work(scd_ctx *c, int nrhs);
void release_work(scd_ctx *c);
int near_status(scd_ctx *c);
// columns of the interleaved matvec input for nrhs right-hand sides: passes
// of 16, at least 2 (16-byte rows for complex64)
inline int xt_columns(int nrhs) { return std::max(2, (nrhs + 15) / 16 * 16); }   // SCD_TIMEOUT if a near-zone pipeline wait ran out (and clears it)
