/* scadyn_gpu — B200 (sm_100a) T-matrix solve path behind a C ABI.
 *
 * Drop-in for jherrane/scadyn's T-matrix solve: the precorrected-FFT JVIE
 * matrix-vector product (compute_Ax2), the restarted GMRES that calls it
 * (gmres), the per-column solve loop (compute_T_matrix), and the
 * per-wavelength setup that feeds them (build_G, pfft_projection_const,
 * compute_near_zone_interactions_const).  A Fortran host binds these entry
 * points through iso_c_binding; every entry point returns an int status.
 *
 * Array conventions are the reference's (Fortran column-major, 1-based ids):
 *   complex arrays   interleaved (re, im) == complex(c_double_complex)
 *   x, rhs, Ax       (3T)          unknowns of tet t at 3(t-1)+1..3(t-1)+3
 *   S, Sx, Sy, Sz    (27, T)       projector coefficients
 *   indS             (27, T)       1-based grid node ids (x fastest)
 *   sp_mat           (3, 3, B)     near-zone blocks, tet_B >= tet_T
 *   sp_ind           (2, B)        1-based (tet_T, tet_B)
 *   Fg               (2Nx,2Ny,2Nz) FFT of the zero-padded Green's function
 *   mat              (3T, nmat)    incident VSWF columns, nmat = 2nm
 *   Tcols            (nmat, ncol)  matᴴ·X, unscaled T_mat columns
 * Host arrays are borrowed for the duration of a call; device copies belong
 * to the context until scd_destroy.  A context is not thread-safe.
 */
#ifndef SCADYN_GPU_H
#define SCADYN_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define SCD_API __attribute__((visibility("default")))
#else
#define SCD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SCD_OK             0
#define SCD_NOT_CONVERGED  1   /* GMRES hit its cycle limit (the reference returns silently) */
#define SCD_NAN            2   /* a non-finite residual or breakdown */
#define SCD_OOM            3   /* device allocation failed */
#define SCD_BAD_ARG        4   /* invalid sizes, pointers or indices */
#define SCD_TIMEOUT        5   /* a deadline expired (host, or a bounded device wait) */
#define SCD_CUDA_ERROR     6   /* CUDA runtime error; see scd_last_error */
#define SCD_NOT_READY      7   /* an operator piece has not been set */
#define SCD_NO_DEVICE      8   /* no usable CUDA device */

typedef struct scd_c128 { double re, im; } scd_c128;   /* complex(c_double_complex) */
typedef struct scd_c64  { float re, im; }  scd_c64;    /* complex(c_float_complex)  */

typedef struct scd_ctx scd_ctx;

/* Grid and mesh sizes (type mesh_struct, src/common.f90:63-90). */
typedef struct scd_grid_desc {
    int32_t Nx, Ny, Nz;      /* grid nodes per axis (mesh%Nx..Nz) */
    double  delta;           /* node spacing (mesh%delta) */
    double  min_coord[3];    /* grid origin (mesh%min_coord) */
    int32_t T;               /* tetrahedra (mesh%N_tet) */
    int32_t order;           /* basis order (mesh%order): 0 constant (3 unknowns per tet), 1 linear
                                (12 per tet, x(12(t-1) + 4c + i)); with 1 the operator comes from the
                                host (scd_set_projectors/scd_set_nearzone) or from the mesh
                                (scd_set_mesh, scd_build_projectors, scd_build_nearzone) for
                                scd_matvec, scd_gmres and scd_solve_columns; scd_vswf_rhs and the
                                T-matrix entry points refuse it, as the reference solves no
                                linear-basis T-matrix (src/T_matrix.f90:250-259 pairs 3T-row
                                right-hand sides with its 12T unknowns) */
    int32_t M_ex;            /* projection order (mesh%M_ex); 2 only */
    int32_t near_zone;       /* near-cube radius (mesh%near_zone); 1 only */
    int32_t device;          /* CUDA device ordinal */
    /* kernel choices fixed at scd_create (0 = the library's default; no
     * counterpart in the reference, whose FFTW plans are made at run time,
     * src/possu.f90:82-89) */
    int32_t fft_lengths;     /* SCD_FFT_*: padded FFT length per axis */
    int32_t near_kernel;     /* SCD_NEAR_*: near-zone kernel of the complex64 matvec */
    int32_t near_split;      /* partial sums per near-zone row/column sum of the FP64 matvec: 1 one, 0 or 2 two */
    int32_t fft_passes;      /* SCD_FFT_PASSES_*: how the y and z transforms run */
} scd_grid_desc;

/* scd_grid_desc.fft_passes */
#define SCD_FFT_PASSES_DEFAULT  0   /* SCD_FFT_PASSES_FUSED_YZ where the lengths and shared memory allow */
#define SCD_FFT_PASSES_FUSED_YZ 1   /* one kernel per (x column, grid) transforms y, z, x Fg, z^-1, y^-1 in
                                       shared memory (y and z lengths 64, 80, 96, 128 or 192) */
#define SCD_FFT_PASSES_THREE    2   /* separate y forward, z (forward, x Fg, inverse), y inverse passes */

/* scd_grid_desc.fft_lengths.  Every choice is an exact linear convolution:
 * the input occupies N <= P/2 samples of each axis. */
#define SCD_FFT_DEFAULT         0   /* SCD_FFT_SMOOTH */
#define SCD_FFT_POW2            1   /* smallest power of two >= 2N */
#define SCD_FFT_SMOOTH          2   /* smallest of the powers of two and 80, 96, 192 that is >= 2N */

/* scd_grid_desc.near_kernel: the near-zone SpMV of the complex64 matvec of the
 * mixed-precision inner solves (the FP64 matvec always runs on the CUDA cores) */
#define SCD_NEAR_DEFAULT        0   /* SCD_NEAR_TENSOR_WIDE when the blocks are stored complex64, else CUDA cores */
#define SCD_NEAR_CUDA_CORES     1   /* complex64 FMAs on the CUDA cores */
#define SCD_NEAR_TENSOR_SPLIT   2   /* tcgen05 MMAs on f16 hi/lo tile planes, 9 MMAs per K step */
#define SCD_NEAR_TENSOR_MERGED  3   /* the same with x hi/lo merged into one operand, 6 MMAs per K step */
#define SCD_NEAR_TENSOR_WIDE    4   /* the merged schedule over 32 right-hand sides per pass while more than
                                       16 remain (each tile read once per 32, one CTA per SM), 16-wide for
                                       the rest; the same bits as SCD_NEAR_TENSOR_MERGED */

/* near-zone storage precision */
#define SCD_STORE_C64   32   /* complex64, as the reference stores sp_mat */
#define SCD_STORE_C128  64   /* complex128 */

/* largest Krylov dimension the solvers accept */
#define SCD_M_MAX       63

/* solve precision */
#define SCD_PREC_FP64   0    /* complex128 GMRES and matvec */
#define SCD_PREC_MIXED  1    /* complex64 inner GMRES, complex128 outer refinement */

typedef struct scd_solve_opts {
    double  tol;          /* GMRES relative residual (mesh%tol) */
    int32_t m;            /* Krylov dimension (mesh%maxit), 1..SCD_M_MAX */
    int32_t cycles;       /* restart cycles (mesh%restart) */
    int32_t block;        /* right-hand sides solved together; 0 = all */
    int32_t precision;    /* SCD_PREC_FP64 or SCD_PREC_MIXED */
    double  inner_tol;    /* mixed: inner complex64 GMRES tolerance */
    int32_t max_outer;    /* mixed: outer refinement steps */
    int32_t gram_schmidt; /* mixed: SCD_GS_* orthogonalisation of the complex64 inner solves */
} scd_solve_opts;

/* scd_solve_opts.gram_schmidt.  FP64 solves always use the reference's
 * modified Gram-Schmidt with its conditional re-orthogonalisation
 * (src/gmres_module.f90:241-258), so that iteration counts match it. */
#define SCD_GS_DEFAULT          0   /* SCD_GS_CLASSICAL */
#define SCD_GS_MODIFIED         1   /* one grid-wide pass per Krylov vector */
#define SCD_GS_CLASSICAL        2   /* all dots in one pass, then the reference's re-orthogonalisation test */

/* --- context ----------------------------------------------------------- */

/* Replaces the workspace set-up of gmres_module (src/gmres_module.f90:34-53). */
SCD_API int scd_create(scd_ctx **ctx, const scd_grid_desc *desc);
SCD_API int scd_destroy(scd_ctx *ctx);
SCD_API const char *scd_last_error(const scd_ctx *ctx);

/* mesh%k for the current wavelength (src/T_matrix.f90:52). */
SCD_API int scd_set_wavenumber(scd_ctx *ctx, double k);

/* matrices%Fg (src/build_G.f90:22-64).  NULL builds it on the device from
 * delta, min_coord and k (requires scd_set_wavenumber first). */
SCD_API int scd_set_green(scd_ctx *ctx, const scd_c128 *Fg);

/* matrices%S/Sx/Sy/Sz/indS (src/projection.f90:155-164). M_box must be 27.
 * T is the number of projector columns: the tets, or 4 per tet for the
 * linear basis (pfft_projection_lin, src/projection.f90:170-338), whose four
 * columns of a tet name its box. */
SCD_API int scd_set_projectors(scd_ctx *ctx, int32_t M_box, int32_t T,
                       const scd_c128 *S, const scd_c128 *Sx, const scd_c128 *Sy,
                       const scd_c128 *Sz, const int32_t *indS);

/* matrices%sp_mat / sp_ind (src/precorrection.f90:251-254).  sp_mat points to
 * scd_c64 when storage_prec == SCD_STORE_C64 and to scd_c128 otherwise; the
 * device copy is kept in the same precision.  Blocks are 3x3 (sp_mat(3,3,B)),
 * or 12x12 (sp_mat(12,12,B), matmul_Acorr, src/sparse_mat.f90:64-92) for the
 * linear basis. */
SCD_API int scd_set_nearzone(scd_ctx *ctx, int64_t B, const void *sp_mat, const int32_t *sp_ind,
                     int32_t storage_prec);

/* --- device-side setup --------------------------------------------------- */

/* build_grid (src/geometry.f90:60-125) on the host: fills desc from the mesh.
 * grid_size is the "cell_size" parameter (mesh%grid_size). */
SCD_API int scd_grid_from_mesh(int32_t Nv, const double *coord, int32_t T, const int32_t *etopol,
                       double grid_size, int32_t M_ex, scd_grid_desc *desc);

/* mesh%coord (3,Nv), mesh%etopol (4,T) 1-based, mesh%param (T) complex eps
 * (mesh_struct, src/common.f90:63-166); bins the tets into projection boxes
 * as tetras_in_cubes does (src/geometry.f90:330-377). */
SCD_API int scd_set_mesh(scd_ctx *ctx, int32_t Nv, const double *coord, const int32_t *etopol,
                 const scd_c128 *param);

/* pfft_projection_const (src/projection.f90:17-166) on the device; with
 * order 1 pfft_projection_lin (src/projection.f90:170-338), 4T columns. */
SCD_API int scd_build_projectors(scd_ctx *ctx);

/* compute_near_zone_interactions_const (src/precorrection.f90:131-264) on the
 * device, FP64 arithmetic, stored in storage_prec; with order 1
 * compute_near_zone_interactions_lin (src/precorrection.f90:268-725). */
SCD_API int scd_build_nearzone(scd_ctx *ctx, int32_t storage_prec);

/* Copy the device operator back in the reference's layouts (for a Fortran
 * host that keeps its own copy, and for checking): matrices%S/Sx/Sy/Sz/indS
 * (src/projection.f90:155-164) and sp_mat / sp_ind
 * (src/precorrection.f90:251-254).  The near zone comes
 * back ordered by (tet_T, tet_B): B = scd_nearzone_count blocks, 3x3
 * (sp_mat(3,3,B)), or 12x12 (sp_mat(12,12,B)) with order 1. */
SCD_API int scd_get_projectors(scd_ctx *ctx, scd_c128 *S, scd_c128 *Sx, scd_c128 *Sy, scd_c128 *Sz,
                       int32_t *indS);
SCD_API int64_t scd_nearzone_count(scd_ctx *ctx);
SCD_API int scd_get_nearzone(scd_ctx *ctx, int64_t B, scd_c128 *sp_mat, int32_t *sp_ind);

/* --- the hot path ------------------------------------------------------- */

/* compute_Ax2 (src/gmres_module.f90:57-176): Ax = A x. */
SCD_API int scd_matvec(scd_ctx *ctx, const scd_c128 *x, scd_c128 *Ax);

/* gmres (src/gmres_module.f90:180-325): x0 = rhs, GMRES(m) (m <= SCD_M_MAX)
 * with `cycles` restarts, stop when |g(i+1)|/||rhs|| < tol.  Returns SCD_NOT_CONVERGED with
 * the last iterate in x when the cycles run out. */
SCD_API int scd_gmres(scd_ctx *ctx, const scd_c128 *rhs, scd_c128 *x, double tol, int32_t m,
              int32_t cycles, int32_t *iters, double *relres);

/* The incident matrix mat (3T, nmat) of vswf2constant (src/T_matrix.f90:252),
 * copied to the device once per wavelength and kept there for
 * scd_solve_columns(mat = NULL) until it is replaced, the context is
 * destroyed, or scd_compute_T_matrix builds its own columns. */
SCD_API int scd_set_rhs_matrix(scd_ctx *ctx, int32_t nmat, const scd_c128 *mat);

/* The column loop of compute_T_matrix (src/T_matrix.f90:254-268) over columns
 * col0+1 .. col0+ncol of mat (3T, nmat): each column is solved (in blocks of
 * opts->block right-hand sides), and Tcols (nmat, ncol) receives
 * T_mat(:, col0+j) = matᴴ·x_j with the whole of mat (src/T_matrix.f90:260),
 * unscaled.  mat is the host array, copied in by this call, or NULL for the
 * matrix of scd_set_rhs_matrix (nmat must match).  iters (ncol) receives
 * per-column Arnoldi steps; X (3T, ncol) receives the solutions when non-NULL. */
SCD_API int scd_solve_columns(scd_ctx *ctx, int32_t nmat, const scd_c128 *mat, int32_t col0, int32_t ncol,
                              scd_c128 *Tcols, const scd_solve_opts *opts, int32_t *iters, scd_c128 *X);

/* vswf2constant (src/T_matrix.f90:280-305) on the device: mat (3T, 2nm) for
 * the mesh set by scd_set_mesh and the current wavenumber. */
SCD_API int scd_vswf_rhs(scd_ctx *ctx, int32_t Nmax, scd_c128 *mat);

/* compute_T_matrix (src/T_matrix.f90:240-277) with device-resident data:
 * the incident VSWF columns are built on the device (vswf2constant, kept for
 * the current Nmax and wavenumber), columns col0 .. col0+ncol-1 are solved,
 * and T(:, col0+j) = i k^3 mat^H x_j is returned in T (2nm, ncol).  With
 * col0 = 0 and ncol = 2nm, T holds [Taa Tab; Tba Tbb] (src/T_matrix.f90:271-275).
 * Needs scd_set_mesh (for the VSWF points) and the operator. */
SCD_API int scd_compute_T_matrix(scd_ctx *ctx, int32_t Nmax, const scd_solve_opts *opts, int32_t col0,
                                 int32_t ncol, scd_c128 *T, int32_t *iters);

/* scd_compute_T_matrix over an arbitrary set of columns: cols (ncol) lists
 * 0-based column indices (each once, any order) of the 2nm columns of the
 * column loop (src/T_matrix.f90:254-268); T (2nm, ncol) receives
 * T(:, j) = i k^3 mat^H x_{cols[j]} and iters (ncol) the Arnoldi steps.  For
 * hosts that deal the columns out to several GPUs round-robin, so that the
 * slow high-order columns spread evenly; a column gives the same bits as in
 * scd_compute_T_matrix. */
SCD_API int scd_compute_T_columns(scd_ctx *ctx, int32_t Nmax, const scd_solve_opts *opts, int32_t ncol,
                                  const int32_t *cols, scd_c128 *T, int32_t *iters);

/* The wavelength loop of calc_T (src/T_matrix.f90:36-79) in one solve: ctxs[w]
 * holds wavelength w's operator (scd_set_wavenumber, scd_set_mesh with the
 * one mesh, Green spectrum, projectors and near zone, each with its own grid),
 * and all 2nm_w columns of every wavelength (nm_w from Nmax[w]) are solved
 * as slots of one batched solver on ctxs[0]'s stream: columns of different
 * wavelengths share each tick, each multiplied by its own operator (the
 * operators' matvecs run on their contexts' streams, joined back per tick).
 * T[w] (2nm_w, 2nm_w) receives [Taa Tab; Tba Tbb] of wavelength w
 * (src/T_matrix.f90:271-275), iters[w] (may be NULL, or hold NULLs) the
 * per-column Arnoldi steps, status[w] (may be NULL) each wavelength's status.
 * The contexts must share the device and the mesh (the same unknowns); a
 * column gives the same bits here as in scd_compute_T_matrix on its context. */
SCD_API int scd_solve_sweep(scd_ctx *const *ctxs, int32_t nw, const int32_t *Nmax, const scd_solve_opts *opts,
                            scd_c128 *const *T, int32_t *const *iters, int32_t *status);

/* Device timing, milliseconds, from CUDA events on the context's stream (no
 * counterpart in the reference, which times nothing on this path). */
typedef struct scd_timing {
    double matvec_ms;      /* average matvec (scd_profile_matvec) */
    double nearzone_ms;    /* average near-zone kernel */
    double fft_ms;         /* average scatter + FFT convolution chain */
    double gather_ms;      /* average interpolation / assembly kernel */
    double arnoldi_ms;     /* average orthogonalisation step */
    double last_call_ms;   /* last scd_solve_columns / scd_compute_T_matrix / scd_gmres */
    double accum_ms;       /* sum of last_call_ms since the last reset */
    int64_t launches;      /* kernels launched since the last reset */
    int64_t matvecs;       /* operator applications since the last reset */
    int64_t arnoldi_steps; /* Arnoldi steps since the last reset */
    double near_kernel_ms; /* average duration of the main near-zone kernel launch (the last pass of a
                              matvec: k_near_mma or k_near_groups), scd_profile_matvec */
} scd_timing;
/* Read the timing block; reset != 0 then clears the fields counted since the
 * last reset (accum_ms, launches, matvecs, arnoldi_steps).  No counterpart
 * in the reference. */
SCD_API int scd_get_timing(scd_ctx *ctx, scd_timing *t, int32_t reset);

/* No counterpart in the reference (a measurement of compute_Ax2,
 * src/gmres_module.f90:57-176).  Run `reps` device-resident matvecs on
 * `nrhs` fixed vectors at once, in FP64 (SCD_PREC_FP64) or in the complex64
 * form the mixed-precision inner solves use (SCD_PREC_MIXED), and record
 * per-kernel averages per call in the timing block (matvec_ms, nearzone_ms,
 * fft_ms, gather_ms). */
SCD_API int scd_profile_matvec(scd_ctx *ctx, int32_t reps, int32_t nrhs, int32_t precision);

/* Matvec kernel settings of a context that can change between calls; the
 * autotuner's result (scd_tune_matvec) and what scd_apply_tuning sets. */
typedef struct scd_tuning {
    int32_t nrhs;             /* right-hand sides per matvec the setting was timed at */
    int32_t precision;        /* SCD_PREC_FP64 or SCD_PREC_MIXED (the complex64 matvec) */
    int32_t near_kernel;      /* SCD_NEAR_CUDA_CORES / _TENSOR_SPLIT / _TENSOR_MERGED / _TENSOR_WIDE (complex64 matvec) */
    int32_t fft_passes;       /* SCD_FFT_PASSES_FUSED_YZ or SCD_FFT_PASSES_THREE */
    int32_t scatter_span;     /* right-hand sides per warp of the anterpolation, 0 = all of a call's */
    int32_t gather_span;      /* right-hand sides per warp of the interpolation, 0 = all */
    double matvec_ms;         /* the chosen setting's matvec time */
    double default_ms;        /* the library defaults' matvec time */
} scd_tuning;

/* Autotuner (no counterpart in the reference, whose analogue is FFTW's
 * planning, src/possu.f90:82-89): times `reps` device-resident matvecs of
 * `nrhs` right-hand sides for the candidate settings of each knob in turn
 * (near-zone kernel, fused or three-pass y-z FFT, anterpolation and
 * interpolation spans), keeps the fastest, applies it to the context and
 * returns it.  Results do not depend on the choice beyond rounding (the
 * near-zone kernels round differently; every choice keeps a column
 * bit-identical alone and in any batch). */
SCD_API int scd_tune_matvec(scd_ctx *ctx, int32_t nrhs, int32_t precision, int32_t reps, scd_tuning *out);

/* Apply a stored tuning (e.g. a cached scd_tune_matvec result for the same
 * grid, tets and right-hand sides) without timing anything.  No counterpart
 * in the reference (like reusing an FFTW plan, src/possu.f90:82-89). */
SCD_API int scd_apply_tuning(scd_ctx *ctx, const scd_tuning *tuning);

/* T = mat^H X without allocating: mat (n, ncol), X (n, ncb) and T (ncol, ncb)
 * are DEVICE pointers owned by the caller; the kernels run on `stream`
 * (a cudaStream_t, NULL = the legacy default stream) and the call returns
 * after launching them.  No counterpart in the reference: it is for callers
 * that cannot let a library call cudaMalloc, such as a Fortran host whose
 * device memory all comes from its own allocator (CUDA Fortran device
 * arrays, OpenACC data regions) and must stay under its accounting.  Scratch
 * is a fixed 4 MiB per-device array, held by every GPU that loads the
 * library until the process exits, so ncol*ncb must not exceed 262144
 * (SCD_BAD_ARG otherwise).  The first call on a device looks up that array's
 * device address and keeps it.  The kept address is not valid after
 * cudaDeviceReset, so do not call this after a reset in the same process.
 * An error left pending by an earlier call of the caller's is returned as
 * SCD_CUDA_ERROR before anything launches, and left pending.  All calls share the array: calls that overlap on the GPU
 * race and must be ordered by the caller (one stream, or events). */
SCD_API int scd_T_assemble_noalloc(const scd_c128 *mat, int64_t n, int32_t ncol, const scd_c128 *X, int32_t ncb,
                                   scd_c128 *T, void *stream);

/* No counterpart in the reference.  Per-column solve latency (admission to
 * completion, milliseconds on the host clock, each tick ending in a stream
 * synchronisation) of the last scd_solve_columns / scd_compute_T_matrix
 * call; ncol must match it. */
SCD_API int scd_column_latency(scd_ctx *ctx, int32_t ncol, double *ms);

/* Near-zone blocks in the reference layout (tet_B >= tet_T; the B of
 * sp_mat(3,3,B), src/precorrection.f90:251-254) and, with no counterpart in
 * the reference, the bytes of the device tile storage. */
SCD_API int64_t scd_nearzone_bytes(scd_ctx *ctx);

/* Failure detection self-test (no counterpart in the reference): runs the
 * library's bounded device waits -- the grid barrier of the cooperative
 * solver kernels and the mbarrier wait of the near-zone pipeline -- against
 * conditions that nothing satisfies, with short limits.  Returns SCD_TIMEOUT
 * when both waits gave up and reported it (the behaviour a stuck launch gets),
 * SCD_CUDA_ERROR otherwise.  The device stays usable. */
SCD_API int scd_selftest_waits(int32_t device);

/* Determinism self-check of the batched matvec (no counterpart in the
 * reference): nrhs fixed input columns (different in every column), one
 * matvec of the current kernel choices as the reference output, then reps
 * more matvecs of the same inputs, each compared with it bit for bit on the
 * device.  *bad_reps = repetitions whose output differs in any bit, *bad_words
 * = differing 32-bit words over all of them.  Every kernel of the matvec sums
 * in a fixed order, so both are 0; anything else is a race.  precision:
 * SCD_PREC_FP64 (complex128 columns) or SCD_PREC_MIXED (complex64). */
SCD_API int scd_check_matvec_repeat(scd_ctx *ctx, int32_t reps, int32_t nrhs, int32_t precision,
                                    int64_t *bad_reps, int64_t *bad_words);

#ifdef __cplusplus
}
#endif
#endif /* SCADYN_GPU_H */
