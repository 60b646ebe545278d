! scadyn_gpu: Fortran 2003 iso_c_binding interface to libscadyn_gpu.so
! (include/scadyn_gpu.h).  A scadyn host links this module and the library
! and replaces the bodies of gmres / compute_Ax2 / the column loop of
! compute_T_matrix with the calls below; the reference's derived types stay
! as they are (the shim passes their array components, which are contiguous
! allocatables, by address).
module scadyn_gpu
   use, intrinsic :: iso_c_binding
   implicit none
   private

   integer(c_int), parameter, public :: SCD_OK = 0, SCD_NOT_CONVERGED = 1, SCD_NAN = 2, SCD_OOM = 3, &
                                        SCD_BAD_ARG = 4, SCD_TIMEOUT = 5, SCD_CUDA_ERROR = 6, &
                                        SCD_NOT_READY = 7, SCD_NO_DEVICE = 8
   integer(c_int), parameter, public :: SCD_STORE_C64 = 32, SCD_STORE_C128 = 64
   integer(c_int), parameter, public :: SCD_PREC_FP64 = 0, SCD_PREC_MIXED = 1
   integer(c_int), parameter, public :: SCD_M_MAX = 63
   ! kernel choices (0 = the library's default)
   integer(c_int), parameter, public :: SCD_FFT_DEFAULT = 0, SCD_FFT_POW2 = 1, SCD_FFT_SMOOTH = 2
   integer(c_int), parameter, public :: SCD_NEAR_DEFAULT = 0, SCD_NEAR_CUDA_CORES = 1, &
                                        SCD_NEAR_TENSOR_SPLIT = 2, SCD_NEAR_TENSOR_MERGED = 3, &
                                        SCD_NEAR_TENSOR_WIDE = 4
   integer(c_int), parameter, public :: SCD_GS_DEFAULT = 0, SCD_GS_MODIFIED = 1, SCD_GS_CLASSICAL = 2
   integer(c_int), parameter, public :: SCD_FFT_PASSES_DEFAULT = 0, SCD_FFT_PASSES_FUSED_YZ = 1, &
                                        SCD_FFT_PASSES_THREE = 2

   type, bind(C), public :: scd_grid_desc
      integer(c_int32_t) :: Nx, Ny, Nz
      real(c_double)     :: delta
      real(c_double)     :: min_coord(3)
      integer(c_int32_t) :: T
      integer(c_int32_t) :: order = 0
      integer(c_int32_t) :: M_ex = 2
      integer(c_int32_t) :: near_zone = 1
      integer(c_int32_t) :: device = 0
      integer(c_int32_t) :: fft_lengths = 0
      integer(c_int32_t) :: near_kernel = 0
      integer(c_int32_t) :: near_split = 0
      integer(c_int32_t) :: fft_passes = 0
   end type

   type, bind(C), public :: scd_solve_opts
      real(c_double)     :: tol
      integer(c_int32_t) :: m
      integer(c_int32_t) :: cycles
      integer(c_int32_t) :: block = 0
      integer(c_int32_t) :: precision = 0
      real(c_double)     :: inner_tol = 1d-4
      integer(c_int32_t) :: max_outer = 10
      integer(c_int32_t) :: gram_schmidt = 0
   end type

   ! device timing block (scd_get_timing), milliseconds
   type, bind(C), public :: scd_timing
      real(c_double)     :: matvec_ms, nearzone_ms, fft_ms, gather_ms, arnoldi_ms
      real(c_double)     :: last_call_ms, accum_ms
      integer(c_int64_t) :: launches, matvecs, arnoldi_steps
      real(c_double)     :: near_kernel_ms
   end type

   ! matvec kernel settings (scd_tune_matvec, scd_apply_tuning)
   type, bind(C), public :: scd_tuning
      integer(c_int32_t) :: nrhs, precision, near_kernel, fft_passes, scatter_span, gather_span
      real(c_double)     :: matvec_ms, default_ms
   end type

   ! request server (include/scadyn_server.h)
   integer(c_int), parameter, public :: SCD_REQ_QUEUED = 0, SCD_REQ_RUNNING = 1, SCD_REQ_DONE = 2, &
                                        SCD_REQ_FAILED = 3, SCD_REQ_CANCELLED = 4

   ! coord, etopol, param: c_loc of the mesh arrays (copied by scd_server_submit)
   type, bind(C), public :: scd_request
      integer(c_int32_t)   :: Nv, T
      type(c_ptr)          :: coord, etopol, param
      real(c_double)       :: k, grid_size
      integer(c_int32_t)   :: Nmax, storage_prec
      type(scd_solve_opts) :: opts
   end type

   type, bind(C), public :: scd_server_stats
      integer(c_int64_t) :: submitted, completed, failed, cancelled
      integer(c_int64_t) :: columns
      integer(c_int32_t) :: queued, running
      integer(c_int32_t) :: peak_running
      integer(c_int64_t) :: bytes_in_use
      integer(c_int64_t) :: peak_bytes
      real(c_double)     :: p50_ms, p99_ms
      real(c_double)     :: busy_s
      integer(c_int64_t) :: pools_built, pool_reuses
      integer(c_int32_t) :: pools_resident
   end type

   public :: scd_create, scd_destroy, scd_set_wavenumber, scd_set_green, scd_set_projectors, &
             scd_set_nearzone, scd_grid_from_mesh, scd_set_mesh, scd_build_projectors, &
             scd_build_nearzone, scd_get_projectors, scd_nearzone_count, scd_get_nearzone, &
             scd_matvec, scd_gmres, scd_set_rhs_matrix, scd_solve_columns, scd_vswf_rhs, scd_compute_T_matrix, &
             scd_compute_T_columns, &
             scd_get_timing, scd_profile_matvec, scd_tune_matvec, scd_apply_tuning, scd_solve_sweep, &
             scd_T_assemble_noalloc, scd_column_latency, &
             scd_nearzone_bytes, scd_selftest_waits, scd_check_matvec_repeat, scd_last_error_f
   public :: scd_server_create, scd_server_submit, scd_server_estimate, scd_server_poll, &
             scd_server_wait, scd_server_result, scd_server_cancel, scd_server_stats_get, &
             scd_server_destroy, scd_server_error_f

   interface
      integer(c_int) function scd_create(ctx, desc) bind(C, name="scd_create")
         import :: c_ptr, c_int, scd_grid_desc
         type(c_ptr), intent(out) :: ctx
         type(scd_grid_desc), intent(in) :: desc
      end function
      integer(c_int) function scd_destroy(ctx) bind(C, name="scd_destroy")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx
      end function
      type(c_ptr) function scd_last_error(ctx) bind(C, name="scd_last_error")
         import :: c_ptr
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function scd_set_wavenumber(ctx, k) bind(C, name="scd_set_wavenumber")
         import :: c_ptr, c_int, c_double
         type(c_ptr), value :: ctx
         real(c_double), value :: k
      end function
      ! Fg: matrices%Fg, or c_null_ptr to build the Green spectrum on the device
      integer(c_int) function scd_set_green(ctx, Fg) bind(C, name="scd_set_green")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx, Fg
      end function
      integer(c_int) function scd_set_projectors(ctx, M_box, T, S, Sx, Sy, Sz, indS) &
            bind(C, name="scd_set_projectors")
         import :: c_ptr, c_int, c_int32_t, c_double_complex
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: M_box, T
         complex(c_double_complex), intent(in) :: S(*), Sx(*), Sy(*), Sz(*)
         integer(c_int32_t), intent(in) :: indS(*)
      end function
      ! sp_mat: matrices%sp_mat (complex, default kind = c_float_complex)
      integer(c_int) function scd_set_nearzone(ctx, B, sp_mat, sp_ind, prec) bind(C, name="scd_set_nearzone")
         import :: c_ptr, c_int, c_int32_t, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: B
         type(c_ptr), value :: sp_mat
         integer(c_int32_t), intent(in) :: sp_ind(*)
         integer(c_int32_t), value :: prec
      end function
      integer(c_int) function scd_grid_from_mesh(Nv, coord, T, etopol, grid_size, M_ex, desc) &
            bind(C, name="scd_grid_from_mesh")
         import :: c_int, c_int32_t, c_double, scd_grid_desc
         integer(c_int32_t), value :: Nv, T, M_ex
         real(c_double), intent(in) :: coord(*)
         integer(c_int32_t), intent(in) :: etopol(*)
         real(c_double), value :: grid_size
         type(scd_grid_desc), intent(out) :: desc
      end function
      integer(c_int) function scd_set_mesh(ctx, Nv, coord, etopol, param) bind(C, name="scd_set_mesh")
         import :: c_ptr, c_int, c_int32_t, c_double, c_double_complex
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: Nv
         real(c_double), intent(in) :: coord(*)
         integer(c_int32_t), intent(in) :: etopol(*)
         complex(c_double_complex), intent(in) :: param(*)
      end function
      integer(c_int) function scd_build_projectors(ctx) bind(C, name="scd_build_projectors")
         import :: c_ptr, c_int
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function scd_build_nearzone(ctx, prec) bind(C, name="scd_build_nearzone")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: prec
      end function
      ! compute_Ax2: Ax = A x (matrices%x -> matrices%Ax)
      integer(c_int) function scd_matvec(ctx, x, Ax) bind(C, name="scd_matvec")
         import :: c_ptr, c_int, c_double_complex
         type(c_ptr), value :: ctx
         complex(c_double_complex), intent(in) :: x(*)
         complex(c_double_complex), intent(out) :: Ax(*)
      end function
      ! gmres: x0 = rhs, GMRES(m) with `cycles` restarts to tol
      integer(c_int) function scd_gmres(ctx, rhs, x, tol, m, cycles, iters, relres) bind(C, name="scd_gmres")
         import :: c_ptr, c_int, c_int32_t, c_double, c_double_complex
         type(c_ptr), value :: ctx
         complex(c_double_complex), intent(in) :: rhs(*)
         complex(c_double_complex), intent(out) :: x(*)
         real(c_double), value :: tol
         integer(c_int32_t), value :: m, cycles
         integer(c_int32_t), intent(out) :: iters
         real(c_double), intent(out) :: relres
      end function
      ! the incident matrix mat(3T, nmat) of vswf2constant, kept on the device
      integer(c_int) function scd_set_rhs_matrix(ctx, nmat, mat) bind(C, name="scd_set_rhs_matrix")
         import :: c_ptr, c_int, c_int32_t, c_double_complex
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: nmat
         complex(c_double_complex), intent(in) :: mat(*)
      end function
      ! the column loop body of compute_T_matrix for columns col0+1..col0+ncol:
      ! Tcols(:, j) = mat(:, :)^H x_j (T_matrix.f90:260); mat = c_loc(mat) or
      ! c_null_ptr for the matrix of scd_set_rhs_matrix
      integer(c_int) function scd_solve_columns(ctx, nmat, mat, col0, ncol, Tcols, opts, iters, X) &
            bind(C, name="scd_solve_columns")
         import :: c_ptr, c_int, c_int32_t, c_double_complex, scd_solve_opts
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: nmat
         type(c_ptr), value :: mat
         integer(c_int32_t), value :: col0, ncol
         complex(c_double_complex), intent(out) :: Tcols(*)
         type(scd_solve_opts), intent(in) :: opts
         integer(c_int32_t), intent(out) :: iters(*)
         type(c_ptr), value :: X
      end function
      ! compute_T_matrix with device-resident incident columns; T = i k^3 mat^H X
      integer(c_int) function scd_compute_T_matrix(ctx, Nmax, opts, col0, ncol, T, iters) &
            bind(C, name="scd_compute_T_matrix")
         import :: c_ptr, c_int, c_int32_t, c_double_complex, scd_solve_opts
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: Nmax, col0, ncol
         type(scd_solve_opts), intent(in) :: opts
         complex(c_double_complex), intent(out) :: T(*)
         integer(c_int32_t), intent(out) :: iters(*)
      end function
      ! cols(ncol): 0-based column indices, e.g. an MPI rank's round-robin share
      integer(c_int) function scd_compute_T_columns(ctx, Nmax, opts, ncol, cols, T, iters) &
            bind(C, name="scd_compute_T_columns")
         import :: c_ptr, c_int, c_int32_t, c_double_complex, scd_solve_opts
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: Nmax, ncol
         type(scd_solve_opts), intent(in) :: opts
         integer(c_int32_t), intent(in) :: cols(*)
         complex(c_double_complex), intent(out) :: T(*)
         integer(c_int32_t), intent(out) :: iters(*)
      end function
      ! the device operator back in the reference's layouts: S(27,T) .. indS(27,T)
      integer(c_int) function scd_get_projectors(ctx, S, Sx, Sy, Sz, indS) bind(C, name="scd_get_projectors")
         import :: c_ptr, c_int, c_int32_t, c_double_complex
         type(c_ptr), value :: ctx
         complex(c_double_complex), intent(out) :: S(*), Sx(*), Sy(*), Sz(*)
         integer(c_int32_t), intent(out) :: indS(*)
      end function
      integer(c_int64_t) function scd_nearzone_count(ctx) bind(C, name="scd_nearzone_count")
         import :: c_ptr, c_int64_t
         type(c_ptr), value :: ctx
      end function
      ! sp_mat(3,3,B) in FP64, sp_ind(2,B)
      integer(c_int) function scd_get_nearzone(ctx, B, sp_mat, sp_ind) bind(C, name="scd_get_nearzone")
         import :: c_ptr, c_int, c_int32_t, c_int64_t, c_double_complex
         type(c_ptr), value :: ctx
         integer(c_int64_t), value :: B
         complex(c_double_complex), intent(out) :: sp_mat(*)
         integer(c_int32_t), intent(out) :: sp_ind(*)
      end function
      ! vswf2constant on the device: mat(3T, 2nm)
      integer(c_int) function scd_vswf_rhs(ctx, Nmax, mat) bind(C, name="scd_vswf_rhs")
         import :: c_ptr, c_int, c_int32_t, c_double_complex
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: Nmax
         complex(c_double_complex), intent(out) :: mat(*)
      end function
      ! reset /= 0 clears the accumulated figures after reading them
      integer(c_int) function scd_get_timing(ctx, t, reset) bind(C, name="scd_get_timing")
         import :: c_ptr, c_int, c_int32_t, scd_timing
         type(c_ptr), value :: ctx
         type(scd_timing), intent(out) :: t
         integer(c_int32_t), value :: reset
      end function
      ! the wavelength loop of calc_T in one batched solve: ctxs(w) = c_ptr of
      ! wavelength w's context, T(w) = c_loc of its T(2nm_w, 2nm_w), iters(w) =
      ! c_loc of its iteration counts or c_null_ptr
      integer(c_int) function scd_solve_sweep(ctxs, nw, Nmax, opts, T, iters, status) &
            bind(C, name="scd_solve_sweep")
         import :: c_ptr, c_int, c_int32_t, scd_solve_opts
         type(c_ptr), intent(in) :: ctxs(*)
         integer(c_int32_t), value :: nw
         integer(c_int32_t), intent(in) :: Nmax(*)
         type(scd_solve_opts), intent(in) :: opts
         type(c_ptr), intent(in) :: T(*)
         type(c_ptr), intent(in) :: iters(*)
         integer(c_int32_t), intent(out) :: status(*)
      end function
      ! autotuner: time the matvec kernel choices, keep and return the fastest
      integer(c_int) function scd_tune_matvec(ctx, nrhs, precision, reps, tuning) bind(C, name="scd_tune_matvec")
         import :: c_ptr, c_int, c_int32_t, scd_tuning
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: nrhs, precision, reps
         type(scd_tuning), intent(out) :: tuning
      end function
      integer(c_int) function scd_apply_tuning(ctx, tuning) bind(C, name="scd_apply_tuning")
         import :: c_ptr, c_int, scd_tuning
         type(c_ptr), value :: ctx
         type(scd_tuning), intent(in) :: tuning
      end function
      integer(c_int) function scd_profile_matvec(ctx, reps, nrhs, precision) bind(C, name="scd_profile_matvec")
         import :: c_ptr, c_int, c_int32_t
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: reps, nrhs, precision
      end function
      integer(c_int) function scd_check_matvec_repeat(ctx, reps, nrhs, precision, bad_reps, bad_words) &
            bind(C, name="scd_check_matvec_repeat")
         import :: c_ptr, c_int, c_int32_t, c_int64_t
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: reps, nrhs, precision
         integer(c_int64_t), intent(out) :: bad_reps, bad_words
      end function
      ! mat, X, T: DEVICE addresses (e.g. c_loc of CUDA Fortran device arrays); stream: a cudaStream_t
      integer(c_int) function scd_T_assemble_noalloc(mat, n, ncol, X, ncb, T, stream) &
            bind(C, name="scd_T_assemble_noalloc")
         import :: c_ptr, c_int, c_int32_t, c_int64_t
         type(c_ptr), value :: mat
         integer(c_int64_t), value :: n
         integer(c_int32_t), value :: ncol
         type(c_ptr), value :: X
         integer(c_int32_t), value :: ncb
         type(c_ptr), value :: T, stream
      end function
      integer(c_int) function scd_column_latency(ctx, ncol, ms) bind(C, name="scd_column_latency")
         import :: c_ptr, c_int, c_int32_t, c_double
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: ncol
         real(c_double), intent(out) :: ms(*)
      end function
      integer(c_int64_t) function scd_nearzone_bytes(ctx) bind(C, name="scd_nearzone_bytes")
         import :: c_ptr, c_int64_t
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function scd_selftest_waits(device) bind(C, name="scd_selftest_waits")
         import :: c_int, c_int32_t
         integer(c_int32_t), value :: device
      end function
      ! request server
      integer(c_int) function scd_server_create(srv, device, hbm_budget, max_running) &
            bind(C, name="scd_server_create")
         import :: c_ptr, c_int, c_int32_t, c_int64_t
         type(c_ptr), intent(out) :: srv
         integer(c_int32_t), value :: device
         integer(c_int64_t), value :: hbm_budget
         integer(c_int32_t), value :: max_running
      end function
      integer(c_int) function scd_server_submit(srv, req, id) bind(C, name="scd_server_submit")
         import :: c_ptr, c_int, c_int64_t, scd_request
         type(c_ptr), value :: srv
         type(scd_request), intent(in) :: req
         integer(c_int64_t), intent(out) :: id
      end function
      integer(c_int) function scd_server_estimate(req, bytes) bind(C, name="scd_server_estimate")
         import :: c_int, c_int64_t, scd_request
         type(scd_request), intent(in) :: req
         integer(c_int64_t), intent(out) :: bytes
      end function
      integer(c_int) function scd_server_poll(srv, id, state, status, latency_ms) bind(C, name="scd_server_poll")
         import :: c_ptr, c_int, c_int32_t, c_int64_t, c_double
         type(c_ptr), value :: srv
         integer(c_int64_t), value :: id
         integer(c_int32_t), intent(out) :: state, status
         real(c_double), intent(out) :: latency_ms
      end function
      integer(c_int) function scd_server_wait(srv, id, timeout_s) bind(C, name="scd_server_wait")
         import :: c_ptr, c_int, c_int64_t, c_double
         type(c_ptr), value :: srv
         integer(c_int64_t), value :: id
         real(c_double), value :: timeout_s
      end function
      ! T(ncol, ncol); iters: c_loc of an (ncol) array, or c_null_ptr
      integer(c_int) function scd_server_result(srv, id, T, iters) bind(C, name="scd_server_result")
         import :: c_ptr, c_int, c_int64_t, c_double_complex
         type(c_ptr), value :: srv
         integer(c_int64_t), value :: id
         complex(c_double_complex), intent(out) :: T(*)
         type(c_ptr), value :: iters
      end function
      integer(c_int) function scd_server_cancel(srv, id) bind(C, name="scd_server_cancel")
         import :: c_ptr, c_int, c_int64_t
         type(c_ptr), value :: srv
         integer(c_int64_t), value :: id
      end function
      integer(c_int) function scd_server_stats_get(srv, st) bind(C, name="scd_server_stats_get")
         import :: c_ptr, c_int, scd_server_stats
         type(c_ptr), value :: srv
         type(scd_server_stats), intent(out) :: st
      end function
      type(c_ptr) function scd_server_error(srv, id) bind(C, name="scd_server_error")
         import :: c_ptr, c_int64_t
         type(c_ptr), value :: srv
         integer(c_int64_t), value :: id
      end function
      integer(c_int) function scd_server_destroy(srv) bind(C, name="scd_server_destroy")
         import :: c_ptr, c_int
         type(c_ptr), value :: srv
      end function
      integer(c_size_t) function c_strlen(s) bind(C, name="strlen")
         import :: c_ptr, c_size_t
         type(c_ptr), value :: s
      end function
   end interface

contains

   ! scd_last_error as a Fortran string
   function scd_last_error_f(ctx) result(msg)
      type(c_ptr), intent(in) :: ctx
      character(len=:), allocatable :: msg
      msg = c_string(scd_last_error(ctx))
   end function

   ! scd_server_error as a Fortran string
   function scd_server_error_f(srv, id) result(msg)
      type(c_ptr), intent(in) :: srv
      integer(c_int64_t), intent(in) :: id
      character(len=:), allocatable :: msg
      msg = c_string(scd_server_error(srv, id))
   end function

   ! a NUL-terminated C string (owned by the library) copied into a Fortran string
   function c_string(s) result(msg)
      type(c_ptr), intent(in) :: s
      character(len=:), allocatable :: msg
      character(kind=c_char), pointer :: p(:)
      integer :: i, n
      n = int(c_strlen(s))
      allocate (character(len=n) :: msg)
      if (n == 0) return
      call c_f_pointer(s, p, [n])
      do i = 1, n
         msg(i:i) = p(i)
      end do
   end function

end module scadyn_gpu
