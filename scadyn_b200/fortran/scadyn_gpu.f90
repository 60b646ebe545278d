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

   type, bind(C), public :: scd_grid_desc
      integer(c_int32_t) :: Nx, Ny, Nz
      real(c_double)     :: delta
      real(c_double)     :: min_coord(3)
      integer(c_int32_t) :: T
      integer(c_int32_t) :: order = 0
      integer(c_int32_t) :: M_ex = 2
      integer(c_int32_t) :: near_zone = 1
      integer(c_int32_t) :: device = 0
   end type

   type, bind(C), public :: scd_solve_opts
      real(c_double)     :: tol
      integer(c_int32_t) :: m
      integer(c_int32_t) :: cycles
      integer(c_int32_t) :: block = 0
      integer(c_int32_t) :: precision = 0
      real(c_double)     :: inner_tol = 1d-4
      integer(c_int32_t) :: max_outer = 10
   end type

   public :: scd_create, scd_destroy, scd_set_wavenumber, scd_set_green, scd_set_projectors, &
             scd_set_nearzone, scd_grid_from_mesh, scd_set_mesh, scd_build_projectors, &
             scd_build_nearzone, scd_matvec, scd_gmres, scd_solve_columns, scd_compute_T_matrix, &
             scd_last_error_f

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
      ! the column loop body of compute_T_matrix: Tcols(:, j) = mat(:, :)^H x_j
      integer(c_int) function scd_solve_columns(ctx, ncol, mat, Tcols, opts, iters, X) &
            bind(C, name="scd_solve_columns")
         import :: c_ptr, c_int, c_int32_t, c_double_complex, scd_solve_opts
         type(c_ptr), value :: ctx
         integer(c_int32_t), value :: ncol
         complex(c_double_complex), intent(in) :: mat(*)
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
      character(kind=c_char), pointer :: p(:)
      type(c_ptr) :: s
      integer :: i, n
      s = scd_last_error(ctx)
      n = int(c_strlen(s))
      call c_f_pointer(s, p, [n])
      allocate (character(len=n) :: msg)
      do i = 1, n
         msg(i:i) = p(i)
      end do
   end function

end module scadyn_gpu
