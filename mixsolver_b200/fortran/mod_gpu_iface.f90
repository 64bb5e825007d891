!-------------------------------------------------------------------------------
! mod_gpu_iface -- ISO_C_BINDING interface to libmixgpu.so (include/mixgpu.h).
!
! Belongs under the reference's src/common/. The derived types below are the C
! structs of mixgpu.h field for field (bind(C), same order, same kinds), and
! each interface block binds one extern "C" entry point by its C name. Status
! codes: 0 success, MGPU_E_* (< 0) library errors; solver outcomes come back
! through the reference's own ier / ierr codes.
!
! The library is built with nvcc (mixsolver_b200/build.py); link the
! Fortran executable with -lmixgpu -lstdc++ and the CUDA runtime.
!-------------------------------------------------------------------------------
module mod_gpu_iface
   use, intrinsic :: iso_c_binding
   implicit none
   private

   integer(c_int), parameter, public :: MGPU_OK = 0, MGPU_E_ARG = -1, MGPU_E_CUDA = -2, &
                                        MGPU_E_MESH = -3, MGPU_E_BC = -4, MGPU_E_TIMEOUT = -5, &
                                        MGPU_E_NOMEM = -6
   integer(c_int), parameter, public :: MGPU_PPE_JACOBI = 0, MGPU_PPE_IC0 = 1, MGPU_PPE_ILU0 = 2
   integer(c_int), parameter, public :: MGPU_MOM_ILU0 = 0, MGPU_MOM_JACOBI = 1
   integer(c_int), parameter, public :: MGPU_PREC_FP64 = 0, MGPU_PREC_MIXED = 1, MGPU_PREC_FP64_POLY = 2
   integer(c_int), parameter, public :: MGPU_MAXBC = 32, MGPU_MAXSOLVE = 8

   ! MgpuBcSpec: one control "bc" line (bc_spec_t without the thermal planes)
   type, bind(C), public :: mgpu_bc_spec
      integer(c_int32_t) :: zone = 0, btype = 0
      real(c_double)     :: uvel(3) = 0.0_c_double, pval = 0.0_c_double, mdot = 0.0_c_double
      real(c_double)     :: umean = 0.0_c_double, uspan = 0.0_c_double, uorigin = 0.0_c_double
      integer(c_int32_t) :: uaxis = 2, has_lid = 0, lid_dir = 0, pad0 = 0
      real(c_double)     :: lid_coord = 0.0_c_double, lid_vel(3) = 0.0_c_double
      integer(c_int32_t) :: ttype = 0, pad1 = 0
      real(c_double)     :: tval = 0.0_c_double, qval = 0.0_c_double
   end type mgpu_bc_spec

   ! MgpuTbcPlane: one tbc_plane line (bc: 0-based index of its bc line)
   type, bind(C), public :: mgpu_tbc_plane
      integer(c_int32_t) :: bc = 0, pdir = 0
      real(c_double)     :: pcoord = 0.0_c_double
      integer(c_int32_t) :: ttype = 0, pad0 = 0
      real(c_double)     :: tval = 0.0_c_double, qval = 0.0_c_double
   end type mgpu_tbc_plane

   ! MgpuCtrl: the ctrl_t scalars of this path plus the library's options
   type, bind(C), public :: mgpu_ctrl
      real(c_double)     :: rho, mu, alpha_u, alpha_p
      integer(c_int32_t) :: outer_max, lin_max
      real(c_double)     :: outer_tol, lin_tol, conv_blend, nonorth_corr
      integer(c_int32_t) :: ppe_precond, mom_solver, transient, time_scheme
      real(c_double)     :: dt
      integer(c_int32_t) :: n_time_max, n_correct
      real(c_double)     :: body_force(3)
      integer(c_int32_t) :: inlet_ramp, precision
      real(c_double)     :: mixed_tol
      integer(c_int32_t) :: nbc, n_outer_iter
      type(mgpu_bc_spec) :: bc(32)
      integer(c_int32_t) :: energy, boussinesq
      real(c_double)     :: cp, k_cond, tref, beta
      real(c_double)     :: gravity(3)
      integer(c_int32_t) :: ntbc, pad_e
      type(mgpu_tbc_plane) :: tbc(32)
   end type mgpu_ctrl

   ! MgpuMesh: the face list of mesh_t, flattened
   type, bind(C), public :: mgpu_mesh
      integer(c_int32_t) :: nnodes = 0, nfaces = 0, ncells = 0, pad0 = 0
      type(c_ptr)        :: x = c_null_ptr, fnode_ptr = c_null_ptr, fnodes = c_null_ptr
      type(c_ptr)        :: c0 = c_null_ptr, c1 = c_null_ptr, zone = c_null_ptr
   end type mgpu_mesh

   ! MgpuIterRec: one outer iteration (SIMPLE) or time step (PISO, PIMPLE)
   type, bind(C), public :: mgpu_iter_rec
      integer(c_int32_t) :: it, itl_max, nsolve, pad0
      integer(c_int32_t) :: lin_it(8), lin_ierr(8)
      real(c_double)     :: lin_res(8), imbal, du_max, dT_max, ressum, umax, cfl_max, t_now
   end type mgpu_iter_rec

   public :: mgpu_set_device, mgpu_last_error, mgpu_case_create, mgpu_case_destroy, &
             mgpu_fields_upload, mgpu_fields_download, mgpu_temperature_upload, &
             mgpu_temperature_download, mgpu_simple_run, mgpu_piso_run, &
             mgpu_pimple_run, mgpu_nan_scan, mgpu_krylov_solve, mgpu_csr_matvec, mgpu_set_tuning, &
             mgpu_error_message

   interface
      integer(c_int) function mgpu_set_device(device) bind(C, name='mgpu_set_device')
         import :: c_int
         integer(c_int), value :: device
      end function mgpu_set_device

      type(c_ptr) function mgpu_last_error() bind(C, name='mgpu_last_error')
         import :: c_ptr
      end function mgpu_last_error

      integer(c_int) function mgpu_case_create(mesh, ctrl, case_h, ier) bind(C, name='mgpu_case_create')
         import :: c_int, c_ptr, mgpu_mesh, mgpu_ctrl
         type(mgpu_mesh), intent(in)  :: mesh
         type(mgpu_ctrl), intent(in)  :: ctrl
         type(c_ptr),     intent(out) :: case_h
         integer(c_int),  intent(out) :: ier
      end function mgpu_case_create

      integer(c_int) function mgpu_case_destroy(case_h) bind(C, name='mgpu_case_destroy')
         import :: c_int, c_ptr
         type(c_ptr), value :: case_h
      end function mgpu_case_destroy

      integer(c_int) function mgpu_fields_upload(case_h, u, p, flux, u_old, u_old_old) &
            bind(C, name='mgpu_fields_upload')
         import :: c_int, c_ptr
         type(c_ptr), value :: case_h, u, p, flux, u_old, u_old_old
      end function mgpu_fields_upload

      integer(c_int) function mgpu_fields_download(case_h, u, p, flux, gp, gu, apc) &
            bind(C, name='mgpu_fields_download')
         import :: c_int, c_ptr
         type(c_ptr), value :: case_h, u, p, flux, gp, gu, apc
      end function mgpu_fields_download

      integer(c_int) function mgpu_temperature_upload(case_h, T, T_old, T_old_old) &
            bind(C, name='mgpu_temperature_upload')
         import :: c_int, c_ptr
         type(c_ptr), value :: case_h, T, T_old, T_old_old
      end function mgpu_temperature_upload

      integer(c_int) function mgpu_temperature_download(case_h, T, gt) &
            bind(C, name='mgpu_temperature_download')
         import :: c_int, c_ptr
         type(c_ptr), value :: case_h, T, gt
      end function mgpu_temperature_download

      integer(c_int) function mgpu_simple_run(case_h, nsteps, log, logcap, nrec, ier) &
            bind(C, name='mgpu_simple_run')
         import :: c_int, c_ptr
         type(c_ptr),    value       :: case_h, log
         integer(c_int), value       :: nsteps, logcap
         integer(c_int), intent(out) :: nrec, ier
      end function mgpu_simple_run

      integer(c_int) function mgpu_simple_run_fields(case_h, nsteps, log, logcap, nrec, ier, &
                                                     u, p, flux, gp, gu, apc) &
            bind(C, name='mgpu_simple_run_fields')
         import :: c_int, c_ptr
         type(c_ptr),    value       :: case_h, log, u, p, flux, gp, gu, apc
         integer(c_int), value       :: nsteps, logcap
         integer(c_int), intent(out) :: nrec, ier
      end function mgpu_simple_run_fields

      integer(c_int) function mgpu_piso_run(case_h, nsteps, log, logcap, nrec, ier) &
            bind(C, name='mgpu_piso_run')
         import :: c_int, c_ptr
         type(c_ptr),    value       :: case_h, log
         integer(c_int), value       :: nsteps, logcap
         integer(c_int), intent(out) :: nrec, ier
      end function mgpu_piso_run

      integer(c_int) function mgpu_pimple_run(case_h, nsteps, log, logcap, nrec, ier) &
            bind(C, name='mgpu_pimple_run')
         import :: c_int, c_ptr
         type(c_ptr),    value       :: case_h, log
         integer(c_int), value       :: nsteps, logcap
         integer(c_int), intent(out) :: nrec, ier
      end function mgpu_pimple_run

      integer(c_int) function mgpu_nan_scan(case_h, ifin, field, cell, val, kind) &
            bind(C, name='mgpu_nan_scan')
         import :: c_int, c_ptr, c_double
         type(c_ptr),    value       :: case_h
         integer(c_int), intent(out) :: ifin, field, cell, kind
         real(c_double), intent(out) :: val
      end function mgpu_nan_scan

      integer(c_int) function mgpu_krylov_solve(n, row_ptr, col_idx, val, b, x, tol, maxit, method, &
                                                norm_mode, it, res, ierr) bind(C, name='mgpu_krylov_solve')
         import :: c_int, c_int32_t, c_double
         integer(c_int),     value         :: n, maxit, method, norm_mode
         integer(c_int32_t), intent(in)    :: row_ptr(*), col_idx(*)
         real(c_double),     intent(in)    :: val(*), b(*)
         real(c_double),     intent(inout) :: x(*)
         real(c_double),     value         :: tol
         integer(c_int),     intent(out)   :: it, ierr
         real(c_double),     intent(out)   :: res
      end function mgpu_krylov_solve

      integer(c_int) function mgpu_pcg_poly_solve(n, row_ptr, col_idx, val, b, x, tol, maxit, precision, &
                                                  cheb_degree, it, res, ierr) bind(C, name='mgpu_pcg_poly_solve')
         import :: c_int, c_int32_t, c_double
         integer(c_int),     value         :: n, maxit, precision, cheb_degree
         integer(c_int32_t), intent(in)    :: row_ptr(*), col_idx(*)
         real(c_double),     intent(in)    :: val(*), b(*)
         real(c_double),     intent(inout) :: x(*)
         real(c_double),     value         :: tol
         integer(c_int),     intent(out)   :: it, ierr
         real(c_double),     intent(out)   :: res
      end function mgpu_pcg_poly_solve

      ! coupled mode (mod_mix_driver.f90 calling uns_solver_step with the
      ! peer's interface data, and uns_solver_extract_iface)
      integer(c_int) function mgpu_interface_set(case_h, n, faces, u, p) bind(C, name='mgpu_interface_set')
         import :: c_int, c_ptr
         type(c_ptr),    value :: case_h, faces, u, p
         integer(c_int), value :: n
      end function mgpu_interface_set

      integer(c_int) function mgpu_interface_set_T(case_h, n, faces, T, q, mode) &
            bind(C, name='mgpu_interface_set_T')
         import :: c_int, c_ptr
         type(c_ptr),    value :: case_h, faces, T, q, mode
         integer(c_int), value :: n
      end function mgpu_interface_set_T

      integer(c_int) function mgpu_interface_mode(case_h, p_dirichlet) bind(C, name='mgpu_interface_mode')
         import :: c_int, c_ptr
         type(c_ptr),    value :: case_h
         integer(c_int), value :: p_dirichlet
      end function mgpu_interface_mode

      integer(c_int) function mgpu_interface_extract(case_h, cap, faces, u, p, T, n) &
            bind(C, name='mgpu_interface_extract')
         import :: c_int, c_ptr
         type(c_ptr),    value       :: case_h, faces, u, p, T
         integer(c_int), value       :: cap
         integer(c_int), intent(out) :: n
      end function mgpu_interface_extract

      integer(c_int) function mgpu_csr_matvec(n, row_ptr, col_idx, val, x, y) bind(C, name='mgpu_csr_matvec')
         import :: c_int, c_int32_t, c_double
         integer(c_int),     value       :: n
         integer(c_int32_t), intent(in)  :: row_ptr(*), col_idx(*)
         real(c_double),     intent(in)  :: val(*), x(*)
         real(c_double),     intent(out) :: y(*)
      end function mgpu_csr_matvec

      integer(c_int) function mgpu_set_tuning(key, value) bind(C, name='mgpu_set_tuning')
         import :: c_int, c_char
         character(kind=c_char), intent(in) :: key(*)
         integer(c_int), value              :: value
      end function mgpu_set_tuning

      integer(c_int) function mgpu_get_tuning(key, value) bind(C, name='mgpu_get_tuning')
         import :: c_int, c_char
         character(kind=c_char), intent(in) :: key(*)
         integer(c_int), intent(out)        :: value
      end function mgpu_get_tuning
   end interface

contains

   ! The library's last error message as a Fortran string (up to 512 characters).
   function mgpu_error_message() result(msg)
      character(len=512) :: msg
      character(kind=c_char), pointer :: chars(:)
      type(c_ptr) :: p
      integer :: i
      msg = ''
      p = mgpu_last_error()
      if (.not. c_associated(p)) return
      call c_f_pointer(p, chars, [512])
      do i = 1, 512
         if (chars(i) == c_null_char) exit
         msg(i:i) = chars(i)
      end do
   end function mgpu_error_message

end module mod_gpu_iface
