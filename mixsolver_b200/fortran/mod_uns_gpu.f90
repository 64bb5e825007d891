!-------------------------------------------------------------------------------
! mod_uns_gpu -- the unstructured SIMPLE / PISO / PIMPLE drivers on the GPU,
! with the argument lists of the reference's own drivers:
!
!   simple_run_gpu  <- simple_run      (src/unstructured/mod_uns_simple.f90:88)
!   piso_run_gpu    <- piso_run_mpi    (src/unstructured/mod_uns_simple_mpi.f90:298)
!   pimple_run_gpu  <- pimple_run_mpi  (src/unstructured/mod_uns_simple_mpi.f90:580)
!
! A caller switches a call site by renaming the routine (uns_solver_step in
! mod_uns_driver.f90:245-255 for SIMPLE, mod_uns_driver_mpi.f90:319-329 for
! PISO / PIMPLE at one rank); nothing else changes. On first use the mesh,
! its derived arrays and the control go to the GPU once (mgpu_case_create) and
! stay there; each call then copies the fields in, runs, and copies them out,
! so the coupling loop (mod_mix_driver.f90:1032), which calls uns_solver_step
! again and again, does not upload the mesh again. uns_gpu_release frees the
! case (at finalisation).
!
! ier: the reference's codes (SIMPLE 20/21/60, PISO 30/31/33/34/60, PIMPLE
! 50/51/53/54/60); GPU_IER (90, unused by the reference) when the library
! itself fails, with its message printed.
!
! Form of the arithmetic: the FP64 parity form by default; the environment
! variable MIXGPU_PRECISION = mixed selects the mixed-precision form (FP32
! inner Krylov inside FP64 refinement), fp64poly the same solvers in FP64.
! Belongs under the reference's src/common/ next to mod_gpu_iface.f90.
!-------------------------------------------------------------------------------
module mod_uns_gpu
   use, intrinsic :: iso_c_binding
   use mod_uns_mesh,         only: mesh_t
   use mod_uns_connectivity, only: conn_t
   use mod_uns_geometry,     only: geom_t
   use mod_uns_control,      only: ctrl_t
   use mod_uns_bc,           only: bc_t
   use mod_uns_fields,       only: fields_t
   use mod_uns_local_mesh,   only: local_mesh_t
   use mod_uns_halo,         only: halo_info_t
   use mod_gpu_iface
   implicit none
   private

   public :: simple_run_gpu, piso_run_gpu, pimple_run_gpu, uns_gpu_release
   integer, parameter, public :: GPU_IER = 90

   ! the resident case and the flattened mesh arrays it was built from
   type(c_ptr), save :: g_case = c_null_ptr
   integer,     save :: g_nfaces = -1, g_ncells = -1
   real(c_double),     allocatable, target, save :: g_x(:,:)
   integer(c_int32_t), allocatable, target, save :: g_fptr(:), g_fnodes(:), g_c0(:), g_c1(:), g_zone(:)

contains

   ! mesh_t -> MgpuMesh: face_t is not interoperable (allocatable nodes), so the
   ! face list is flattened into offset / node arrays (nodes and cells 1-based).
   subroutine pack_mesh(m, mm)
      type(mesh_t),    intent(in)  :: m
      type(mgpu_mesh), intent(out) :: mm
      integer :: i, k, nn
      if (allocated(g_x)) deallocate(g_x, g_fptr, g_fnodes, g_c0, g_c1, g_zone)
      allocate(g_x(3, m%nnodes), g_fptr(m%nfaces + 1), g_c0(m%nfaces), g_c1(m%nfaces), g_zone(m%nfaces))
      g_x = m%x(:, 1:m%nnodes)
      g_fptr(1) = 0
      do i = 1, m%nfaces
         g_fptr(i + 1) = g_fptr(i) + size(m%f(i)%nodes)
      end do
      allocate(g_fnodes(max(1, int(g_fptr(m%nfaces + 1)))))
      k = 0
      do i = 1, m%nfaces
         nn = size(m%f(i)%nodes)
         g_fnodes(k + 1:k + nn) = m%f(i)%nodes(1:nn)
         k = k + nn
         g_c0(i) = m%f(i)%c0
         g_c1(i) = m%f(i)%c1
         g_zone(i) = m%f(i)%zone
      end do
      mm%nnodes = m%nnodes
      mm%nfaces = m%nfaces
      mm%ncells = m%ncells
      mm%x = c_loc(g_x)
      mm%fnode_ptr = c_loc(g_fptr)
      mm%fnodes = c_loc(g_fnodes)
      mm%c0 = c_loc(g_c0)
      mm%c1 = c_loc(g_c1)
      mm%zone = c_loc(g_zone)
   end subroutine pack_mesh

   ! ctrl_t -> MgpuCtrl (the bc lines included)
   subroutine pack_ctrl(ctrl, cc)
      type(ctrl_t),    intent(in)  :: ctrl
      type(mgpu_ctrl), intent(out) :: cc
      integer :: i, k
      character(len=32) :: form
      cc%rho = ctrl%rho
      cc%mu = ctrl%mu
      cc%alpha_u = ctrl%alpha_u
      cc%alpha_p = ctrl%alpha_p
      cc%outer_max = ctrl%outer_max
      cc%lin_max = ctrl%lin_max
      cc%outer_tol = ctrl%outer_tol
      cc%lin_tol = ctrl%lin_tol
      cc%conv_blend = ctrl%conv_blend
      cc%nonorth_corr = ctrl%nonorth_corr
      cc%ppe_precond = MGPU_PPE_JACOBI
      if (trim(ctrl%ppe_precond) == 'ic0') cc%ppe_precond = MGPU_PPE_IC0
      cc%mom_solver = MGPU_MOM_ILU0
      cc%transient = merge(1, 0, ctrl%transient)
      cc%time_scheme = ctrl%time_scheme
      cc%dt = ctrl%dt
      cc%n_time_max = ctrl%n_time_max
      cc%n_correct = ctrl%n_correct
      cc%body_force = ctrl%body_force
      cc%inlet_ramp = ctrl%inlet_ramp
      cc%precision = MGPU_PREC_FP64
      call get_environment_variable('MIXGPU_PRECISION', form)
      if (trim(form) == 'mixed') cc%precision = MGPU_PREC_MIXED
      if (trim(form) == 'fp64poly') cc%precision = MGPU_PREC_FP64_POLY
      cc%mixed_tol = 1.0e-4_c_double
      cc%n_outer_iter = ctrl%n_outer_iter
      cc%nbc = min(ctrl%nbc, MGPU_MAXBC)
      do i = 1, cc%nbc
         cc%bc(i)%zone = ctrl%bc(i)%zone
         cc%bc(i)%btype = ctrl%bc(i)%btype
         cc%bc(i)%uvel = ctrl%bc(i)%uvel
         cc%bc(i)%pval = ctrl%bc(i)%pval
         cc%bc(i)%mdot = ctrl%bc(i)%mdot
         cc%bc(i)%umean = ctrl%bc(i)%umean
         cc%bc(i)%uspan = ctrl%bc(i)%uspan
         cc%bc(i)%uorigin = ctrl%bc(i)%uorigin
         cc%bc(i)%uaxis = ctrl%bc(i)%uaxis
         cc%bc(i)%has_lid = merge(1, 0, ctrl%bc(i)%has_lid)
         cc%bc(i)%lid_dir = ctrl%bc(i)%lid_dir
         cc%bc(i)%lid_coord = ctrl%bc(i)%lid_coord
         cc%bc(i)%lid_vel = ctrl%bc(i)%lid_vel
         cc%bc(i)%ttype = ctrl%bc(i)%ttype
         cc%bc(i)%tval = ctrl%bc(i)%tval
         cc%bc(i)%qval = ctrl%bc(i)%qval
      end do
      ! the energy equation, which the reference's drivers always solve
      cc%energy = 1
      cc%boussinesq = merge(1, 0, ctrl%boussinesq)
      cc%cp = ctrl%cp
      cc%k_cond = ctrl%k_cond
      cc%tref = ctrl%tref
      cc%beta = ctrl%beta
      cc%gravity = ctrl%gravity
      cc%ntbc = 0
      do i = 1, cc%nbc
         do k = 1, ctrl%bc(i)%ntbc_plane
            if (cc%ntbc >= 32) exit
            cc%ntbc = cc%ntbc + 1
            cc%tbc(cc%ntbc)%bc = i - 1
            cc%tbc(cc%ntbc)%pdir = ctrl%bc(i)%tbc_pdir(k)
            cc%tbc(cc%ntbc)%pcoord = ctrl%bc(i)%tbc_pcoord(k)
            cc%tbc(cc%ntbc)%ttype = ctrl%bc(i)%tbc_pttype(k)
            cc%tbc(cc%ntbc)%tval = ctrl%bc(i)%tbc_ptval(k)
            cc%tbc(cc%ntbc)%qval = ctrl%bc(i)%tbc_pqval(k)
         end do
      end do
   end subroutine pack_ctrl

   ! The resident case of this mesh (made on first use or after the mesh changed).
   subroutine ensure_case(m, ctrl, ier)
      type(mesh_t), intent(in)  :: m
      type(ctrl_t), intent(in)  :: ctrl
      integer,      intent(out) :: ier
      type(mgpu_mesh) :: mm
      type(mgpu_ctrl) :: cc
      integer(c_int)  :: rc, bier
      ier = 0
      if (c_associated(g_case) .and. g_nfaces == m%nfaces .and. g_ncells == m%ncells) return
      call uns_gpu_release()
      call pack_mesh(m, mm)
      call pack_ctrl(ctrl, cc)
      rc = mgpu_case_create(mm, cc, g_case, bier)
      if (rc /= MGPU_OK) then
         write(*,'(a,i0,a,i0,2a)') '[uns-gpu] mgpu_case_create failed, status ', rc, ', build_bc ier ', &
                                   bier, ': ', trim(mgpu_error_message())
         g_case = c_null_ptr
         ier = GPU_IER
         return
      end if
      g_nfaces = m%nfaces
      g_ncells = m%ncells
   end subroutine ensure_case

   ! fields in, one run of the given kind (1 SIMPLE, 2 PISO, 3 PIMPLE), fields out
   subroutine run_case(kind, nsteps, fld, ier)
      integer,                intent(in)    :: kind, nsteps
      type(fields_t), target, intent(inout) :: fld
      integer,                intent(out)   :: ier
      integer(c_int) :: rc, nrec, cier
      type(c_ptr) :: uo, uoo, to, too
      ier = 0
      uo = c_null_ptr
      uoo = c_null_ptr
      to = c_null_ptr
      too = c_null_ptr
      if (kind /= 1 .and. allocated(fld%u_old)) uo = c_loc(fld%u_old)
      if (kind /= 1 .and. allocated(fld%u_old_old)) uoo = c_loc(fld%u_old_old)
      if (kind /= 1 .and. allocated(fld%T_old)) to = c_loc(fld%T_old)
      if (kind /= 1 .and. allocated(fld%T_old_old)) too = c_loc(fld%T_old_old)
      rc = mgpu_fields_upload(g_case, c_loc(fld%u), c_loc(fld%p), c_loc(fld%flux), uo, uoo)
      if (rc == MGPU_OK) rc = mgpu_temperature_upload(g_case, c_loc(fld%T), to, too)
      if (rc == MGPU_OK) then
         select case (kind)
         case (1)
            ! run and download in one call: gp, gu and apc are copied during the
            ! last iteration's pressure solve when their arrays are page-locked
            rc = mgpu_simple_run_fields(g_case, int(nsteps, c_int), c_null_ptr, 0_c_int, nrec, cier, &
                                        c_loc(fld%u), c_loc(fld%p), c_loc(fld%flux), c_loc(fld%gp), &
                                        c_loc(fld%gu), c_loc(fld%apc))
         case (2)
            rc = mgpu_piso_run(g_case, int(nsteps, c_int), c_null_ptr, 0_c_int, nrec, cier)
         case default
            rc = mgpu_pimple_run(g_case, int(nsteps, c_int), c_null_ptr, 0_c_int, nrec, cier)
         end select
      end if
      if (rc == MGPU_OK .and. kind /= 1) rc = mgpu_fields_download(g_case, c_loc(fld%u), c_loc(fld%p), &
                                                   c_loc(fld%flux), c_loc(fld%gp), c_loc(fld%gu), c_loc(fld%apc))
      if (rc == MGPU_OK) rc = mgpu_temperature_download(g_case, c_loc(fld%T), c_loc(fld%gt))
      if (rc /= MGPU_OK) then
         write(*,'(a,i0,2a)') '[uns-gpu] run failed, status ', rc, ': ', trim(mgpu_error_message())
         ier = GPU_IER
         return
      end if
      ier = cier
   end subroutine run_case

   ! simple_run (mod_uns_simple.f90:88-288): conn, g and bcs are built on the
   ! device from m and ctrl; the optional nsteps caps the outer iterations.
   subroutine simple_run_gpu(m, conn, g, ctrl, bcs, fld, ier, nsteps)
      type(mesh_t),           intent(in)    :: m
      type(conn_t),           intent(in)    :: conn
      type(geom_t),           intent(in)    :: g
      type(ctrl_t),           intent(in)    :: ctrl
      type(bc_t),             intent(in)    :: bcs
      type(fields_t), target, intent(inout) :: fld
      integer,                intent(out)   :: ier
      integer, optional,      intent(in)    :: nsteps
      integer :: n
      call ensure_case(m, ctrl, ier)
      if (ier /= 0) return
      n = 0
      if (present(nsteps)) n = nsteps
      call run_case(1, n, fld, ier)
   end subroutine simple_run_gpu

   ! piso_run_mpi at one rank (mod_uns_simple_mpi.f90:298-571): the global mesh
   ! m_g is the rank's mesh; lm, hi, part and fld_g are not needed on one GPU.
   subroutine piso_run_gpu(lm, hi, ctrl, bcs, fld, vtu_prefix, m_g, c_g, g_g, part, fld_g, ier)
      type(local_mesh_t),     intent(in)    :: lm
      type(halo_info_t),      intent(in)    :: hi
      type(ctrl_t),           intent(in)    :: ctrl
      type(bc_t),             intent(in)    :: bcs
      type(fields_t), target, intent(inout) :: fld
      character(len=*),       intent(in)    :: vtu_prefix
      type(mesh_t),           intent(in)    :: m_g
      type(conn_t),           intent(in)    :: c_g
      type(geom_t),           intent(in)    :: g_g
      integer,                intent(in)    :: part(:)
      type(fields_t),         intent(inout) :: fld_g
      integer,                intent(out)   :: ier
      call ensure_case(m_g, ctrl, ier)
      if (ier /= 0) return
      call run_case(2, 0, fld, ier)
   end subroutine piso_run_gpu

   ! pimple_run_mpi at one rank (mod_uns_simple_mpi.f90:580-850)
   subroutine pimple_run_gpu(lm, hi, ctrl, bcs, fld, vtu_prefix, m_g, c_g, g_g, part, fld_g, ier)
      type(local_mesh_t),     intent(in)    :: lm
      type(halo_info_t),      intent(in)    :: hi
      type(ctrl_t),           intent(in)    :: ctrl
      type(bc_t),             intent(in)    :: bcs
      type(fields_t), target, intent(inout) :: fld
      character(len=*),       intent(in)    :: vtu_prefix
      type(mesh_t),           intent(in)    :: m_g
      type(conn_t),           intent(in)    :: c_g
      type(geom_t),           intent(in)    :: g_g
      integer,                intent(in)    :: part(:)
      type(fields_t),         intent(inout) :: fld_g
      integer,                intent(out)   :: ier
      call ensure_case(m_g, ctrl, ier)
      if (ier /= 0) return
      call run_case(3, 0, fld, ier)
   end subroutine pimple_run_gpu

   ! Free the resident case (call once at finalisation).
   subroutine uns_gpu_release()
      integer(c_int) :: rc
      if (c_associated(g_case)) rc = mgpu_case_destroy(g_case)
      g_case = c_null_ptr
      g_nfaces = -1
      g_ncells = -1
   end subroutine uns_gpu_release

end module mod_uns_gpu
