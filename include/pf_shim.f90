! ISO_C_BINDING interface to libpipeflow_b200 (include/pipeflow_b200.h) for
! the reference's Fortran drivers: main.f90, newton.f90 / NewtonHook.f90 /
! GMRESm.f90 and arnoldi.f.  It keeps the reference's calling conventions:
! the module arrays (vel_ur%Re(i_N, 0:i_H1) and so on, n fastest) pass
! straight through, and a nonzero status becomes the reference's `stop`
! (timestep.f90:93,117,222-240; velocity.f90:166-168) via pf_check.
!
! Every entry point of the header binds the same way: plain pointers, sizes
! and double/int values; opaque handles (pf_ctx*, pf_coll*, pf_lumesh*) are
! type(c_ptr), value.  Link with
!    -L<repo>/softx-d-17-00015_b200/pipeflow -lpipeflow_b200 -lcudart
module pf_shim
   use iso_c_binding
   implicit none

   integer(c_int), parameter :: PF_OK = 0, PF_PREC_FP64 = 0, PF_PREC_MIXED = 1
   integer(c_int), parameter :: PF_ERR_CONVERGE = -6

   ! typedef struct pf_config (parameters.f90:15-51 as run-time values)
   type, bind(c) :: pf_config
      integer(c_int)  :: N, K, M, Mp
      real(c_double)  :: Re, alpha, dt, implicit, dterr, courant, maxdt
      integer(c_int)  :: const_flux, mirrorsym, shiftrefl, shiftrott
      type(c_ptr)     :: r                ! c_null_ptr = default mesh (meshs.f90:90-99)
      integer(c_int)  :: precision        ! PF_PREC_FP64 = the reference's arithmetic
   end type

   ! typedef struct pf_tim_state (timestep.f90:12-21)
   type, bind(c) :: pf_tim_state
      real(c_double)  :: t, dt, dterr, corr_dt, cfl_dt
      integer(c_int)  :: it, step, cfl_dir, new_dt, pcn
   end type

   type(c_ptr), save :: pf = c_null_ptr   ! the context: module state of one run

   interface
      ! ------------------------------------------------------- context
      type(c_ptr) function pf_last_error() bind(c)
         import
      end function
      integer(c_int) function pf_ctx_create(cfg, device, out) bind(c)
         import
         type(pf_config), intent(in) :: cfg
         integer(c_int), value :: device
         type(c_ptr), intent(out) :: out
      end function
      integer(c_int) function pf_ctx_destroy(ctx) bind(c)
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_ctx_sync(ctx) bind(c)
         import
         type(c_ptr), value :: ctx
      end function
      ! ----------------------------------------------------- velocity.f90
      integer(c_int) function pf_vel_matrices(ctx) bind(c)          ! velocity.f90:120-146
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_vel_set_state(ctx, rr, ri, tr, ti, zr, zi) bind(c)
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: rr(*), ri(*), tr(*), ti(*), zr(*), zi(*)
      end function
      integer(c_int) function pf_vel_get_state(ctx, rr, ri, tr, ti, zr, zi) bind(c)
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: rr(*), ri(*), tr(*), ti(*), zr(*), zi(*)
      end function
      integer(c_int) function pf_vel_imposesym(ctx) bind(c)         ! velocity.f90:61-74
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_vel_transform(ctx) bind(c)         ! velocity.f90:304-317
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_vel_nonlinear(ctx) bind(c)         ! velocity.f90:323-335
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_vel_predictor(ctx) bind(c)         ! velocity.f90:400-410
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_vel_corrector(ctx) bind(c)         ! velocity.f90:416-432
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_vel_maxtstep(ctx) bind(c)          ! velocity.f90:438-481
         import
         type(c_ptr), value :: ctx
      end function
      ! the loop body of main.f90:20-44 (one CUDA graph replay per pass)
      integer(c_int) function pf_timestep(ctx, ncorr) bind(c)
         import
         type(c_ptr), value :: ctx
         integer(c_int), intent(out) :: ncorr
      end function
      ! the loop body of steporbit, newton.f90:740-762 (one corrector per step)
      integer(c_int) function pf_steporbit(ctx, nsteps) bind(c)
         import
         type(c_ptr), value :: ctx
         integer(c_int), value :: nsteps
      end function
      ! ----------------------------------------------------- timestep.f90
      integer(c_int) function pf_tim_get(ctx, s) bind(c)
         import
         type(c_ptr), value :: ctx
         type(pf_tim_state), intent(out) :: s
      end function
      integer(c_int) function pf_tim_set(ctx, s) bind(c)
         import
         type(c_ptr), value :: ctx
         type(pf_tim_state), intent(in) :: s
      end function
      integer(c_int) function pf_tim_check_cgce(ctx) bind(c)        ! timestep.f90:214-253
         import
         type(c_ptr), value :: ctx
      end function
      integer(c_int) function pf_tim_new_tstep(ctx) bind(c)         ! timestep.f90:259-278
         import
         type(c_ptr), value :: ctx
      end function
      ! ---------------------------------------------------- variables.f90
      integer(c_int) function pf_vel_coll(ctx, which, out) bind(c)  ! the module fields as handles
         import
         type(c_ptr), value :: ctx
         integer(c_int), value :: which
         type(c_ptr), intent(out) :: out
      end function
      integer(c_int) function pf_var_coll_shift(dt, dz, a, b) bind(c)   ! variables.f90:487-528
         import
         real(c_double), value :: dt, dz
         type(c_ptr), value :: a, b
      end function
      ! ------------------------------------------------------ io.f90 metrics
      integer(c_int) function pf_diag_energy(ctx, E) bind(c)        ! io.f90:501-514
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: E
      end function
      integer(c_int) function pf_diag_friction(ctx, Ub, Uc, utau) bind(c)   ! io.f90:627-639
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(out) :: Ub, Uc, utau
      end function
      ! ------------------------------------------- newton.f90 (device vectors)
      ! x and y are DEVICE vectors of 8 + 6*i_N*(i_H1+1) doubles
      integer(c_int) function pf_orbit_set_scales(ctx, scaleU, scaleT) bind(c)
         import
         type(c_ptr), value :: ctx
         real(c_double), intent(in) :: scaleU(3)
         real(c_double), value :: scaleT
      end function
      integer(c_int) function pf_orbit_step(ctx, ndts, x, y) bind(c)     ! newton.f90:721-831
         import
         type(c_ptr), value :: ctx, x, y
         integer(c_int), value :: ndts
      end function
      integer(c_int) function pf_orbit_dotprod(ctx, n_, a, b, d) bind(c) ! newton.f90:652-672
         import
         type(c_ptr), value :: ctx, a, b
         integer(c_int), value :: n_
         real(c_double), intent(out) :: d
      end function
      integer(c_int) function pf_orbit_shiftdir(ctx, i, x, s) bind(c)    ! newton.f90:533-561
         import
         type(c_ptr), value :: ctx, x, s
         integer(c_int), value :: i
      end function
      ! ---------------------------------------------------- io.f90 state files
      integer(c_int) function pf_io_save_state(ctx, path) bind(c)        ! io.f90:303-378
         import
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
      end function
      integer(c_int) function pf_io_load_state(ctx, path, flags, changes) bind(c)   ! io.f90:98-226
         import
         type(c_ptr), value :: ctx
         character(kind=c_char), intent(in) :: path(*)
         integer(c_int), value :: flags
         integer(c_int), intent(out) :: changes
      end function
      ! -------------------------------------- the var_null(flag) plug-in hook
      integer(c_int) function pf_util_set(ctx, kind, params, np) bind(c)
         import
         type(c_ptr), value :: ctx
         integer(c_int), value :: kind, np
         real(c_double), intent(in) :: params(*)
      end function
      integer(c_int) function pf_util_set_callback(ctx, fn, user) bind(c)
         import
         type(c_ptr), value :: ctx, user
         type(c_funptr), value :: fn
      end function
   end interface

contains

   ! nonzero status -> the reference's error behaviour: print the message, stop
   subroutine pf_check(s)
      integer(c_int), intent(in) :: s
      character(kind=c_char), pointer :: msg(:)
      integer :: n
      if (s == PF_OK) return
      call c_f_pointer(pf_last_error(), msg, [512])
      n = 0
      do while (n < 512)
         if (msg(n + 1) == c_null_char) exit
         n = n + 1
      end do
      print*, 'pipeflow_b200: ', msg(1:n)
      stop 'pipeflow_b200 error'
   end subroutine pf_check

end module pf_shim
