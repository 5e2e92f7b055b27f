! The reference's run loop on the device.  Compiled together with the
! reference's own modules (parameters, variables, velocity, timestep, io) and
! include/pf_shim.f90, it replaces the body of main.f90's time loop
! (main.f90:20-44) and of steporbit (newton.f90:740-762) while the drivers
! keep their control flow, output and module variables:
!
!    main.f90, after initialise():   call pf_drive_init()
!    main.f90, the loop body:        call pf_drive_step()
!    newton.f90, steporbit's loop:   call pf_drive_steporbit(ndts)
!    main.f90, cleanup():            call pf_drive_free()
!
! The module arrays stay the reference's (vel_ur%Re(i_N, 0:i_H1), n fastest);
! the device state is authoritative while stepping, and the host arrays are
! refreshed exactly when io_write2files (io.f90:67-85) will read them, every
! i_save_rate2 steps, and at the end.
module pf_drive
   use iso_c_binding
   use pf_shim
   use parameters
   use timestep
   use velocity
   implicit none

contains

   ! context from the compile-time parameters (parameters.f90:15-51), the
   ! state io_load_state left in vel_ur/ut/uz, and vel_matrices
   subroutine pf_drive_init()
      type(pf_config) :: cfg
      type(pf_tim_state) :: ts
      cfg = pf_config(i_N, i_K, i_M, i_Mp, d_Re, d_alpha, d_timestep, d_implicit, d_dterr, &
                      d_courant, d_maxdt, merge(1, 0, b_const_flux), merge(1, 0, b_mirrorsym), &
                      merge(1, 0, b_shiftrefl), merge(1, 0, b_shiftrott), c_null_ptr, PF_PREC_FP64)
      call pf_check(pf_ctx_create(cfg, -1_c_int, pf))
      call pf_check(pf_vel_set_state(pf, vel_ur%Re, vel_ur%Im, vel_ut%Re, vel_ut%Im, &
                                         vel_uz%Re, vel_uz%Im))
      call pf_check(pf_tim_get(pf, ts))
      ts%t = tim_t
      ts%dt = tim_dt
      ts%step = tim_step
      call pf_check(pf_tim_set(pf, ts))
      call pf_check(pf_vel_matrices(pf))
   end subroutine pf_drive_init

   ! copy the device state back into the module arrays
   subroutine pf_drive_to_host()
      call pf_check(pf_vel_get_state(pf, vel_ur%Re, vel_ur%Im, vel_ut%Re, vel_ut%Im, &
                                         vel_uz%Re, vel_uz%Im))
   end subroutine pf_drive_to_host

   ! one pass of main.f90:20-44: imposesym, nonlinear terms, [new dt],
   ! predictor, correctors until tim_check_cgce says converged; the
   ! timestep module's counters come back to the host
   subroutine pf_drive_step()
      type(pf_tim_state) :: ts
      integer(c_int) :: ncorr, s
      s = pf_timestep(pf, ncorr)
      call pf_check(pf_tim_get(pf, ts))
      tim_t = ts%t
      tim_dt = ts%dt
      tim_step = ts%step
      tim_new_dt = ts%new_dt /= 0
      if (s == PF_ERR_CONVERGE) then
         ! tim_check_cgce's aborts end the run as the reference's do
         ! (tim_step = i_maxtstep-1, timestep.f90:222-240)
         print*, 'pipeflow_b200: corrector check aborted the run'
         tim_step = i_maxtstep - 1
         s = PF_OK
      end if
      call pf_check(s)
      if (modulo(tim_step, i_save_rate2) == 0) call pf_drive_to_host()
   end subroutine pf_drive_step

   ! steporbit's ndts steps (newton.f90:740-762: one corrector each); the
   ! caller's var_coll_shift and rtz2vec then read the refreshed module arrays
   subroutine pf_drive_steporbit(ndts)
      integer, intent(in) :: ndts
      type(pf_tim_state) :: ts
      call pf_check(pf_steporbit(pf, int(ndts, c_int)))
      call pf_check(pf_tim_get(pf, ts))
      tim_t = ts%t
      tim_step = ts%step
      call pf_drive_to_host()
   end subroutine pf_drive_steporbit

   subroutine pf_drive_free()
      call pf_drive_to_host()
      call pf_check(pf_ctx_destroy(pf))
      pf = c_null_ptr
   end subroutine pf_drive_free

end module pf_drive
