!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
!   Drop-in replacement of SIMP's single_step (integration/               !
!   single_step.f90:5-109) for a host that keeps its own integrator       !
!   (time_integration.f90) on the CPU.  Every call hands the module        !
!   state to the library and reads the rates dxdt, dvxdt, dhdt, dAdt      !
!   back.  While the state continues the one of the previous call (same   !
!   particles, walls and hsml, moved less than a cell) the library keeps  !
!   its sort and neighbour lists, so a call costs the two copies and one  !
!   right-hand side.  Link with -lsimp_gpu; compile simp_gpu_mod.f90 and  !
!   simp_host_params.f90 first, and leave the reference's single_step.f90 out of the build.    !
!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
module simp_single_step_ctx
    use, intrinsic :: iso_c_binding
    implicit none
    type(c_ptr), save :: ss_ctx = c_null_ptr
end module simp_single_step_ctx

subroutine single_step

    use, intrinsic :: iso_c_binding
    use globals
    use data_variables
    use simp_gpu_mod
    use simp_host_params_mod
    use simp_single_step_ctx

    implicit none

    type(simp_params) :: prm
    integer(c_int32_t) :: rc

    IF (.NOT. c_associated(ss_ctx)) THEN
        ! the host's switches and constants (globals.f90, data_variables.f90)
        call simp_params_from_host(prm)
        rc = simp_gpu_create(prm, int(maxn, c_int32_t), int(maxnb, c_int32_t), ss_ctx)
        call simp_gpu_stop(ss_ctx, rc)
    ENDIF
    rc = simp_gpu_set_state(ss_ctx, int(ntotal, c_int32_t), x, vx, mass, rho,  &
                            hsml, A, h, int(ntotalb, c_int32_t), xb, massb,    &
                            dt, current_time)
    call simp_gpu_stop(ss_ctx, rc)
    rc = simp_gpu_single_step(ss_ctx, current_time, dxdt, dvxdt, dhdt, dAdt)
    call simp_gpu_stop(ss_ctx, rc)

end subroutine single_step
