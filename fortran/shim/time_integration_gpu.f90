!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
!   Drop-in replacement of SIMP's time_integration (integration/          !
!   time_integration.f90:6-71) that runs the predictor-corrector on       !
!   the GPU.  State goes up once, steps stay resident, and the module     !
!   globals are refreshed only when output is due (save_step).            !
!   Link with -lsimp_gpu; compile simp_gpu_mod.f90 and                   !
!   simp_host_params.f90 first.                                            !
!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
subroutine time_integration

    use, intrinsic :: iso_c_binding
    use globals
    use data_variables
    use simp_gpu_mod
    use simp_host_params_mod

    implicit none

    type(simp_params) :: prm
    type(c_ptr) :: ctx
    integer(c_int32_t) :: rc, nchunk
    REAL(kind=8) :: last_save, t_gpu, dt_gpu

    ! the host's switches and constants (globals.f90, data_variables.f90)
    call simp_params_from_host(prm)

    rc = simp_gpu_create(prm, int(maxn, c_int32_t), int(maxnb, c_int32_t), ctx)
    call simp_gpu_stop(ctx, rc)
    rc = simp_gpu_set_state(ctx, int(ntotal, c_int32_t), x, vx, mass, rho,   &
                            hsml, A, h, int(ntotalb, c_int32_t), xb, massb,  &
                            dt, current_time)
    call simp_gpu_stop(ctx, rc)
    rc = simp_gpu_keep_diag(ctx, 1_c_int32_t)

    last_save = - save_step
    itimestep = 0
    DO WHILE (current_time .LT. integration_time)
        ! advance to the next output time (one step when dt is unknown)
        nchunk = 1
        IF (dt .GT. 0.) nchunk = int(max(1.d0, min(dble(print_step),        &
                    (save_step + last_save - current_time) / dt)), c_int32_t)
        rc = simp_gpu_step(ctx, nchunk, t_gpu, dt_gpu)
        call simp_gpu_stop(ctx, rc)
        itimestep = itimestep + nchunk
        current_time = t_gpu
        dt = dt_gpu
        IF ( current_time .GT. save_step + last_save ) THEN
            rc = simp_gpu_get_state(ctx, x, vx, mass, rho, hsml, A, h, dt_gpu, t_gpu)
            call simp_gpu_stop(ctx, rc)
            rc = simp_gpu_get_diag(ctx, epsilon_11, epsilon_12, epsilon_22,  &
                                   zeta, eta, p, sigma_11, sigma_12, sigma_22)
            call simp_gpu_stop(ctx, rc)
            call output
            last_save = current_time
        ENDIF
    ENDDO

    rc = simp_gpu_get_state(ctx, x, vx, mass, rho, hsml, A, h, dt_gpu, t_gpu)
    rc = simp_gpu_destroy(ctx)

end subroutine time_integration
