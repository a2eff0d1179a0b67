!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
!   ISO_C_BINDING interface to libsimp_gpu.so (include/simp_gpu.h).       !
!                                                                          !
!   SIMP's module globals (data_variables.f90) are contiguous column-     !
!   major arrays, so x(dim,maxn) is passed as is: it is the interleaved   !
!   2*n layout the C ABI expects.  Status codes follow simp_gpu.h; the    !
!   helper simp_gpu_stop prints the library's banner and STOPs, as the    !
!   reference does on the same conditions.                                !
!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
module simp_gpu_mod
    use, intrinsic :: iso_c_binding
    implicit none

    integer(c_int32_t), parameter :: SIMP_OK = 0

    ! Mirror of struct simp_params (same member order and types).
    type, bind(C) :: simp_params
        integer(c_int32_t) :: int_algorithm, nnps_algorithm, sle, tse,      &
                              rheology, eos_alg, pa_sph, skf, den_alg, bfa, &
                              viscosity, pressure_force, wind_force,       &
                              water_force, boundary_pressure,              &
                              boundary_friction, mass_from_area,           &
                              max_ind_int, hsml_multiplicity, wind_kind,   &
                              precision, reserved0
        real(c_double) :: P_star, c_eos, e, delta_min, k_t,                 &
                          rho_ice, rho_air, rho_water, c_wind, c_water,     &
                          b_length, kappa_n, kappa_t, alpha,                &
                          wind_u, wind_v, current_u, current_v,             &
                          vortex_x, vortex_y, vortex_umax, vortex_radius,   &
                          dt, max_hsml, skin, zeta_max, eta_max, phi,       &
                          xi, Y, nu
        integer(c_int32_t) :: artificial_visc, xsph_regularization,         &
                              art_visc_alg, reserved1
        real(c_double) :: alpha_pi, beta_pi, chi
    end type simp_params

    ! Mirror of struct simp_forcing (per-basin wind of a batch).
    type, bind(C) :: simp_forcing
        integer(c_int32_t) :: wind_kind, reserved0
        real(c_double) :: wind_u, wind_v, vortex_x, vortex_y, vortex_umax, vortex_radius
    end type simp_forcing

    interface
        subroutine simp_params_reference_default(p) bind(C, name="simp_params_reference_default")
            import :: simp_params
            type(simp_params), intent(out) :: p
        end subroutine

        function simp_gpu_create(p, maxn, maxnb, ctx) bind(C, name="simp_gpu_create")
            import :: simp_params, c_int32_t, c_ptr
            type(simp_params), intent(in) :: p
            integer(c_int32_t), value :: maxn, maxnb
            type(c_ptr), intent(out) :: ctx
            integer(c_int32_t) :: simp_gpu_create
        end function

        function simp_gpu_destroy(ctx) bind(C, name="simp_gpu_destroy")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int32_t) :: simp_gpu_destroy
        end function

        function simp_gpu_set_state(ctx, ntotal, x, vx, mass, rho, hsml, A, h, &
                                    ntotalb, xb, massb, dt, current_time)      &
                                    bind(C, name="simp_gpu_set_state")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: ntotal, ntotalb
            real(c_double), intent(in) :: x(*), vx(*), mass(*), rho(*),        &
                                          hsml(*), A(*), h(*), xb(*), massb(*)
            real(c_double), value :: dt, current_time
            integer(c_int32_t) :: simp_gpu_set_state
        end function

        function simp_gpu_get_state(ctx, x, vx, mass, rho, hsml, A, h, dt,    &
                                    current_time) bind(C, name="simp_gpu_get_state")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: x(*), vx(*), mass(*), rho(*),       &
                                           hsml(*), A(*), h(*), dt, current_time
            integer(c_int32_t) :: simp_gpu_get_state
        end function

        function simp_gpu_nnps(ctx, nip, p_i, p_j, r_ij, hsml_ij, cap,         &
                               bnip, bp_i, bp_j, br_ij, bcap)                  &
                               bind(C, name="simp_gpu_nnps")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            integer(c_int32_t), intent(out) :: nip, p_i(*), p_j(*), bnip,      &
                                               bp_i(*), bp_j(*)
            real(c_double), intent(out) :: r_ij(*), hsml_ij(*), br_ij(*)
            integer(c_int32_t), value :: cap, bcap
            integer(c_int32_t) :: simp_gpu_nnps
        end function

        function simp_gpu_single_step(ctx, current_time, dxdt, dvxdt, dhdt,   &
                                      dAdt) bind(C, name="simp_gpu_single_step")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: current_time
            real(c_double), intent(out) :: dxdt(*), dvxdt(*), dhdt(*), dAdt(*)
            integer(c_int32_t) :: simp_gpu_single_step
        end function

        function simp_gpu_get_diag(ctx, eps11, eps12, eps22, zeta, eta, p,    &
                                   sig11, sig12, sig22)                        &
                                   bind(C, name="simp_gpu_get_diag")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: eps11(*), eps12(*), eps22(*),       &
                                           zeta(*), eta(*), p(*), sig11(*),    &
                                           sig12(*), sig22(*)
            integer(c_int32_t) :: simp_gpu_get_diag
        end function

        function simp_gpu_keep_diag(ctx, keep) bind(C, name="simp_gpu_keep_diag")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: keep
            integer(c_int32_t) :: simp_gpu_keep_diag
        end function

        function simp_gpu_sum_density(ctx, rho_out) bind(C, name="simp_gpu_sum_density")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            real(c_double), intent(out) :: rho_out(*)
            integer(c_int32_t) :: simp_gpu_sum_density
        end function

        function simp_gpu_step(ctx, nsteps, current_time, dt) bind(C, name="simp_gpu_step")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: nsteps
            real(c_double), intent(out) :: current_time, dt
            integer(c_int32_t) :: simp_gpu_step
        end function

        function simp_gpu_set_forcing(ctx, f) bind(C, name="simp_gpu_set_forcing")
            import :: c_ptr, c_int32_t, simp_forcing
            type(c_ptr), value :: ctx
            type(simp_forcing), intent(in) :: f
            integer(c_int32_t) :: simp_gpu_set_forcing
        end function

        ! b_normal(2, ntotalb) of the walls, for the Wang boundary force.
        function simp_gpu_set_wall_normals(ctx, ntotalb, b_normal)         &
                bind(C, name="simp_gpu_set_wall_normals")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: ntotalb
            real(c_double), intent(in) :: b_normal(*)
            integer(c_int32_t) :: simp_gpu_set_wall_normals
        end function

        ! The reference's output files (output.f90:61-78), appended from the
        ! device state; folder is a NUL-terminated path.
        function simp_csv_create_output(folder)                            &
                bind(C, name="simp_csv_create_output")
            import :: c_int32_t, c_char
            character(kind=c_char), intent(in) :: folder(*)
            integer(c_int32_t) :: simp_csv_create_output
        end function

        function simp_gpu_write_output(ctx, folder)                        &
                bind(C, name="simp_gpu_write_output")
            import :: c_ptr, c_int32_t, c_char
            type(c_ptr), value :: ctx
            character(kind=c_char), intent(in) :: folder(*)
            integer(c_int32_t) :: simp_gpu_write_output
        end function

        ! Batches of basins advanced together by simp_gpu_step.
        function simp_gpu_create_batch(p, maxn, maxnb, max_instances, ctx)  &
                                       bind(C, name="simp_gpu_create_batch")
            import :: simp_params, c_int32_t, c_ptr
            type(simp_params), intent(in) :: p
            integer(c_int32_t), value :: maxn, maxnb, max_instances
            type(c_ptr), intent(out) :: ctx
            integer(c_int32_t) :: simp_gpu_create_batch
        end function

        function simp_gpu_batch_add(ctx, f, ntotal, x, vx, mass, rho, hsml,    &
                                    A, h, ntotalb, xb, massb, slot)            &
                                    bind(C, name="simp_gpu_batch_add")
            import :: c_ptr, c_int32_t, c_double, simp_forcing
            type(c_ptr), value :: ctx
            type(simp_forcing), intent(in) :: f
            integer(c_int32_t), value :: ntotal, ntotalb
            real(c_double), intent(in) :: x(*), vx(*), mass(*), rho(*),        &
                                          hsml(*), A(*), h(*), xb(*), massb(*)
            integer(c_int32_t), intent(out) :: slot
            integer(c_int32_t) :: simp_gpu_batch_add
        end function

        function simp_gpu_batch_remove(ctx, slot) bind(C, name="simp_gpu_batch_remove")
            import :: c_ptr, c_int32_t
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: slot
            integer(c_int32_t) :: simp_gpu_batch_remove
        end function

        function simp_gpu_batch_get_state(ctx, slot, x, vx, mass, rho, hsml,   &
                                          A, h, current_time)                  &
                                          bind(C, name="simp_gpu_batch_get_state")
            import :: c_ptr, c_int32_t, c_double
            type(c_ptr), value :: ctx
            integer(c_int32_t), value :: slot
            real(c_double), intent(out) :: x(*), vx(*), mass(*), rho(*),       &
                                           hsml(*), A(*), h(*), current_time
            integer(c_int32_t) :: simp_gpu_batch_get_state
        end function

        function simp_gpu_last_error_c(ctx) bind(C, name="simp_gpu_last_error")
            import :: c_ptr
            type(c_ptr), value :: ctx
            type(c_ptr) :: simp_gpu_last_error_c
        end function
    end interface

contains

    ! Print the library's message and STOP (the reference's reaction to the
    ! same conditions, e.g. nnps.f90:132-139).
    subroutine simp_gpu_stop(ctx, rc)
        type(c_ptr), intent(in) :: ctx
        integer(c_int32_t), intent(in) :: rc
        character(kind=c_char), pointer :: msg(:)
        integer :: k
        type(c_ptr) :: cmsg
        if (rc .EQ. SIMP_OK) return
        cmsg = simp_gpu_last_error_c(ctx)
        call c_f_pointer(cmsg, msg, [4096])
        WRITE (*,*) '******************************************************'
        WRITE (*,'(A,I3)') ' simp_gpu error code ', rc
        k = 1
        do while (msg(k) .NE. c_null_char .AND. k .LT. 4096)
            k = k + 1
        enddo
        WRITE (*,*) msg(1:k-1)
        WRITE (*,*) '******************************************************'
        STOP
    end subroutine simp_gpu_stop

end module simp_gpu_mod
