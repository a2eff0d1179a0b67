!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
!   The host's compile-time configuration as a simp_params: every switch  !
!   and constant the GPU path reads is taken from the module variable of  !
!   the same name in globals.f90 (switches :58-187, max_ind_int :21-25)   !
!   and data_variables.f90 (hsml_multiplicity :105, constants :153-180,   !
!   max_hsml :90, dt :66), so a SIMP build with other PARAMETERs runs      !
!   them on the GPU too.  Only what the reference has no variable for      !
!   keeps the library's value: the wind and current, hard-coded in        !
!   wind_forcing.f90:36-37 and water_drag.f90:36-37 (the library's         !
!   reference defaults are those values), and the GPU's own settings      !
!   (precision, cell-list skin, wind kind, mass_from_area).  Compile      !
!   after simp_gpu_mod.f90 and the reference's modules.                  !
!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!!
module simp_host_params_mod

    use, intrinsic :: iso_c_binding
    use simp_gpu_mod

    implicit none

contains

subroutine simp_params_from_host(prm)

    use globals
    use data_variables

    type(simp_params), intent(out) :: prm

    ! the fields the reference has no variable for
    call simp_params_reference_default(prm)

    ! algorithm switches (globals.f90:58-155)
    prm%int_algorithm  = int(int_algorithm, c_int32_t)
    prm%nnps_algorithm = int(nnps_algorithm, c_int32_t)
    prm%sle            = int(sle, c_int32_t)
    prm%tse            = int(tse, c_int32_t)
    prm%rheology       = int(rheology, c_int32_t)
    prm%eos_alg        = int(eos_alg, c_int32_t)
    prm%pa_sph         = int(pa_sph, c_int32_t)
    prm%skf            = int(skf, c_int32_t)
    prm%den_alg        = int(den_alg, c_int32_t)
    prm%bfa            = int(bfa, c_int32_t)
    prm%art_visc_alg   = int(art_visc_alg, c_int32_t)

    ! logical switches (globals.f90:180-187)
    prm%viscosity           = merge(1_c_int32_t, 0_c_int32_t, viscosity)
    prm%pressure_force      = merge(1_c_int32_t, 0_c_int32_t, pressure_force)
    prm%wind_force          = merge(1_c_int32_t, 0_c_int32_t, wind_force)
    prm%water_force         = merge(1_c_int32_t, 0_c_int32_t, water_force)
    prm%boundary_pressure   = merge(1_c_int32_t, 0_c_int32_t, boundary_pressure)
    prm%boundary_friction   = merge(1_c_int32_t, 0_c_int32_t, boundary_friction)
    prm%artificial_visc     = merge(1_c_int32_t, 0_c_int32_t, artificial_visc)
    prm%xsph_regularization = merge(1_c_int32_t, 0_c_int32_t, xsph_regularization)

    ! capacities and multiplicities
    prm%max_ind_int       = int(max_ind_int, c_int32_t)
    prm%hsml_multiplicity = int(hsml_multiplicity, c_int32_t)

    ! material constants (data_variables.f90:153-180)
    prm%P_star    = P_star
    prm%c_eos     = c_eos
    prm%e         = e
    prm%delta_min = delta_min
    prm%k_t       = k_t
    prm%rho_ice   = rho_ice
    prm%rho_air   = rho_air
    prm%rho_water = rho_water
    prm%c_wind    = c_wind
    prm%c_water   = c_water
    prm%b_length  = b_length
    prm%kappa_n   = kappa_n
    prm%kappa_t   = kappa_t
    prm%alpha     = alpha
    prm%zeta_max  = zeta_max
    prm%eta_max   = eta_max
    prm%phi       = phi
    prm%xi        = xi
    prm%Y         = Y
    prm%nu        = nu
    prm%alpha_pi  = alpha_pi
    prm%beta_pi   = beta_pi
    prm%chi       = chi

    ! integrator state set by initialize (initialize.f90:191, 199)
    prm%max_hsml = max_hsml
    prm%dt       = dt

end subroutine simp_params_from_host

end module simp_host_params_mod
