! feram_gpu_iface.F90 -- ISO_C_BINDING view of include/feram_gpu.h for feram.
!
! Module feram_gpu_c     : bind(C) interfaces and the interoperable mirrors of
!                          fg_params / fg_energy / fg_average.
! Module feram_gpu_dropin: subroutines with the reference's names and argument
!                          lists (nose_poincare(p,c,e), leapfrog(p,c,e,i_step),
!                          mirror_force_mirror(p,c,e)) that keep the state on the
!                          device and refresh the host copies in Coord_type only
!                          where the reference's driver reads them.
!
! This file is delivered as source: the build image has no Fortran compiler.
! Its calls are exercised by feram_b200/host/feram_driver.cpp, which replays
! molecular_dynamics (molecular-dynamics.F:10-160) through the same C-ABI.
module feram_gpu_c
  use, intrinsic :: iso_c_binding
  implicit none
  integer(c_int), parameter :: FG_OK = 0, FG_PREC_FP64 = 0, FG_PREC_MIXED = 1
  integer(c_int), parameter :: FG_RELAXOR_MAX = 3, FG_FILENAME_LEN = 300

  type, bind(C) :: fg_params
     integer(c_int) :: method, continue_run
     real(c_double) :: GPa(3), kelvin
     real(c_double) :: mass_dipo(FG_RELAXOR_MAX), mass_acou(FG_RELAXOR_MAX), Q_Nose
     integer(c_int) :: bulk_or_film, Lx, Ly, Lz, gap_id, padding_y
     real(c_double) :: gap_dipole_u(3), a0, epi_strain, dt
     integer(c_int) :: n_thermalize, n_average, n_E_wave_period
     integer(c_int) :: n_coord_freq, n_hl_freq, n_hysteresis_loop_continue
     real(c_double) :: external_E_field(3)
     integer(c_int) :: E_wave_type
     real(c_double) :: P_kappa2(FG_RELAXOR_MAX), P_alpha(FG_RELAXOR_MAX), P_gamma(FG_RELAXOR_MAX)
     real(c_double) :: P_k1(FG_RELAXOR_MAX), P_k2(FG_RELAXOR_MAX), P_k3(FG_RELAXOR_MAX), P_k4(FG_RELAXOR_MAX)
     real(c_double) :: j(7)
     real(c_double) :: B11, B12, B44, B1xx, B1yy, B4yz, modulation_constant
     integer(c_int) :: seed(2)
     real(c_double) :: init_dipo_avg(3), init_dipo_dev(3), k_stripe(3)
     real(c_double) :: Z_star(FG_RELAXOR_MAX), epsilon_inf, kappa
     integer(c_int) :: plot_dispersion, output_polarization
     real(c_double) :: delta_e, delta_e_acou
     integer(c_int) :: verbose
     character(kind=c_char) :: coord_directory(FG_FILENAME_LEN)
     character(kind=c_char) :: slice_directory(FG_FILENAME_LEN)
     character(kind=c_char) :: distribution_directory(FG_FILENAME_LEN)
     character(kind=c_char) :: filename(FG_FILENAME_LEN)
     integer(c_int) :: N
     real(c_double) :: Ninv, dt_2
     integer(c_int) :: n_freedom
     real(c_double) :: unit_cell_volume, pNa03(3), temperature_eV, target_kinetic_energy
     integer(c_int) :: E_field_always_zero
  end type fg_params

  type, bind(C) :: fg_energy
     real(c_double) :: acou_kinetic, dipo_kinetic, short_range, long_range, dipole_E_field, &
          &            unharmonic, homo_strain, homo_coupling, inho_strain, inho_coupling, &
          &            inho_modulation, total, H_Nose_Poincare
  end type fg_energy

  interface
     integer(c_int) function fg_create(p, precision, ctx) bind(C, name='fg_create')
       import :: c_int, c_ptr, fg_params
       type(fg_params), intent(in) :: p
       integer(c_int), value :: precision
       type(c_ptr), intent(out) :: ctx
     end function fg_create
     subroutine fg_destroy(ctx) bind(C, name='fg_destroy')
       import :: c_ptr
       type(c_ptr), value :: ctx
     end subroutine fg_destroy
     integer(c_int) function fg_upload_tables(ctx, short_range, long_range) bind(C, name='fg_upload_tables')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, short_range, long_range
     end function fg_upload_tables
     integer(c_int) function fg_build_tables(ctx) bind(C, name='fg_build_tables')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function fg_build_tables
     integer(c_int) function fg_upload_modulation(ctx, ck) bind(C, name='fg_upload_modulation')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx, ck
     end function fg_upload_modulation
     integer(c_int) function fg_set_state(ctx, dipoR, dipoP, s, pi, H0) bind(C, name='fg_set_state')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx, dipoR, dipoP
       real(c_double), value :: s, pi, H0
     end function fg_set_state
     integer(c_int) function fg_get_state(ctx, dipoR, dipoP, dVddi, strain, s, pi, H0) bind(C, name='fg_get_state')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx, dipoR, dipoP, dVddi
       real(c_double), intent(out) :: strain(6), s, pi, H0
     end function fg_get_state
     integer(c_int) function fg_set_thermostat(ctx, s, pi, H0) bind(C, name='fg_set_thermostat')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), value :: s, pi, H0
     end function fg_set_thermostat
     integer(c_int) function fg_set_uniform_E(ctx, E) bind(C, name='fg_set_uniform_E')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: E(3)
     end function fg_set_uniform_E
     integer(c_int) function fg_mirror_force_mirror(ctx, e) bind(C, name='fg_mirror_force_mirror')
       import :: c_int, c_ptr, fg_energy
       type(c_ptr), value :: ctx
       type(fg_energy), intent(inout) :: e
     end function fg_mirror_force_mirror
     integer(c_int) function fg_nose_poincare(ctx, e) bind(C, name='fg_nose_poincare')
       import :: c_int, c_ptr, fg_energy
       type(c_ptr), value :: ctx
       type(fg_energy), intent(inout) :: e
     end function fg_nose_poincare
     integer(c_int) function fg_leapfrog(ctx, e, i_step) bind(C, name='fg_leapfrog')
       import :: c_int, c_ptr, fg_energy
       type(c_ptr), value :: ctx
       type(fg_energy), intent(inout) :: e
       integer(c_int), value :: i_step
     end function fg_leapfrog
     integer(c_int) function fg_kinetic_energy_dipo(ctx, ke) bind(C, name='fg_kinetic_energy_dipo')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: ke
     end function fg_kinetic_energy_dipo
     type(c_ptr) function fg_last_error(ctx) bind(C, name='fg_last_error')
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function fg_last_error
     ! next sweep point from the device state (replaces the .restart chaining
     ! of the sweep scripts, e.g. cooling.sh:64-69)
     integer(c_int) function fg_chain_point(ctx, kelvin, E, e) bind(C, name='fg_chain_point')
       import :: c_int, c_ptr, c_double, fg_energy
       type(c_ptr), value :: ctx
       real(c_double), value :: kelvin
       real(c_double), intent(in) :: E(3)
       type(fg_energy), intent(out) :: e
     end function fg_chain_point
     ! write_system's .coord (coord_module.F:434-486); full_precision /= 0
     ! writes 17 significant digits per value
     integer(c_int) function fg_write_coord(ctx, path, full_precision) bind(C, name='fg_write_coord')
       import :: c_int, c_ptr, c_char
       type(c_ptr), value :: ctx
       character(kind=c_char), intent(in) :: path(*)
       integer(c_int), value :: full_precision
     end function fg_write_coord
     ! the per-step field of molecular-dynamics.F:66-76 evaluated on the device
     integer(c_int) function fg_set_wave(ctx, on, i_step) bind(C, name='fg_set_wave')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int), value :: on, i_step
     end function fg_set_wave
     ! a sweep point (cooling.sh:64-69: n_thermalize + n_average steps from
     ! the previous point's state) with a device sample row every `every`
     ! averaging steps; rows of FG_SAMPLE_COLS = 16 doubles
     integer(c_int) function fg_run_point(ctx, kelvin, E, n_therm, n_avg, every, e) &
          & bind(C, name='fg_run_point')
       import :: c_int, c_ptr, c_double, fg_energy
       type(c_ptr), value :: ctx
       real(c_double), value :: kelvin
       real(c_double), intent(in) :: E(3)
       integer(c_int), value :: n_therm, n_avg, every
       type(fg_energy), intent(out) :: e
     end function fg_run_point
     integer(c_int) function fg_sample(ctx) bind(C, name='fg_sample')
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function fg_sample
     integer(c_int) function fg_samples_read(ctx, rows, max_rows, n_rows) bind(C, name='fg_samples_read')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       real(c_double), intent(out) :: rows(16, *)
       integer(c_int), value :: max_rows
       integer(c_int), intent(out) :: n_rows
     end function fg_samples_read
     ! launch plans: the autotuner (FFTW_MEASURE's role, coord_module.F:155-377)
     ! and its wisdom as text (feram_common.F:56-69, feram_fftw_wisdom.F)
     integer(c_int) function fg_tune(ctx, steps, zcw, waves, ms) bind(C, name='fg_tune')
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: ctx
       integer(c_int), value :: steps
       integer(c_int), intent(out) :: zcw, waves
       real(c_double), intent(out) :: ms
     end function fg_tune
     integer(c_int) function fg_wisdom_import(text, n_plans) bind(C, name='fg_wisdom_import')
       import :: c_int, c_char
       character(kind=c_char), intent(in) :: text(*)
       integer(c_int), intent(out) :: n_plans
     end function fg_wisdom_import
     integer(c_int) function fg_wisdom_export(buf, len, needed) bind(C, name='fg_wisdom_export')
       import :: c_int, c_char
       character(kind=c_char), intent(out) :: buf(*)
       integer(c_int), value :: len
       integer(c_int), intent(out) :: needed
     end function fg_wisdom_export
  end interface
end module feram_gpu_c

module feram_gpu_dropin
  use, intrinsic :: iso_c_binding
  use feram_gpu_c
  use Param_module
  use Coord_module
  use Energy_module
  implicit none
  type(c_ptr), save :: gctx = c_null_ptr
  logical, save :: device_owns_state = .false.
  private :: to_c_params, to_c_energy, from_c_energy, check
contains
  subroutine check(rc, where)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: where
    if (rc /= FG_OK) then
       write(0,'(a,a,i0)') where, ': feram_gpu error ', rc
       stop 1
    end if
  end subroutine check

  subroutine to_c_params(p, q)
    type(Param_type), intent(in) :: p
    type(fg_params), intent(out) :: q
    q%method = 0
    if (p%method == 'vs') q%method = 1
    if (p%method == 'lf') q%method = 2
    if (p%method == 'hl') q%method = 3
    q%continue_run = merge(1, 0, p%continue)
    q%GPa = p%GPa; q%kelvin = p%kelvin
    q%mass_dipo = p%mass_dipo; q%mass_acou = p%mass_acou; q%Q_Nose = p%Q_Nose
    q%bulk_or_film = 0
    if (p%bulk_or_film == 'film') q%bulk_or_film = 1
    if (p%bulk_or_film == 'epit') q%bulk_or_film = 2
    if (p%bulk_or_film == 'e110') q%bulk_or_film = 3
    q%Lx = p%Lx; q%Ly = p%Ly; q%Lz = p%Lz; q%gap_id = p%gap_id; q%padding_y = p%padding_y
    q%gap_dipole_u = p%gap_dipole_u; q%a0 = p%a0; q%epi_strain = p%epi_strain; q%dt = p%dt
    q%n_thermalize = p%n_thermalize; q%n_average = p%n_average; q%n_E_wave_period = p%n_E_wave_period
    q%n_coord_freq = p%n_coord_freq; q%n_hl_freq = p%n_hl_freq
    q%n_hysteresis_loop_continue = p%n_hysteresis_loop_continue
    q%external_E_field = p%external_E_field
    q%E_wave_type = 0
    if (p%E_wave_type == 'triangular_cos') q%E_wave_type = 1
    if (p%E_wave_type == 'triangular_sin') q%E_wave_type = 2
    if (p%E_wave_type == 'ramping_on')     q%E_wave_type = 3
    if (p%E_wave_type == 'ramping_off')    q%E_wave_type = 4
    q%P_kappa2 = p%P_kappa2; q%P_alpha = p%P_alpha; q%P_gamma = p%P_gamma
    q%P_k1 = p%P_k1; q%P_k2 = p%P_k2; q%P_k3 = p%P_k3; q%P_k4 = p%P_k4
    q%j = p%j
    q%B11 = p%B11; q%B12 = p%B12; q%B44 = p%B44
    q%B1xx = p%B1xx; q%B1yy = p%B1yy; q%B4yz = p%B4yz; q%modulation_constant = p%modulation_constant
    q%seed = p%seed; q%init_dipo_avg = p%init_dipo_avg; q%init_dipo_dev = p%init_dipo_dev
    q%k_stripe = p%k_stripe; q%Z_star = p%Z_star; q%epsilon_inf = p%epsilon_inf; q%kappa = p%kappa
    q%plot_dispersion = 0; q%output_polarization = 0
    q%delta_e = p%delta_e; q%delta_e_acou = p%delta_e_acou; q%verbose = p%verbose
    q%coord_directory = c_null_char; q%slice_directory = c_null_char
    q%distribution_directory = c_null_char; q%filename = c_null_char
    q%N = p%N; q%Ninv = p%Ninv; q%dt_2 = p%dt_2; q%n_freedom = p%n_freedom
    q%unit_cell_volume = p%unit_cell_volume; q%pNa03 = p%pNa03
    q%temperature_eV = p%temperature_eV; q%target_kinetic_energy = p%target_kinetic_energy
    q%E_field_always_zero = merge(1, 0, p%E_field_always_zero)
  end subroutine to_c_params

  subroutine to_c_energy(e, q)
    type(Energy_type), intent(in) :: e
    type(fg_energy), intent(out) :: q
    q%acou_kinetic = e%acou_kinetic; q%dipo_kinetic = e%dipo_kinetic
    q%short_range = e%short_range; q%long_range = e%long_range; q%dipole_E_field = e%dipole_E_field
    q%unharmonic = e%unharmonic; q%homo_strain = e%homo_strain; q%homo_coupling = e%homo_coupling
    q%inho_strain = e%inho_strain; q%inho_coupling = e%inho_coupling; q%inho_modulation = e%inho_modulation
    q%total = e%total; q%H_Nose_Poincare = e%H_Nose_Poincare
  end subroutine to_c_energy

  subroutine from_c_energy(q, e)
    type(fg_energy), intent(in) :: q
    type(Energy_type), intent(inout) :: e
    e%acou_kinetic = q%acou_kinetic; e%dipo_kinetic = q%dipo_kinetic
    e%short_range = q%short_range; e%long_range = q%long_range; e%dipole_E_field = q%dipole_E_field
    e%unharmonic = q%unharmonic; e%homo_strain = q%homo_strain; e%homo_coupling = q%homo_coupling
    e%inho_strain = q%inho_strain; e%inho_coupling = q%inho_coupling; e%inho_modulation = q%inho_modulation
    e%total = q%total; e%H_Nose_Poincare = q%H_Nose_Poincare
  end subroutine from_c_energy

  ! Call once after dipole_dipole(p,c) and elastic(p,c) (feram_common.F:82-83).
  subroutine gpu_attach(p, c, precision)
    type(Param_type), intent(in) :: p
    type(Coord_type), intent(inout), target :: c
    integer(c_int), intent(in) :: precision
    type(fg_params) :: q
    call to_c_params(p, q)
    if (c_associated(gctx)) call fg_destroy(gctx)
    call check(fg_create(q, precision, gctx), 'fg_create')
    call check(fg_upload_tables(gctx, c_loc(c%short_range), c_loc(c%long_range)), 'fg_upload_tables')
    if (p%modulation_constant /= 0.0d0) &
         & call check(fg_upload_modulation(gctx, c_loc(c%c_k_modulation_k)), 'fg_upload_modulation')
    device_owns_state = .false.
  end subroutine gpu_attach

  subroutine push_state(c)
    type(Coord_type), intent(inout), target :: c
    call check(fg_set_state(gctx, c_loc(c%dipoR), c_loc(c%dipoP), c%s_Nose, c%pi_Nose, c%H0), 'fg_set_state')
    device_owns_state = .true.
  end subroutine push_state

  ! Refresh c%dipoR, c%dipoP, c%dVddi, c%strain, s, pi, H0 from the device
  ! (before write_system, add_to_Average on the host, .hl output ...).
  subroutine gpu_pull_state(c)
    type(Coord_type), intent(inout), target :: c
    call check(fg_get_state(gctx, c_loc(c%dipoR), c_loc(c%dipoP), c_loc(c%dVddi), c%strain, &
         &                  c%s_Nose, c%pi_Nose, c%H0), 'fg_get_state')
  end subroutine gpu_pull_state

  ! mirror_force_mirror(p,c,e) of mirror_force_mirror.F:6-89
  subroutine mirror_force_mirror_gpu(p, c, e)
    type(Param_type), intent(inout) :: p
    type(Coord_type), intent(inout), target :: c
    type(Energy_type), intent(inout) :: e
    type(fg_energy) :: q
    if (.not. device_owns_state) call push_state(c)
    call to_c_energy(e, q)
    call check(fg_mirror_force_mirror(gctx, q), 'fg_mirror_force_mirror')
    call from_c_energy(q, e)
  end subroutine mirror_force_mirror_gpu

  ! nose_poincare(p,c,e) of nose-poincare.F:10-78
  subroutine nose_poincare_gpu(p, c, e)
    type(Param_type), intent(inout) :: p
    type(Coord_type), intent(inout), target :: c
    type(Energy_type), intent(inout) :: e
    type(fg_energy) :: q
    if (.not. device_owns_state) call push_state(c)
    call to_c_energy(e, q)
    call check(fg_nose_poincare(gctx, q), 'fg_nose_poincare')
    call from_c_energy(q, e)
  end subroutine nose_poincare_gpu

  ! leapfrog(p,c,e,i_step) of leapfrog.F:9-157
  subroutine leapfrog_gpu(p, c, e, i_step)
    type(Param_type), intent(inout) :: p
    type(Coord_type), intent(inout), target :: c
    type(Energy_type), intent(inout) :: e
    integer, intent(in) :: i_step
    type(fg_energy) :: q
    if (.not. device_owns_state) call push_state(c)
    call to_c_energy(e, q)
    call check(fg_leapfrog(gctx, q, int(i_step, c_int)), 'fg_leapfrog')
    call from_c_energy(q, e)
  end subroutine leapfrog_gpu

  ! The per-step E-field update of molecular-dynamics.F:66-76 (uniform field)
  subroutine gpu_set_field(E_field_add)
    real(c_double), intent(in) :: E_field_add(3)
    call check(fg_set_uniform_E(gctx, E_field_add), 'fg_set_uniform_E')
  end subroutine gpu_set_field

  ! The next point of a temperature sweep started from the device state, in
  ! place of reading the previous point's .coord as .restart
  ! (initialize-dipoR.F:22-38): p / s, the new kelvin and field, the force,
  ! s = 1, pi = 0 and H0 (molecular-dynamics.F:52-55)
  subroutine gpu_chain_point(p, e)
    type(Param_type), intent(in) :: p
    type(Energy_type), intent(inout) :: e
    type(fg_energy) :: q
    call check(fg_chain_point(gctx, real(p%kelvin, c_double), real(p%external_E_field, c_double), q), &
         & 'fg_chain_point')
    call from_c_energy(q, e)
  end subroutine gpu_chain_point
end module feram_gpu_dropin
