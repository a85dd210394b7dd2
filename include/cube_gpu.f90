! cube_gpu.f90 -- iso_c_binding interface to libcube_b200.so (include/cube_gpu.h)
! and the no-argument wrappers a CUBE host program calls in place of its own
! particle_mesh / update_x / ext_pp_force (main.f90:57-64).
!
! The wrappers read and write the host's module variables (variables.f90:28-81)
! exactly where the reference routines do: the scalar block is filled from the
! module scalars before each call and copied back after it; the particle and
! mesh arrays stay on the GPU between calls and come back only at checkpoints
! (cube_gpu_checkpoint_out), in the checkpoint layout of checkpoint.f90:24-75.
! Build: gfortran -c cube_gpu.f90 ; link with -L<pkg> -lcube_b200 -lcudart.
module cube_gpu
  use iso_c_binding
  implicit none

  type, bind(c) :: cube_params_t
    integer(c_int32_t) :: nc, nnt, ncell, ncb, np_nc, izipx, izipv, nf_cutoff, pp_range
    integer(c_int32_t) :: ext_pp_force, use_pid, neutrino
    real(c_float) :: rsoft, tile_buffer, image_buffer, vbuf
    real(c_double) :: vrel_boost
    real(c_float) :: box, h0, omega_m, omega_l, wde, ra_max, dt_max
    real(c_float) :: z_i_nu, f_neu, m_nu_ev, deg_nu
    integer(c_int32_t) :: nu_nc(3), stockham_only, poisson_fp64, reserved(6)
  end type

  type, bind(c) :: cube_scalars_t
    real(c_float) :: a, a_mid, da, dt, dt_old, dt_mid, t, tau
    real(c_float) :: sigma_vi, sigma_vi_new, mass_p_cdm, vz_max
    real(c_float) :: dt_fine, dt_coarse, dt_pp, dt_vmax, dt_vmax_nu, dt_e, dt_neu
    real(c_float) :: vmax(3), f2_max_fine, f2_max_coarse, f2_max_pp, vsim2phys
    integer(c_int32_t) :: nlayer, timestep
    real(c_double) :: std_vsim, std_vsim_c, std_vsim_res, testrhof, testrhoc
    integer(c_int64_t) :: nplocal, npglobal, npairs, itest1
    integer(c_int32_t) :: reserved(16)
  end type

  ! cube_make_ic arguments (in place of running ic.x and reading its files)
  type, bind(c) :: cube_ic_params_t
    integer(c_int64_t) :: seed
    integer(c_int32_t) :: np_nc, pad0
    real(c_double) :: a, norm_d2, n_s, h, eh_s, eh_alpha, eh_omh, eh_theta2, vf, amplitude, f_cdm
  end type

  ! cube_halofind: one record is type_halo_info (halofind.f90:10-15)
  type, bind(c) :: cube_halo_t
    real(c_float) :: hpos(3), mass_odc, radius_odc, v_disp
    real(c_float) :: x_mean(3), v_mean(3), ang_mom(3), var_x(3), inertia(3,3)
    real(c_float) :: q_mean(3), inertia_q(3,3), s_mean(3)
  end type

  type, bind(c) :: cube_halo_args_t
    real(c_float) :: den_odc
    integer(c_int32_t) :: capacity
    type(c_ptr) :: halos, member_pid
    integer(c_int64_t) :: member_capacity
    type(c_ptr) :: hid
    integer(c_int64_t) :: hid_len
  end type

  type, bind(c) :: cube_halo_result_t
    integer(c_int32_t) :: nhalo, npeak
    integer(c_int64_t) :: nmember
  end type

  interface
    integer(c_int32_t) function cube_create(p, cap, fk, ck, ctx) bind(c, name="cube_create")
      import :: c_int32_t, c_int64_t, c_float, c_ptr, cube_params_t
      type(cube_params_t), intent(in) :: p
      integer(c_int64_t), value :: cap
      real(c_float), intent(in) :: fk(*), ck(*)
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int32_t) function cube_load_state(ctx, np, xp, vp, pid, rhoc, vfield) bind(c, name="cube_load_state")
      import :: c_int32_t, c_int64_t, c_float, c_ptr
      type(c_ptr), value :: ctx, xp, vp
      integer(c_int64_t), value :: np
      integer(c_int32_t), intent(in) :: pid(*), rhoc(*)
      real(c_float), intent(in) :: vfield(*)
    end function
    integer(c_int32_t) function cube_store_state(ctx, np, xp, vp, pid, rhoc, vfield) bind(c, name="cube_store_state")
      import :: c_int32_t, c_int64_t, c_float, c_ptr
      type(c_ptr), value :: ctx, xp, vp
      integer(c_int64_t), intent(out) :: np
      integer(c_int32_t), intent(out) :: pid(*), rhoc(*)
      real(c_float), intent(out) :: vfield(*)
    end function
    integer(c_int32_t) function cube_update_x(ctx, s) bind(c, name="cube_update_x")
      import :: c_int32_t, c_ptr, cube_scalars_t
      type(c_ptr), value :: ctx
      type(cube_scalars_t), intent(inout) :: s
    end function
    integer(c_int32_t) function cube_ext_pp_force(ctx, s) bind(c, name="cube_ext_pp_force")
      import :: c_int32_t, c_ptr, cube_scalars_t
      type(c_ptr), value :: ctx
      type(cube_scalars_t), intent(inout) :: s
    end function
    integer(c_int32_t) function cube_particle_mesh(ctx, s) bind(c, name="cube_particle_mesh")
      import :: c_int32_t, c_ptr, cube_scalars_t
      type(c_ptr), value :: ctx
      type(cube_scalars_t), intent(inout) :: s
    end function
    function cube_last_error(ctx) bind(c, name="cube_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
      type(c_ptr) :: cube_last_error
    end function
    ! neu(nu)%evolve(dt,dtg,dir,a) (hydrodf.f90:86)
    integer(c_int32_t) function cube_nu_evolve(ctx, dt, dtg, dir, a) bind(c, name="cube_nu_evolve")
      import :: c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), value :: dt, a
      real(c_float), intent(inout) :: dtg
      integer(c_int32_t), value :: dir
    end function
    ! one fluid's physical cells fld(1:5,1:n,1:n,1:n)
    integer(c_int32_t) function cube_nu_load(ctx, fluid, fld) bind(c, name="cube_nu_load")
      import :: c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: fluid
      real(c_float), intent(in) :: fld(*)
    end function
    integer(c_int32_t) function cube_nu_store(ctx, fluid, fld) bind(c, name="cube_nu_store")
      import :: c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: fluid
      real(c_float), intent(out) :: fld(*)
    end function
    ! Zel'dovich state on the device in place of ic.x
    integer(c_int32_t) function cube_make_ic(ctx, ic, s) bind(c, name="cube_make_ic")
      import :: c_int32_t, c_ptr, cube_ic_params_t, cube_scalars_t
      type(c_ptr), value :: ctx
      type(cube_ic_params_t), intent(in) :: ic
      type(cube_scalars_t), intent(inout) :: s
    end function

    ! cicpower analysis into xip(10,nbin)
    integer(c_int32_t) function cube_power_spectrum(ctx, log_bins, xip, capacity, nbin) &
        bind(c, name="cube_power_spectrum")
      import :: c_int32_t, c_ptr, c_float
      type(c_ptr), value :: ctx
      integer(c_int32_t), value :: log_bins, capacity
      real(c_float), intent(out) :: xip(10, *)
      integer(c_int32_t), intent(out) :: nbin
    end function

    ! run-time halo finder (halofind.f90:18-598)
    integer(c_int32_t) function cube_halofind(ctx, s, args, res) bind(c, name="cube_halofind")
      import :: c_int32_t, c_ptr, cube_scalars_t, cube_halo_args_t, cube_halo_result_t
      type(c_ptr), value :: ctx
      type(cube_scalars_t), intent(in) :: s
      type(cube_halo_args_t), intent(in) :: args
      type(cube_halo_result_t), intent(out) :: res
    end function
  end interface

  type(c_ptr), save :: gpu_ctx = c_null_ptr
  type(cube_scalars_t), save :: gpu_s

contains

  subroutine gpu_check(rc, where)
    integer(c_int32_t), intent(in) :: rc
    character(*), intent(in) :: where
    if (rc /= 0) then
      print*, 'cube_gpu error in ', where, ' status', rc
      stop
    endif
  end subroutine

end module cube_gpu

! The host keeps its own subroutine names; replace the bodies of
! particle_mesh (pm.f90), update_x (update_particle.f90) and ext_pp_force
! (ext_pp_force.f90) with these (buffer_grid/buffer_x/buffer_v become empty).
!
!   subroutine update_x
!     use variables; use cube_gpu
!     gpu_s%dt = dt; gpu_s%dt_old = dt_old; gpu_s%sigma_vi = sigma_vi
!     gpu_s%vz_max = sim%vz_max; gpu_s%npglobal = sim%npglobal
!     call gpu_check(cube_update_x(gpu_ctx, gpu_s), 'update_x')
!     dt_mid = gpu_s%dt_mid; sigma_vi_new = gpu_s%sigma_vi_new; sim%nplocal = gpu_s%nplocal
!   end subroutine
!
!   subroutine particle_mesh
!     use variables; use cube_gpu
!     gpu_s%a = a; gpu_s%a_mid = a_mid; gpu_s%dt = dt; gpu_s%mass_p_cdm = sim%mass_p_cdm
!     gpu_s%sigma_vi = sigma_vi; gpu_s%sigma_vi_new = sigma_vi_new
!     call gpu_check(cube_particle_mesh(gpu_ctx, gpu_s), 'particle_mesh')
!     sigma_vi = gpu_s%sigma_vi; sim%dt_fine = gpu_s%dt_fine; sim%dt_coarse = gpu_s%dt_coarse
!     sim%dt_vmax = gpu_s%dt_vmax; sim%vz_max = gpu_s%vz_max; sim%vsim2phys = gpu_s%vsim2phys
!   end subroutine
!
! and the neutrino half steps of main.f90:51-54, 66-69:
!
!     call gpu_check(cube_nu_evolve(gpu_ctx, dt/2., dt_neu, 1, a_mid), 'nu evolve')
!
! and halofind (halofind.f90:18) as
!
!   subroutine halofind
!     use variables; use cube_gpu
!     type(cube_halo_t), allocatable, target :: h(:)
!     integer(c_int32_t), allocatable, target :: mem(:), hid4(:)
!     type(cube_halo_args_t) :: ha
!     type(cube_halo_result_t) :: hr
!     allocate(h(200000), mem(sim%nplocal), hid4(nf**3))
!     ha%den_odc = 200; ha%capacity = size(h); ha%halos = c_loc(h)
!     ha%member_pid = c_loc(mem); ha%member_capacity = size(mem, kind=c_int64_t)
!     ha%hid = c_loc(hid4); ha%hid_len = size(hid4, kind=c_int64_t)
!     gpu_s%a = a; gpu_s%sigma_vi = sigma_vi; gpu_s%mass_p_cdm = sim%mass_p_cdm
!     gpu_s%vsim2phys = sim%vsim2phys
!     call gpu_check(cube_halofind(gpu_ctx, gpu_s, ha, hr), 'halofind')
!     ! then write(11) hr%nhalo, hr%nhalo, 200., h(:hr%nhalo); the halo_pid records from
!     ! mem(1:hr%nmember) split by int(h%mass_odc); write(21) int(hid4, 2)
!   end subroutine
