! msg123_gpu.f90 -- ISO_C_BINDING interface module over msg123_gpu.h, for a Msg123
! build that calls libmsg123gpu.so (add as src/Msg_gpu.f90, compile with -DMSG_GPU and
! link -lmsg123gpu -lcudart).
!
! Every derived type is bind(C) and lists the C struct's fields in the same order, so
! the companion C compiler's layout applies to both.  Every procedure binds the entry
! point of the same name in msg123_gpu.h with the same arguments.  Host arrays are
! passed as assumed-size arrays (the library copies them; it keeps no Fortran pointer
! after a call returns, except for msg_grid_t, whose arrays are read only inside
! msg_gpu_create).
module msg_gpu
  use, intrinsic :: iso_c_binding
  implicit none

  ! Problem description read by msg_gpu_create (set_cell_info / make_cell / set_connect).
  type, bind(C) :: msg_grid_t
    integer(c_int32_t) :: nx, ny, nz, sea_top, free_drainage, pad0
    type(c_ptr) :: reta, retn, resi, poro, ss, ksx, ksy, ksz
    type(c_ptr) :: cell_top, cell_vol, dis2face, face_area, area_r
    type(c_ptr) :: surf_top, surf_bott, surf_reli, surf_parm, sea_head
  end type

  ! Solver knobs (set_solution / set_amg namelists plus the library's extensions).
  type, bind(C) :: msg_params_t
    real(c_double) :: len_scal, criteria, lin_tol
    integer(c_int32_t) :: criteria_rel, maxout_iter, maxinn_iter, precon_type, ref_quirks
    integer(c_int32_t) :: precision, amg_nlevel, amg_coarse_max, amg_sweeps
    real(c_float) :: jac_omega, amg_theta, smooth_omega
    integer(c_int32_t) :: sim_type, amg_lag
    real(c_double) :: ini_step, inc_fact, max_step, end_time
    integer(c_int32_t) :: guess_mode, guess_select, vg_form, jv_mode
  end type

  ! One Newton solve (the columns of the reference's convergence log).
  type, bind(C) :: msg_stats_t
    integer(c_int32_t) :: status, out_iter, inner_total, back_total
    integer(c_int32_t) :: in_iter_last, back_iter_last, maxnun, pad
    real(c_double) :: maxvar, l2_new
  end type

  ! One time loop call (msg_gpu_advance).
  type, bind(C) :: msg_run_stats_t
    integer(c_int32_t) :: status, accepted, rejected, newton_total, krylov_total, back_total
    real(c_double) :: current_t, delt
  end type

  ! One Newton iteration of the convergence log (format 11 of calc_numsol).
  type, bind(C) :: msg_convrec_t
    real(c_double) :: time, delt
    integer(c_int32_t) :: out_iter, in_iter, back_iter, cell
    real(c_double) :: maxvar, dmat, rhs, head
    integer(c_int32_t) :: status, pad
  end type

  ! The context, kept here between set_connect (where it is created) and the time loop.
  type(c_ptr), save :: msg_gpu_ctx = c_null_ptr

  interface
    integer(c_int) function msg_gpu_create(g, p, ctx) bind(C)
      import; type(msg_grid_t), intent(in) :: g; type(msg_params_t), intent(in) :: p
      type(c_ptr), intent(out) :: ctx
    end function
    subroutine msg_gpu_destroy(ctx) bind(C)
      import; type(c_ptr), value :: ctx
    end subroutine
    type(c_ptr) function msg_gpu_last_error() bind(C)
      import
    end function
    integer(c_int) function msg_gpu_get_connect(ctx, offind, offrow, conn_dir, left_off, right_off, hydf, abyd, nnz) &
        bind(C)
      import; type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: offind(*), offrow(*), conn_dir(*), left_off(*), right_off(*), nnz
      real(c_double), intent(out) :: hydf(*), abyd(*)
    end function
    integer(c_int) function msg_gpu_init_state(ctx, head, delt) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: head(*)
      real(c_double), value :: delt
    end function
    integer(c_int) function msg_gpu_set_state(ctx, hn, ho, so, sh, delt) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: hn(*), ho(*), so(*), sh(*)
      real(c_double), value :: delt
    end function
    integer(c_int) function msg_gpu_get_state(ctx, hn, ho, sn, so, sh) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: hn(*), ho(*), sn(*), so(*), sh(*)
    end function
    integer(c_int) function msg_gpu_copy_state(dst, src) bind(C)
      import; type(c_ptr), value :: dst, src
    end function
    integer(c_int) function msg_gpu_set_recharge(ctx, rech) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: rech(*)
    end function
    integer(c_int) function msg_gpu_srat_rperm(ctx, pres, pertur, srat, rperm, sstor) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: pres(*)
      real(c_double), value :: pertur; real(c_double), intent(out) :: srat(*), rperm(*), sstor(*)
    end function
    integer(c_int) function msg_gpu_calc_func(ctx, x, f) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: x(*); real(c_double), intent(out) :: f(*)
    end function
    integer(c_int) function msg_gpu_make_matvec(ctx, dmat, lumat, rhs) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: dmat(*), lumat(*), rhs(*)
    end function
    integer(c_int) function msg_gpu_solve_linalg(ctx, init_norm, errtol, inx, last_norm, in_iter, conv) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), value :: init_norm, errtol
      real(c_double), intent(inout) :: inx(*); real(c_double), intent(out) :: last_norm
      integer(c_int32_t), intent(out) :: in_iter, conv
    end function
    integer(c_int) function msg_gpu_vecjacf(ctx, x, v, out) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(in) :: x(*), v(*)
      real(c_double), intent(out) :: out(*)
    end function
    integer(c_int) function msg_gpu_set_wells(ctx, nwell, well_index, well_conn, abyd_well, well_bott, read_well) &
        bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: nwell
      integer(c_int32_t), intent(in) :: well_index(*), well_conn(*)
      real(c_double), intent(in) :: abyd_well(*), well_bott(*), read_well(*)
    end function
    integer(c_int) function msg_gpu_set_rivers(ctx, n, rive2cals, rive_head, rive_bott, abyd_rive) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: n; integer(c_int32_t), intent(in) :: rive2cals(*)
      real(c_double), intent(in) :: rive_head(*), rive_bott(*), abyd_rive(*)
    end function
    integer(c_int) function msg_gpu_set_lakes(ctx, n, lake2cals, lake_head, lake_bott, abyd_lake) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: n; integer(c_int32_t), intent(in) :: lake2cals(*)
      real(c_double), intent(in) :: lake_head(*), lake_bott(*), abyd_lake(*)
    end function
    integer(c_int) function msg_gpu_calc_numsol(ctx, st) bind(C)
      import; type(c_ptr), value :: ctx; type(msg_stats_t), intent(out) :: st
    end function
    integer(c_int) function msg_gpu_advance(ctx, nsteps, rech_until, rech_after, st) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: nsteps
      real(c_double), value :: rech_until, rech_after; type(msg_run_stats_t), intent(out) :: st
    end function
    integer(c_int) function msg_gpu_calc_mass(ctx, out9) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: out9(9)
    end function
    ! per-cell volumes of the step, as calc_cell_mas adds them into st_msloc
    integer(c_int) function msg_gpu_cell_mass(ctx, sto, con, sea, wel, rec, sur, riv, lak, drn) bind(C)
      import; type(c_ptr), value :: ctx
      real(c_double), intent(out) :: sto(*), con(*), sea(*), wel(*), rec(*), sur(*), riv(*), lak(*), drn(*)
    end function
    ! calc_outvelc: facev(ncalc, 6) and pointv(ncalc, 3) in the layout of facev / pointv
    integer(c_int) function msg_gpu_velocity(ctx, facev, pointv) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: facev(*), pointv(*)
    end function
    integer(c_int) function msg_gpu_water_table(ctx, wtable) bind(C)
      import; type(c_ptr), value :: ctx; real(c_double), intent(out) :: wtable(*)
    end function
    integer(c_int) function msg_gpu_write_restart(ctx, path) bind(C)
      import; type(c_ptr), value :: ctx; character(kind=c_char), intent(in) :: path(*)
    end function
    integer(c_int) function msg_gpu_read_restart(path, ncalc, len_scal, head, time) bind(C)
      import; character(kind=c_char), intent(in) :: path(*); integer(c_int32_t), value :: ncalc
      real(c_double), value :: len_scal; real(c_double), intent(out) :: head(*), time
    end function
    integer(c_int) function msg_gpu_set_convlog(ctx, on) bind(C)
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: on
    end function
    integer(c_int) function msg_gpu_convlog(ctx, out, cap) bind(C)
      import; type(c_ptr), value :: ctx; type(msg_convrec_t), intent(out) :: out(*)
      integer(c_int32_t), value :: cap
    end function
    ! a_dev, inv_dev: device arrays the caller owns (c_devloc of CUDA Fortran / OpenACC data)
    integer(c_int) function msg_gpu_dense_inverse_noalloc(n, a_dev, inv_dev, stream) bind(C)
      import; integer(c_int32_t), value :: n; type(c_ptr), value :: a_dev, inv_dev, stream
    end function
  end interface
end module msg_gpu
