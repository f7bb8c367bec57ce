! chimera_gpu_iface.f90 -- iso_c_binding interface to libchimera_gpu.so
! (include/chimera_gpu.h) for the CHIMERA Fortran time loop.
!
! The derived types mirror the C structs field for field (bind(C)); every
! routine returns an integer status (0 = ok, negative = CHIMERA_ERR_*).
! Arrays are passed by address: real(c_double) (ld, ny), the layout of the
! reference's module arrays Mass, Momx, Momy, Energy, b_x, b_y.
module chimera_gpu_iface
    use, intrinsic :: iso_c_binding
    implicit none
    private
    public :: chimera_cfg, chimera_diag_out
    public :: chimera_create, chimera_destroy, chimera_set_state, chimera_get_state
    public :: chimera_set_time, chimera_step, chimera_advance, chimera_advance_output, chimera_diag
    public :: chimera_step_host
    public :: chimera_batch_create, chimera_batch_set_state, chimera_batch_get_state
    public :: chimera_batch_set_time, chimera_batch_diag, chimera_set_graph_steps
    public :: chimera_autotune, chimera_set_variant
    public :: chimera_halo_pack, chimera_halo_unpack, chimera_slab_ghost_rows
    public :: chimera_refresh_dt, chimera_get_dt_device, chimera_set_dt_device
    public :: chimera_stage, chimera_get_stage_buffer, chimera_set_counters, chimera_set_profiling
    public :: chimera_get_profile, chimera_stream, chimera_batch_size, chimera_variant_count
    public :: chimera_get_variant, chimera_rk3_step_noalloc, chimera_strerror, chimera_version
    public :: chimera_adjoint_create, chimera_adjoint_step, chimera_adjoint_forward_step
    public :: chimera_adjoint_destroy
    public :: chimera_op_average_face_to_cell_B, chimera_op_get_primitive, chimera_op_get_conserved
    public :: chimera_op_apply_conserved_floors, chimera_op_fill_ghost_cells
    public :: chimera_op_compute_gradients, chimera_op_apply_slope_limiter, chimera_op_reconstruction
    public :: chimera_op_thermal_pressure_check, chimera_op_compute_fluxes
    public :: chimera_op_update_conserved, chimera_op_constrained_transport
    public :: chimera_op_compute_curl_2d, chimera_op_compute_divB
    public :: CHIMERA_HOST, CHIMERA_DEVICE, CHIMERA_FP64, CHIMERA_FP32_BULK, CHIMERA_FP32_MIXED

    integer(c_int), parameter :: CHIMERA_HOST = 0, CHIMERA_DEVICE = 1
    integer(c_int), parameter :: CHIMERA_FP64 = 0, CHIMERA_FP32_BULK = 1, CHIMERA_FP32_MIXED = 2

    type, bind(C) :: chimera_cfg
        integer(c_int)  :: nx, ny
        real(c_double)  :: dx, dy, gamma, courant, t_out, t_end
        integer(c_int)  :: bc_xlo, bc_xhi, bc_ylo, bc_yhi
        integer(c_int)  :: riemann, limiter, use_slope_limiting, mood, precision
    end type chimera_cfg

    type, bind(C) :: chimera_diag_out
        real(c_double)     :: t, dt
        integer(c_int)     :: output_count, active
        integer(c_long_long) :: steps
        real(c_double)     :: divb_max, divb_mean, bmax, divb_rel, mass, energy, cfl_speed
        integer(c_long_long) :: mood_resets, floor_hits
        integer(c_int)     :: status
    end type chimera_diag_out

    interface
        integer(c_int) function chimera_create(cfg, stream, h) bind(C, name="chimera_create")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: stream
            type(c_ptr), intent(out) :: h
        end function

        subroutine chimera_destroy(h) bind(C, name="chimera_destroy")
            import :: c_ptr
            type(c_ptr), value :: h
        end subroutine

        integer(c_int) function chimera_set_state(h, Mass, Momx, Momy, Energy, b_x, b_y, ld, where) &
                bind(C, name="chimera_set_state")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: Mass(*), Momx(*), Momy(*), Energy(*), b_x(*), b_y(*)
            integer(c_int), value :: ld, where
        end function

        integer(c_int) function chimera_get_state(h, Mass, Momx, Momy, Energy, b_x, b_y, ld, where) &
                bind(C, name="chimera_get_state")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: Mass(*), Momx(*), Momy(*), Energy(*), b_x(*), b_y(*)
            integer(c_int), value :: ld, where
        end function

        integer(c_int) function chimera_set_time(h, t, output_count) bind(C, name="chimera_set_time")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), value :: t
            integer(c_int), value :: output_count
        end function

        integer(c_int) function chimera_step(h, nsteps) bind(C, name="chimera_step")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: nsteps
        end function

        ! one step on host arrays: ptrs = [c_loc(Mass), c_loc(Momx), ..., c_loc(b_y)] of
        ! target arrays (ld, ny); out_ptrs may equal in_ptrs
        integer(c_int) function chimera_step_host(h, in_ptrs, out_ptrs, ld) bind(C, name="chimera_step_host")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            type(c_ptr), intent(in) :: in_ptrs(6), out_ptrs(6)
            integer(c_int), value :: ld
        end function

        integer(c_int) function chimera_advance(h, max_steps, steps_taken) bind(C, name="chimera_advance")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: max_steps
            integer(c_int), intent(out) :: steps_taken
        end function

        ! as chimera_advance, stopping after the step that reaches the next output time
        integer(c_int) function chimera_advance_output(h, max_steps, steps_taken) &
                bind(C, name="chimera_advance_output")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: max_steps
            integer(c_int), intent(out) :: steps_taken
        end function

        integer(c_int) function chimera_diag(h, out) bind(C, name="chimera_diag")
            import :: c_int, c_ptr, chimera_diag_out
            type(c_ptr), value :: h
            type(chimera_diag_out), intent(out) :: out
        end function
        ! ---- batched ensembles ----------------------------------------------------
        integer(c_int) function chimera_batch_create(n_members, cfgs, stream, h) &
                bind(C, name="chimera_batch_create")
            import :: c_int, c_ptr, chimera_cfg
            integer(c_int), value :: n_members
            type(chimera_cfg), intent(in) :: cfgs(*)
            type(c_ptr), value :: stream
            type(c_ptr), intent(out) :: h
        end function

        integer(c_int) function chimera_batch_set_state(h, member, Mass, Momx, Momy, Energy, b_x, b_y, &
                ld, where) bind(C, name="chimera_batch_set_state")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: member
            real(c_double), intent(in) :: Mass(*), Momx(*), Momy(*), Energy(*), b_x(*), b_y(*)
            integer(c_int), value :: ld, where
        end function

        integer(c_int) function chimera_batch_get_state(h, member, Mass, Momx, Momy, Energy, b_x, b_y, &
                ld, where) bind(C, name="chimera_batch_get_state")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: member
            real(c_double), intent(out) :: Mass(*), Momx(*), Momy(*), Energy(*), b_x(*), b_y(*)
            integer(c_int), value :: ld, where
        end function

        integer(c_int) function chimera_batch_set_time(h, member, t, output_count) &
                bind(C, name="chimera_batch_set_time")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: member
            real(c_double), value :: t
            integer(c_int), value :: output_count
        end function

        integer(c_int) function chimera_batch_diag(h, member, out) bind(C, name="chimera_batch_diag")
            import :: c_int, c_ptr, chimera_diag_out
            type(c_ptr), value :: h
            integer(c_int), value :: member
            type(chimera_diag_out), intent(out) :: out
        end function

        integer(c_int) function chimera_set_graph_steps(h, nsteps) bind(C, name="chimera_set_graph_steps")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: nsteps
        end function

        integer(c_int) function chimera_autotune(h, reps, chosen, best_ms_per_step) &
                bind(C, name="chimera_autotune")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: reps
            integer(c_int), intent(out) :: chosen
            real(c_double), intent(out) :: best_ms_per_step
        end function

        integer(c_int) function chimera_set_variant(h, variant) bind(C, name="chimera_set_variant")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: variant
        end function

        ! ---- one grid split into y-slabs across ranks (an MPI or NCCL caller moves
        !      the packed ghost rows and takes the minimum dt between the calls) --------
        integer(c_int) function chimera_halo_pack(h, rows, lo, hi) bind(C, name="chimera_halo_pack")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, lo, hi
            integer(c_int), value :: rows
        end function

        integer(c_int) function chimera_halo_unpack(h, rows, lo, hi) bind(C, name="chimera_halo_unpack")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, lo, hi
            integer(c_int), value :: rows
        end function

        integer(c_int) function chimera_slab_ghost_rows(h, ghost_lo, ghost_hi) &
                bind(C, name="chimera_slab_ghost_rows")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: ghost_lo, ghost_hi
        end function

        ! ---- stage-level access, counters, timing, tile variants ------------------------
        integer(c_int) function chimera_stage(h, k, dt) bind(C, name="chimera_stage")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: k
            real(c_double), value :: dt
        end function

        integer(c_int) function chimera_get_stage_buffer(h, b, Mass, Momx, Momy, Energy, b_x, b_y, ld, where) &
                bind(C, name="chimera_get_stage_buffer")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: b
            real(c_double), intent(out) :: Mass(*), Momx(*), Momy(*), Energy(*), b_x(*), b_y(*)
            integer(c_int), value :: ld, where
        end function

        integer(c_int) function chimera_set_counters(h, on) bind(C, name="chimera_set_counters")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: on
        end function

        integer(c_int) function chimera_set_profiling(h, on) bind(C, name="chimera_set_profiling")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: on
        end function

        integer(c_int) function chimera_get_profile(h, ms, launches, reset) bind(C, name="chimera_get_profile")
            import :: c_int, c_ptr, c_double, c_long_long
            type(c_ptr), value :: h
            real(c_double), intent(out) :: ms(4)
            integer(c_long_long), intent(out) :: launches(4)
            integer(c_int), value :: reset
        end function

        type(c_ptr) function chimera_stream(h) bind(C, name="chimera_stream")
            import :: c_ptr
            type(c_ptr), value :: h
        end function

        integer(c_int) function chimera_batch_size(h) bind(C, name="chimera_batch_size")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function

        integer(c_int) function chimera_variant_count(h) bind(C, name="chimera_variant_count")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function

        integer(c_int) function chimera_get_variant(h, variant, tile_x, tile_y, threads) &
                bind(C, name="chimera_get_variant")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), intent(out) :: variant, tile_x, tile_y, threads
        end function

        ! ---- one step without device allocation (device arrays updated in place) --------
        integer(c_int) function chimera_rk3_step_noalloc(cfg, Mass, Momx, Momy, Energy, b_x, b_y, t, &
                output_count, dt_next, stream) bind(C, name="chimera_rk3_step_noalloc")
            import :: c_int, c_ptr, c_double, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: Mass, Momx, Momy, Energy, b_x, b_y
            real(c_double), intent(inout) :: t
            integer(c_int), intent(inout) :: output_count
            real(c_double), intent(out) :: dt_next
            type(c_ptr), value :: stream
        end function

        ! ---- discrete adjoint of one RK3 step (arrays of six device pointers) ------------
        integer(c_int) function chimera_adjoint_create(cfg, stream, a) bind(C, name="chimera_adjoint_create")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: stream
            type(c_ptr), intent(out) :: a
        end function

        integer(c_int) function chimera_adjoint_step(a, U_n, dt, lambda_next, lambda_n) &
                bind(C, name="chimera_adjoint_step")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: a
            type(c_ptr), intent(in) :: U_n(6), lambda_next(6), lambda_n(6)
            real(c_double), value :: dt
        end function

        integer(c_int) function chimera_adjoint_forward_step(a, U_n, dt, U_next) &
                bind(C, name="chimera_adjoint_forward_step")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: a
            type(c_ptr), intent(in) :: U_n(6), U_next(6)
            real(c_double), value :: dt
        end function

        subroutine chimera_adjoint_destroy(a) bind(C, name="chimera_adjoint_destroy")
            import :: c_ptr
            type(c_ptr), value :: a
        end subroutine

        ! ---- error text (a C string: c_f_pointer it to a character array) and version ----
        type(c_ptr) function chimera_strerror(code) bind(C, name="chimera_strerror")
            import :: c_int, c_ptr
            integer(c_int), value :: code
        end function

        integer(c_int) function chimera_version() bind(C, name="chimera_version")
            import :: c_int
        end function

        integer(c_int) function chimera_refresh_dt(h, d_dt) bind(C, name="chimera_refresh_dt")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, d_dt
        end function

        integer(c_int) function chimera_get_dt_device(h, d_dt) bind(C, name="chimera_get_dt_device")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, d_dt
        end function

        integer(c_int) function chimera_set_dt_device(h, d_dt) bind(C, name="chimera_set_dt_device")
            import :: c_int, c_ptr
            type(c_ptr), value :: h, d_dt
        end function

        ! ---- per-routine entry points: device arrays (c_ptr from the caller's allocator),
        !      asynchronous on the given stream ---------------------------------------
        integer(c_int) function chimera_op_average_face_to_cell_B(cfg, b_x, b_y, Bx, By, stream) &
                bind(C, name="chimera_op_average_face_to_cell_B")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: b_x, b_y, Bx, By, stream
        end function

        integer(c_int) function chimera_op_get_primitive(cfg, Mass, Momx, Momy, Energy, Bx, By, &
                rho, vx, vy, P, stream) bind(C, name="chimera_op_get_primitive")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: Mass, Momx, Momy, Energy, Bx, By, rho, vx, vy, P, stream
        end function

        integer(c_int) function chimera_op_get_conserved(cfg, rho, vx, vy, P, Bx, By, &
                Mass, Momx, Momy, Energy, stream) bind(C, name="chimera_op_get_conserved")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: rho, vx, vy, P, Bx, By, Mass, Momx, Momy, Energy, stream
        end function

        integer(c_int) function chimera_op_apply_conserved_floors(cfg, Mass, Momx, Momy, Energy, Bx, By, &
                stream) bind(C, name="chimera_op_apply_conserved_floors")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: Mass, Momx, Momy, Energy, Bx, By, stream
        end function

        integer(c_int) function chimera_op_fill_ghost_cells(cfg, f, f_pad, stream) &
                bind(C, name="chimera_op_fill_ghost_cells")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: f, f_pad, stream
        end function

        integer(c_int) function chimera_op_compute_gradients(cfg, f_pad, f_dx, f_dy, stream) &
                bind(C, name="chimera_op_compute_gradients")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: f_pad, f_dx, f_dy, stream
        end function

        integer(c_int) function chimera_op_apply_slope_limiter(cfg, f_pad, f_dx, f_dy, stream) &
                bind(C, name="chimera_op_apply_slope_limiter")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: f_pad, f_dx, f_dy, stream
        end function

        integer(c_int) function chimera_op_reconstruction(cfg, f, f_dx, f_dy, f_XL, f_XR, f_YL, f_YR, &
                rho_or_p, stream) bind(C, name="chimera_op_reconstruction")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: f, f_dx, f_dy, f_XL, f_XR, f_YL, f_YR
            integer(c_int), value :: rho_or_p
            type(c_ptr), value :: stream
        end function

        ! faces24(s*6+q+1): slot s in (XL, XR, YL, YR), field q in (P, Bx, By, rho, vx, vy)
        integer(c_int) function chimera_op_thermal_pressure_check(cfg, faces24, cell6, stream) &
                bind(C, name="chimera_op_thermal_pressure_check")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), intent(in) :: faces24(24), cell6(6)
            type(c_ptr), value :: stream
        end function

        ! in12: rho_L, rho_R, vn_L, vn_R, vt_L, vt_R, P_L, P_R, Bn_L, Bn_R, Bt_L, Bt_R
        integer(c_int) function chimera_op_compute_fluxes(cfg, in12, out5, stream) &
                bind(C, name="chimera_op_compute_fluxes")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), intent(in) :: in12(12), out5(5)
            type(c_ptr), value :: stream
        end function

        integer(c_int) function chimera_op_update_conserved(cfg, F, flux_X, flux_Y, dt, stream) &
                bind(C, name="chimera_op_update_conserved")
            import :: c_int, c_ptr, c_double, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: F, flux_X, flux_Y
            real(c_double), value :: dt
            type(c_ptr), value :: stream
        end function

        integer(c_int) function chimera_op_constrained_transport(cfg, b_x, b_y, flux_By_X, flux_Bx_Y, dt, &
                scratch, stream) bind(C, name="chimera_op_constrained_transport")
            import :: c_int, c_ptr, c_double, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: b_x, b_y, flux_By_X, flux_Bx_Y
            real(c_double), value :: dt
            type(c_ptr), value :: scratch, stream
        end function

        integer(c_int) function chimera_op_compute_curl_2d(cfg, Az, b_x, b_y, stream) &
                bind(C, name="chimera_op_compute_curl_2d")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: Az, b_x, b_y, stream
        end function

        integer(c_int) function chimera_op_compute_divB(cfg, b_x, b_y, divB, stream) &
                bind(C, name="chimera_op_compute_divB")
            import :: c_int, c_ptr, chimera_cfg
            type(chimera_cfg), intent(in) :: cfg
            type(c_ptr), value :: b_x, b_y, divB, stream
        end function
    end interface
end module chimera_gpu_iface
