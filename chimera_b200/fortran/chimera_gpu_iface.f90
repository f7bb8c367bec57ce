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
    public :: chimera_set_time, chimera_step, chimera_advance, chimera_diag, chimera_step_host
    public :: chimera_batch_create, chimera_batch_set_state, chimera_batch_get_state
    public :: chimera_batch_set_time, chimera_batch_diag, chimera_set_graph_steps
    public :: chimera_autotune, chimera_set_variant
    public :: chimera_op_average_face_to_cell_B, chimera_op_get_primitive, chimera_op_get_conserved
    public :: chimera_op_apply_conserved_floors, chimera_op_fill_ghost_cells
    public :: chimera_op_compute_gradients, chimera_op_apply_slope_limiter, chimera_op_reconstruction
    public :: chimera_op_thermal_pressure_check, chimera_op_compute_fluxes
    public :: chimera_op_update_conserved, chimera_op_constrained_transport
    public :: chimera_op_compute_curl_2d, chimera_op_compute_divB
    public :: CHIMERA_HOST, CHIMERA_DEVICE, CHIMERA_FP64, CHIMERA_FP32_BULK

    integer(c_int), parameter :: CHIMERA_HOST = 0, CHIMERA_DEVICE = 1
    integer(c_int), parameter :: CHIMERA_FP64 = 0, CHIMERA_FP32_BULK = 1

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
