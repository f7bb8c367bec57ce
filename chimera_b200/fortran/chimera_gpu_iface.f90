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
    public :: chimera_set_time, chimera_step, chimera_advance, chimera_diag
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
    end interface
end module chimera_gpu_iface
