! ============================================================================ !
!   lssph_cuda_mod -- iso_c_binding interface of the B200 LS-SPH engine
!   (include/lssph.h).  A Fortran host that keeps the LS-SPH-Benchmarks driver
!   (source/main.f90) replaces its time loop, main.f90:119-166, with calls to
!   lssph_step; see main_gpu.f90 beside this file.
!
!   Indices on the C side are 0-based; arrays are passed whole (1-based in
!   Fortran, same memory).  Every function returns 0 on success or a negative
!   LSSPH_E_* status; lssph_last_error_f returns the message.
! ============================================================================ !
module lssph_cuda_mod
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: LSSPH_OK = 0
    integer(c_int), parameter :: LSSPH_PRECISION_FP64 = 0, LSSPH_PRECISION_MIXED = 1
    integer(c_int), parameter :: LSSPH_PRECISION_MIXED_COMPENSATED = 2

    ! Mirror of lssph_params (same field order and padding as include/lssph.h)
    type, bind(c) :: lssph_params
        integer(c_int32_t) :: target_problem
        integer(c_int32_t) :: u_bc_top, u_bc_bottom, u_bc_left, u_bc_right
        integer(c_int32_t) :: tem_bc_top, tem_bc_bottom, tem_bc_left, tem_bc_right
        real(c_double)     :: u_top
        real(c_double)     :: tem_top, tem_bottom, tem_left, tem_right
        character(kind=c_char) :: save_name(256)
        character(kind=c_char) :: read_name(256)
        integer(c_int32_t) :: omp_threads
        integer(c_int32_t) :: rk
        real(c_double)     :: len_x, len_y
        integer(c_int32_t) :: num_x, num_y
        integer(c_int32_t) :: start_step, end_step, write_step
        integer(c_int32_t) :: pad0_
        real(c_double)     :: threshold, coe_CFL, coe_dif, zeta_RSST, xi_VIM
        real(c_double)     :: rho_ref, vis_ref, K_ref, k_th_ref, cp_ref, alpha_ref
        real(c_double)     :: gravity, pos_pert
        integer(c_int32_t) :: tg_a, tg_b
        real(c_double)     :: coe_h, PST_c, coe_delta_sph
        integer(c_int32_t) :: kernel_type, sph_model, wall_model
        integer(c_int32_t) :: total_step, num_WL
        integer(c_int32_t) :: pad1_
        real(c_double)     :: dx, SP_mass, h, h_eff, W_ave, WL_thick
        real(c_double)     :: delta_tem, tem_ave
        real(c_double)     :: sound_speed, kinematic_vis, thermal_dif
        real(c_double)     :: Re, Ra, Pr
        real(c_double)     :: dt, dt_CFL, dt_vis, dt_th, dt_CFL_relax, dt_vis_relax
        integer(c_int32_t) :: precision
        integer(c_int32_t) :: lanes
        integer(c_int64_t) :: seed
        integer(c_int32_t) :: periodic, pad2_
    end type lssph_params

    interface
        integer(c_int) function lssph_params_from_config(path, p) bind(c, name="lssph_params_from_config")
            import :: c_int, c_char, lssph_params
            character(kind=c_char), intent(in) :: path(*)
            type(lssph_params), intent(out) :: p
        end function

        integer(c_int) function lssph_setup_counts(p, num_total, num_int) bind(c, name="lssph_setup_counts")
            import :: c_int, c_int32_t, lssph_params
            type(lssph_params), intent(in) :: p
            integer(c_int32_t), intent(out) :: num_total, num_int
        end function

        integer(c_int) function lssph_setup_particles(p, num_total, ptype, x, y, u, v, rho, pre, tem) &
                bind(c, name="lssph_setup_particles")
            import :: c_int, c_int32_t, c_double, lssph_params
            type(lssph_params), intent(in) :: p
            integer(c_int32_t), value :: num_total
            integer(c_int32_t), intent(out) :: ptype(*)
            real(c_double), intent(out) :: x(*), y(*), u(*), v(*), rho(*), pre(*), tem(*)
        end function

        integer(c_int) function lssph_create(p, num_total, num_int, ptype, x, y, u, v, rho, pre, tem, h) &
                bind(c, name="lssph_create")
            import :: c_int, c_int32_t, c_double, c_ptr, lssph_params
            type(lssph_params), intent(in) :: p
            integer(c_int32_t), value :: num_total, num_int
            integer(c_int32_t), intent(in) :: ptype(*)
            real(c_double), intent(in) :: x(*), y(*), u(*), v(*), rho(*), pre(*), tem(*)
            type(c_ptr), intent(out) :: h
        end function

        subroutine lssph_destroy(h) bind(c, name="lssph_destroy")
            import :: c_ptr
            type(c_ptr), value :: h
        end subroutine

        integer(c_int) function lssph_ghost(h) bind(c, name="lssph_ghost")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function

        integer(c_int) function lssph_step(h, nsteps, steady_step) bind(c, name="lssph_step")
            import :: c_int, c_int32_t, c_ptr
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nsteps
            integer(c_int32_t), intent(out) :: steady_step
        end function

        integer(c_int) function lssph_download(h, ptype, x, y, u, v, rho, pre, tem) bind(c, name="lssph_download")
            import :: c_int, c_int32_t, c_double, c_ptr
            type(c_ptr), value :: h
            integer(c_int32_t), intent(out) :: ptype(*)
            real(c_double), intent(out) :: x(*), y(*), u(*), v(*), rho(*), pre(*), tem(*)
        end function

        ! upload + nsteps steps + download in one call, the state updated in place
        integer(c_int) function lssph_advance_host(h, nsteps, x, y, u, v, rho, pre, tem, steady_step) &
                bind(c, name="lssph_advance_host")
            import :: c_int, c_int32_t, c_double, c_ptr
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nsteps
            real(c_double), intent(inout) :: x(*), y(*), u(*), v(*), rho(*), pre(*), tem(*)
            integer(c_int32_t), intent(out) :: steady_step
        end function

        integer(c_int) function lssph_write_param(h, results_root, config_h) bind(c, name="lssph_write_param")
            import :: c_int, c_char, c_ptr
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: results_root(*), config_h(*)
        end function

        integer(c_int) function lssph_write_data(h, results_root, step) bind(c, name="lssph_write_data")
            import :: c_int, c_int32_t, c_char, c_ptr
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: results_root(*)
            integer(c_int32_t), value :: step
        end function

        ! write_data that returns at once (device-side capture, background file write)
        integer(c_int) function lssph_write_data_async(h, results_root, step) bind(c, name="lssph_write_data_async")
            import :: c_int, c_int32_t, c_char, c_ptr
            type(c_ptr), value :: h
            character(kind=c_char), intent(in) :: results_root(*)
            integer(c_int32_t), value :: step
        end function

        integer(c_int) function lssph_snapshot_wait(h) bind(c, name="lssph_snapshot_wait")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function

        ! analysis/common/lssph_b.py main(): value, d/dx, d/dy at n_targets points
        integer(c_int) function lssph_lsb_interpolate(p, n, x, y, val, rho, n_targets, tx, ty, out) &
                bind(c, name="lssph_lsb_interpolate")
            import :: c_int, c_int32_t, c_double, lssph_params
            type(lssph_params), intent(in) :: p
            integer(c_int32_t), value :: n, n_targets
            real(c_double), intent(in) :: x(*), y(*), val(*), rho(*), tx(*), ty(*)
            real(c_double), intent(out) :: out(*)
        end function

        integer(c_int) function lssph_read_data(path, num_total, with_tem, ptype, x, y, u, v, rho, pre, tem) &
                bind(c, name="lssph_read_data")
            import :: c_int, c_int32_t, c_char, c_double
            character(kind=c_char), intent(in) :: path(*)
            integer(c_int32_t), value :: num_total, with_tem
            integer(c_int32_t), intent(out) :: ptype(*)
            real(c_double), intent(out) :: x(*), y(*), u(*), v(*), rho(*), pre(*), tem(*)
        end function

        ! ---- batched time loop, step budgets, device memory (no reference counterpart) ----
        integer(c_int) function lssph_batch_create(b) bind(c, name="lssph_batch_create")
            import :: c_int, c_ptr
            type(c_ptr), intent(out) :: b
        end function

        subroutine lssph_batch_destroy(b) bind(c, name="lssph_batch_destroy")
            import :: c_ptr
            type(c_ptr), value :: b
        end subroutine

        integer(c_int) function lssph_batch_add(b, h) bind(c, name="lssph_batch_add")
            import :: c_int, c_ptr
            type(c_ptr), value :: b, h
        end function

        integer(c_int) function lssph_batch_remove(b, h) bind(c, name="lssph_batch_remove")
            import :: c_int, c_ptr
            type(c_ptr), value :: b, h
        end function

        integer(c_int) function lssph_batch_step(b, nsteps, status, steady, steps_taken) &
                bind(c, name="lssph_batch_step")
            import :: c_int, c_int32_t, c_ptr
            type(c_ptr), value :: b
            integer(c_int32_t), value :: nsteps
            integer(c_int32_t), intent(out) :: status(*), steady(*), steps_taken(*)
        end function

        integer(c_int) function lssph_set_step_budget(h, nsteps) bind(c, name="lssph_set_step_budget")
            import :: c_int, c_int32_t, c_ptr
            type(c_ptr), value :: h
            integer(c_int32_t), value :: nsteps
        end function

        integer(c_int) function lssph_get_progress(h, steps_done, stopped) bind(c, name="lssph_get_progress")
            import :: c_int, c_int32_t, c_ptr
            type(c_ptr), value :: h
            integer(c_int32_t), intent(out) :: steps_done, stopped
        end function

        integer(c_int) function lssph_estimate_device_bytes(p, bytes) bind(c, name="lssph_estimate_device_bytes")
            import :: c_int, c_int64_t, lssph_params
            type(lssph_params), intent(in) :: p
            integer(c_int64_t), intent(out) :: bytes
        end function

        type(c_ptr) function lssph_last_error_c() bind(c, name="lssph_last_error")
            import :: c_ptr
        end function
    end interface

contains

    ! Message of the last failed call, as a Fortran string.
    function lssph_last_error_f() result(msg)
        character(len=:), allocatable :: msg
        character(kind=c_char), pointer :: cs(:)
        integer :: n
        interface
            integer(c_size_t) function c_strlen(s) bind(c, name="strlen")
                import :: c_size_t, c_ptr
                type(c_ptr), value :: s
            end function
        end interface
        type(c_ptr) :: p
        p = lssph_last_error_c()
        n = int(c_strlen(p))
        call c_f_pointer(p, cs, [n])
        allocate(character(len=n) :: msg)
        msg = transfer(cs(1:n), msg)
    end function

end module lssph_cuda_mod
