! ============================================================================ !
!   main_gpu -- the time loop of LS-SPH-Benchmarks (source/main.f90:15-168) on
!   the B200 engine.  Parameters, particle setup, restart files and the
!   results/ layout are those of the reference; every RK stage, ghost update,
!   particle shift and steady-state check runs on the GPU inside lssph_step.
!
!   Build (where a Fortran compiler exists):
!     gfortran -O2 lssph_cuda_mod.f90 main_gpu.f90 \
!              -L../lib -llssph -Wl,-rpath,'$ORIGIN/../lib' -o start_calculation_gpu
!   Run from the directory that holds config.h, like ./start_calculation.
! ============================================================================ !
program main_gpu
    use iso_c_binding
    use lssph_cuda_mod
    implicit none

    type(lssph_params) :: p
    type(c_ptr)        :: h
    integer(c_int32_t) :: num_total, num_int, steady, chunk
    integer            :: step, loop_start, rc
    integer(c_int32_t), allocatable :: ptype(:)
    real(c_double), allocatable :: x(:), y(:), u(:), v(:), rho(:), pre(:), tem(:)
    character(len=1024) :: restart_file, step_str

    ! init_param + check_param (main.f90:53-56)
    rc = lssph_params_from_config("config.h" // c_null_char, p)
    if (rc /= LSSPH_OK) then
        write(*,*) "Fatal Error in setup: ", lssph_last_error_f()
        error stop
    endif

    ! init_particle (main.f90:73): fresh start or restart
    rc = lssph_setup_counts(p, num_total, num_int)
    allocate(ptype(num_total), x(num_total), y(num_total), u(num_total), v(num_total), &
             rho(num_total), pre(num_total), tem(num_total))
    rc = lssph_setup_particles(p, num_total, ptype, x, y, u, v, rho, pre, tem)
    if (trim(adjustl(c_to_f(p%read_name))) /= "new") then
        write(step_str, *) p%start_step
        restart_file = "results/" // trim(adjustl(c_to_f(p%read_name))) // "/data/" // &
                       trim(adjustl(step_str)) // ".dat"
        rc = lssph_read_data(trim(restart_file) // c_null_char, num_total, merge(1, 0, p%target_problem == 4), &
                             ptype, x, y, u, v, rho, pre, tem)
        if (rc /= LSSPH_OK) then
            write(*,*) "Fatal Error in restart: ", lssph_last_error_f()
            error stop
        endif
    endif

    ! init_virtual_markers + init_cell + update_cell on the device (main.f90:77-85)
    rc = lssph_create(p, num_total, num_int, ptype, x, y, u, v, rho, pre, tem, h)
    if (rc /= LSSPH_OK) then
        write(*,*) "Fatal Error in setup: ", lssph_last_error_f()
        error stop
    endif

    ! write_param (with its ghost call) + write_data(0) for a fresh start (main.f90:91-94)
    if (trim(adjustl(c_to_f(p%read_name))) == "new") then
        rc = lssph_write_param(h, "results" // c_null_char, "config.h" // c_null_char)
        rc = lssph_write_data(h, "results" // c_null_char, 0)
        loop_start = p%start_step
    else
        loop_start = p%start_step + 1
    endif

    ! time loop (main.f90:119-166): advance to the next write step at a time
    step = loop_start
    do while (step <= p%end_step)
        chunk = min(p%end_step, ((step - 1) / p%write_step + 1) * p%write_step) - step + 1
        rc = lssph_step(h, chunk, steady)
        if (rc /= LSSPH_OK) then
            write(*,*) "Fatal Error in the time loop: ", lssph_last_error_f()
            error stop
        endif
        if (steady > 0) then
            write(*,*) "  Reached a steady state at step: ", step + steady - 1
            rc = lssph_write_data(h, "results" // c_null_char, step + steady - 1)
            exit
        endif
        step = step + chunk
        ! the snapshot is written in the background while the next chunk steps
        if (mod(step - 1, p%write_step) == 0) rc = lssph_write_data_async(h, "results" // c_null_char, step - 1)
        if (rc /= LSSPH_OK) then
            write(*,*) "Fatal Error while writing data: ", lssph_last_error_f()
            error stop
        endif
    enddo

    rc = lssph_snapshot_wait(h)
    call lssph_destroy(h)

contains

    function c_to_f(cs) result(s)
        character(kind=c_char), intent(in) :: cs(:)
        character(len=size(cs)) :: s
        integer :: i
        s = " "
        do i = 1, size(cs)
            if (cs(i) == c_null_char) exit
            s(i:i) = cs(i)
        enddo
    end function

end program main_gpu
