! gatt_dns_mod.f90 -- ISO_C_BINDING interface to the B200 hot-path library
! (include/gatt_dns.h).  A reference build adds this module to its makefile and calls
! these functions from main.F90 in place of RK4_2D/RK4_3D, applyFilters2D/3D, the SFD
! block and applyBoundCond.  Arrays are passed exactly as main.F90
! already holds them (explicit-shape real*8 / integer arrays, column-major, 1-based
! indices inside index arrays).
module gatt_dns
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: GATT_OK = 0, GATT_ERR_CUDA = 1, GATT_ERR_BADARG = 2, &
        GATT_ERR_BADCOEF = 3, GATT_ERR_DIVERGED = 4, GATT_ERR_TIMEOUT = 5, GATT_ERR_STATE = 6, &
        GATT_ERR_NOMEM = 7
    integer(c_int), parameter :: GATT_VAR_U = 0, GATT_VAR_V = 1, GATT_VAR_W = 2, GATT_VAR_R = 3, &
        GATT_VAR_E = 4
    integer(c_int), parameter :: GATT_BC_DIRICHLET = 0, GATT_BC_NEUMANN = 1, GATT_BC_SECOND = 2
    integer(c_int), parameter :: GATT_DIST_LID_DRIVEN = 1
    integer(c_int), parameter :: GATT_DIST_PERIODIC_SINE = 2
    integer(c_int), parameter :: GATT_DIST_HOLD_INLET = 3

    interface
        function gatt_strerror(code) bind(C, name='gatt_strerror')
            import :: c_int, c_ptr
            integer(c_int), value :: code
            type(c_ptr) :: gatt_strerror
        end function
        function gatt_last_error() bind(C, name='gatt_last_error')
            import :: c_ptr
            type(c_ptr) :: gatt_last_error
        end function
        function gatt_create(ctx, nx, ny, nz, nbatch) bind(C, name='gatt_create')
            import :: c_int, c_ptr
            type(c_ptr) :: ctx
            integer(c_int), value :: nx, ny, nz, nbatch
            integer(c_int) :: gatt_create
        end function
        subroutine gatt_destroy(ctx) bind(C, name='gatt_destroy')
            import :: c_ptr
            type(c_ptr), value :: ctx
        end subroutine
        function gatt_set_stream(ctx, stream) bind(C, name='gatt_set_stream')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx, stream
            integer(c_int) :: gatt_set_stream
        end function
        function gatt_set_physics(ctx, Re, Ma, Pr, gamma, T0) bind(C, name='gatt_set_physics')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: Re, Ma, Pr, gamma, T0
            integer(c_int) :: gatt_set_physics
        end function
        function gatt_set_matrices(ctx, dir, kind, periodic, nRHS, nTypes, A, B, C, D, R, nBlocks, blocks) &
                bind(C, name='gatt_set_matrices')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: dir, kind, periodic, nRHS, nTypes, nBlocks
            real(c_double), dimension(*) :: A, B, C, D, R
            integer(c_int), dimension(*) :: blocks
            integer(c_int) :: gatt_set_matrices
        end function
        function gatt_set_filter(ctx, fx, fy, fz, filterCharTime) bind(C, name='gatt_set_filter')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: fx, fy, fz
            real(c_double), value :: filterCharTime
            integer(c_int) :: gatt_set_filter
        end function
        function gatt_set_time_stepping(ctx, timeStepping) bind(C, name='gatt_set_time_stepping')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), value :: timeStepping
            integer(c_int) :: gatt_set_time_stepping
        end function
        function gatt_set_neumann(ctx, n1, c1, n2, c2) bind(C, name='gatt_set_neumann')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: n1, n2
            real(c_double), dimension(*) :: c1, c2
            integer(c_int) :: gatt_set_neumann
        end function
        function gatt_set_bc(ctx, var, kind, n, ind, val, dirs) bind(C, name='gatt_set_bc')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: var, kind, n
            integer(c_int), dimension(*) :: ind, dirs
            real(c_double), dimension(*) :: val
            integer(c_int) :: gatt_set_bc
        end function
        function gatt_set_corners(ctx, cN, cL, cD, cAdiabatic) bind(C, name='gatt_set_corners')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), value :: cN
            integer(c_int), dimension(*) :: cL, cD, cAdiabatic
            integer(c_int) :: gatt_set_corners
        end function
        function gatt_add_disturbance(ctx, dtype, var, ind, x, npar, par) bind(C, name='gatt_add_disturbance')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: dtype, var, npar
            integer(c_int), dimension(6) :: ind
            real(c_double), dimension(*) :: x, par
            integer(c_int) :: gatt_add_disturbance
        end function
        function gatt_clear_disturbances(ctx) bind(C, name='gatt_clear_disturbances')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int) :: gatt_clear_disturbances
        end function
        function gatt_add_forcing(ctx, ftype, ind, npar, par) bind(C, name='gatt_add_forcing')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: ftype, npar
            integer(c_int), dimension(6) :: ind
            real(c_double), dimension(*) :: par
            integer(c_int) :: gatt_add_forcing
        end function
        function gatt_clear_forcings(ctx) bind(C, name='gatt_clear_forcings')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int) :: gatt_clear_forcings
        end function
        function gatt_set_sfd(ctx, stype, Delta, chiValue, chi) bind(C, name='gatt_set_sfd')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: stype
            real(c_double), value :: Delta, chiValue
            real(c_double), dimension(*) :: chi
            integer(c_int) :: gatt_set_sfd
        end function
        function gatt_upload(ctx, b, U, V, W, R, E) bind(C, name='gatt_upload')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b
            real(c_double), dimension(*) :: U, V, W, R, E
            integer(c_int) :: gatt_upload
        end function
        function gatt_download(ctx, b, U, V, W, R, E) bind(C, name='gatt_download')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b
            real(c_double), dimension(*) :: U, V, W, R, E
            integer(c_int) :: gatt_download
        end function
        function gatt_upload_mean(ctx, b, U, V, W, R, E) bind(C, name='gatt_upload_mean')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b
            real(c_double), dimension(*) :: U, V, W, R, E
            integer(c_int) :: gatt_upload_mean
        end function
        function gatt_download_mean(ctx, b, U, V, W, R, E) bind(C, name='gatt_download_mean')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b
            real(c_double), dimension(*) :: U, V, W, R, E
            integer(c_int) :: gatt_download_mean
        end function
        function gatt_upload_wnew(ctx, b, Wnew) bind(C, name='gatt_upload_wnew')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b
            real(c_double), dimension(*) :: Wnew
            integer(c_int) :: gatt_upload_wnew
        end function
        function gatt_download_wnew(ctx, b, Wnew) bind(C, name='gatt_download_wnew')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b
            real(c_double), dimension(*) :: Wnew
            integer(c_int) :: gatt_download_wnew
        end function
        function gatt_state_device_ptr(ctx, b, var, dptr) bind(C, name='gatt_state_device_ptr')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int), value :: b, var
            type(c_ptr) :: dptr
            integer(c_int) :: gatt_state_device_ptr
        end function
        function gatt_apply_bc(ctx, t) bind(C, name='gatt_apply_bc')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: t
            integer(c_int) :: gatt_apply_bc
        end function
        function gatt_deriv_dir(ctx, dir, kind, F, dF) bind(C, name='gatt_deriv_dir')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: dir, kind
            real(c_double), dimension(*) :: F, dF
            integer(c_int) :: gatt_deriv_dir
        end function
        function gatt_rhs(ctx, U, V, W, R, E, dU, dV, dW, dR, dE) bind(C, name='gatt_rhs')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*) :: U, V, W, R, E, dU, dV, dW, dR, dE
            integer(c_int) :: gatt_rhs
        end function
        function gatt_filter(ctx, blend) bind(C, name='gatt_filter')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: blend
            integer(c_int) :: gatt_filter
        end function
        function gatt_step(ctx, t, dt, maxChange) bind(C, name='gatt_step')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: t, dt
            real(c_double), dimension(*) :: maxChange
            integer(c_int) :: gatt_step
        end function
        function gatt_run(ctx, nsteps, t0, dt, maxChange) bind(C, name='gatt_run')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: nsteps
            real(c_double), value :: t0, dt
            real(c_double), dimension(*) :: maxChange
            integer(c_int) :: gatt_run
        end function
        function gatt_arnoldi(ctx, m, nsteps, t0, dt, eps, base, v0, region, H) bind(C, name='gatt_arnoldi')
            import :: c_int, c_ptr, c_double, c_signed_char
            type(c_ptr), value :: ctx
            integer(c_int), value :: m, nsteps
            real(c_double), value :: t0, dt, eps
            real(c_double), dimension(*) :: base, v0, H
            integer(c_signed_char), dimension(*) :: region
            integer(c_int) :: gatt_arnoldi
        end function
        function gatt_arnoldi_vector(ctx, b, j, out) bind(C, name='gatt_arnoldi_vector')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: b, j
            real(c_double), dimension(*) :: out
            integer(c_int) :: gatt_arnoldi_vector
        end function
        function gatt_rhs_jvp(ctx, q, dq, dk) bind(C, name='gatt_rhs_jvp')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*) :: q, dq, dk
            integer(c_int) :: gatt_rhs_jvp
        end function
        function gatt_rhs_vjp(ctx, q, a, lam) bind(C, name='gatt_rhs_vjp')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*) :: q, a, lam
            integer(c_int) :: gatt_rhs_vjp
        end function
        function gatt_jvp(ctx, nsteps, t0, dt, dq0, dqN) bind(C, name='gatt_jvp')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: nsteps
            real(c_double), value :: t0, dt
            real(c_double), dimension(*) :: dq0, dqN
            integer(c_int) :: gatt_jvp
        end function
        function gatt_vjp(ctx, nsteps, t0, dt, checkpoint_every, lamN, lam0) bind(C, name='gatt_vjp')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: nsteps, checkpoint_every
            real(c_double), value :: t0, dt
            real(c_double), dimension(*) :: lamN, lam0
            integer(c_int) :: gatt_vjp
        end function
        function gatt_autotune(ctx, reps, family, blocks, us) bind(C, name='gatt_autotune')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            integer(c_int), value :: reps
            integer(c_int), dimension(*) :: family, blocks
            real(c_double), dimension(*) :: us
            integer(c_int) :: gatt_autotune
        end function
        function gatt_selftest_pipeline_timeout(ctx) bind(C, name='gatt_selftest_pipeline_timeout')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int) :: gatt_selftest_pipeline_timeout
        end function
        function gatt_max_velocity(ctx, vmax) bind(C, name='gatt_max_velocity')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), dimension(*) :: vmax
            integer(c_int) :: gatt_max_velocity
        end function
        function gatt_synchronize(ctx) bind(C, name='gatt_synchronize')
            import :: c_int, c_ptr
            type(c_ptr), value :: ctx
            integer(c_int) :: gatt_synchronize
        end function
        function gatt_kernel_launches(ctx) bind(C, name='gatt_kernel_launches')
            import :: c_ptr, c_long_long
            type(c_ptr), value :: ctx
            integer(c_long_long) :: gatt_kernel_launches
        end function
        function gatt_profile_kernels(ctx, t0, dt, nsteps, ms, launches) bind(C, name='gatt_profile_kernels')
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: ctx
            real(c_double), value :: t0, dt
            integer(c_int), value :: nsteps
            real(c_double), dimension(*) :: ms, launches
            integer(c_int) :: gatt_profile_kernels
        end function
        function gatt_profile_name(cls) bind(C, name='gatt_profile_name')
            import :: c_int, c_ptr
            integer(c_int), value :: cls
            type(c_ptr) :: gatt_profile_name
        end function
        function gatt_max_change_noalloc(nsets, nvar, n, a, b, maxChange, stream) &
                bind(C, name='gatt_max_change_noalloc')
            import :: c_int, c_ptr, c_double, c_long_long
            integer(c_int), value :: nsets, nvar
            integer(c_long_long), value :: n
            type(c_ptr), dimension(*) :: a, b
            real(c_double), dimension(*) :: maxChange
            type(c_ptr), value :: stream
            integer(c_int) :: gatt_max_change_noalloc
        end function
    end interface
end module gatt_dns
