! module_gpu.f90 -- iso_c_binding interface of the B200 time-step engine
! (include/hercules_b200.h) for the HERCULES Fortran host.
!
! The reference advances its state with argument-less subroutines on module
! globals: set-up in drive (src/module_navier_stokes.f90:53-129), the loop body
! (:142-165: screen_cpu_time, update_ri, time_advancement_fd/_sp, calculate_ubar)
! and the outputs that read the module arrays (:169-203). A patched drive calls
! the functions below in their place; host I/O stays in Fortran.
!
! The derived types mirror the C structs field for field (bind(C) gives them the
! C compiler's layout); tests/test_fortran_binding.py checks the offsets and the
! size of each against the compiled header and checks that every entry point of
! the header is bound here with the same number of arguments.
module module_gpu
    use, intrinsic :: iso_c_binding
    implicit none

    ! error codes
    integer(c_int), parameter :: HC_OK = 0, HC_ERR_ARG = -1, HC_ERR_PARAM = -2, HC_ERR_CUDA = -3, &
        HC_ERR_NOMEM = -4, HC_ERR_NAN = -5, HC_ERR_STATE = -6, HC_ERR_UNSUPPORTED = -7, HC_ERR_SIZE = -8

    ! precision modes
    integer(c_int), parameter :: HC_PREC_FP64 = 0, HC_PREC_MIXED = 1

    ! field ids of hc_upload / hc_download
    integer(c_int), parameter :: HC_FIELD_U = 0, HC_FIELD_V = 1, HC_FIELD_W = 2, HC_FIELD_P = 3, &
        HC_FIELD_T = 4, HC_FIELD_FF = 5, HC_FIELD_GG = 6, HC_FIELD_HH = 7, HC_FIELD_SS = 8,       &
        HC_FIELD_PHI = 9, HC_FIELD_MEAN_U = 10, HC_FIELD_MEAN_V = 11, HC_FIELD_MEAN_W = 12,      &
        HC_FIELD_MEAN_T = 13, HC_FIELD_MEAN_UU = 14, HC_FIELD_MEAN_VV = 15, HC_FIELD_MEAN_WW = 16, &
        HC_FIELD_MEAN_UW = 17, HC_FIELD_MEAN_VW = 18, HC_FIELD_MEAN_TT = 19, HC_FIELD_MEAN_TW = 20

    ! the namelists &domain &modeling &constants (src/module_parameters.f90:40-157)
    type, bind(C) :: hc_params
        integer(c_int) :: nx
        integer(c_int) :: ny
        integer(c_int) :: nz
        real(c_double) :: lx
        real(c_double) :: ly
        real(c_double) :: lz
        real(c_double) :: zstretch
        integer(c_int) :: ochannel
        integer(c_int) :: dp_opt
        integer(c_int) :: cds
        integer(c_int) :: issk
        integer(c_int) :: dts
        integer(c_int) :: isdamp
        integer(c_int) :: nzdamp
        real(c_double) :: cdamp
        real(c_double) :: nu
        real(c_double) :: alpha
        real(c_double) :: got
        real(c_double) :: fc
        real(c_double) :: ug
        real(c_double) :: vg
        real(c_double) :: dt
        integer(c_int) :: imax
        real(c_double) :: u_mrf
        integer(c_int) :: isscalar
        real(c_double) :: t_ref
        real(c_double) :: tbot
        real(c_double) :: ttop
        integer(c_int) :: is_ri_var
        real(c_double) :: ri_str
        real(c_double) :: ri_end
        integer(c_int) :: precision
        integer(c_int) :: tile(4)
        integer(c_int) :: tbc_bot         ! 0: T = tbot at the bottom wall; 1: dT/dz = tbot there
        integer(c_int) :: reserved(2)
    end type

    ! per-step diagnostics (screen_cpu_time, screen_div_error, calculate_ubar)
    type, bind(C) :: hc_diag
        real(c_double) :: time_sim
        real(c_double) :: cfl
        real(c_double) :: div_avg
        real(c_double) :: div_max
        real(c_double) :: div_hist_max
        real(c_double) :: ubar
        real(c_double) :: dpx_drive
        real(c_double) :: got
        real(c_double) :: div_avg_sub(3)
        real(c_double) :: div_max_sub(3)
        integer(c_int) :: nan_flag
        integer(c_int) :: step
    end type

    interface
        ! ---- the seam of drive
        integer(c_int) function hc_create(p, h) bind(C, name="hc_create")
            import :: c_int, c_ptr, hc_params
            type(hc_params), intent(in) :: p
            type(c_ptr), intent(out)    :: h
        end function
        integer(c_int) function hc_set_grid(h, dz, l_t, l_b, dz_t, dz_b) bind(C, name="hc_set_grid")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: dz(*), l_t(*), l_b(*), dz_t(*), dz_b(*)
        end function
        integer(c_int) function hc_get_grid(h, dz, l_t, l_b, dz_t, dz_b) bind(C, name="hc_get_grid")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: dz(*), l_t(*), l_b(*), dz_t(*), dz_b(*)
        end function
        integer(c_int) function hc_upload(h, id, a, ld1, ld2, ghost) bind(C, name="hc_upload")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: id
            real(c_double), intent(in) :: a(*)
            integer(c_int), value :: ld1, ld2, ghost
        end function
        integer(c_int) function hc_download(h, id, a, ld1, ld2, ghost) bind(C, name="hc_download")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: id
            real(c_double), intent(inout) :: a(*)
            integer(c_int), value :: ld1, ld2, ghost
        end function
        integer(c_int) function hc_initialize(h) bind(C, name="hc_initialize")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        integer(c_int) function hc_step(h, n, d) bind(C, name="hc_step")
            import :: c_int, c_ptr, hc_diag
            type(c_ptr), value :: h
            integer(c_int), value :: n
            type(hc_diag), intent(out) :: d(*)
        end function
        integer(c_int) function hc_get_scalars(h, time_sim, dpx_drive, ubar, got, div_hist_max, step) &
                bind(C, name="hc_get_scalars")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: time_sim, dpx_drive, ubar, got, div_hist_max
            integer(c_int), intent(out) :: step
        end function
        integer(c_int) function hc_destroy(h) bind(C, name="hc_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
        end function
        type(c_ptr) function hc_error_string(code) bind(C, name="hc_error_string")
            import :: c_int, c_ptr
            integer(c_int), value :: code
        end function

        ! ---- device-pointer variants, timing, profiling
        integer(c_int) function hc_upload_dev(h, id, dev) bind(C, name="hc_upload_dev")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: id
            type(c_ptr), value :: dev
        end function
        integer(c_int) function hc_download_dev(h, id, dev) bind(C, name="hc_download_dev")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: id
            type(c_ptr), value :: dev
        end function
        integer(c_int) function hc_last_step_ms(h, ms) bind(C, name="hc_last_step_ms")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(out) :: ms
        end function
        integer(c_int) function hc_last_launch_count(h, n) bind(C, name="hc_last_launch_count")
            import :: c_int, c_ptr, c_long_long
            type(c_ptr), value :: h
            integer(c_long_long), intent(out) :: n
        end function
        integer(c_int) function hc_set_profiling(h, enable) bind(C, name="hc_set_profiling")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: enable
        end function
        integer(c_int) function hc_kernel_profile(h, max, names, total_ms, launches, count) &
                bind(C, name="hc_kernel_profile")
            import :: c_int, c_ptr, c_double, c_long_long, c_char
            type(c_ptr), value :: h
            integer(c_int), value :: max
            character(kind=c_char), intent(out) :: names(*)        ! max slots of 32 characters
            real(c_double), intent(out) :: total_ms(*)
            integer(c_long_long), intent(out) :: launches(*)
            integer(c_int), intent(out) :: count
        end function
        integer(c_int) function hc_divergence_noalloc(p, dz, u, v, w, out_dev, stream) &
                bind(C, name="hc_divergence_noalloc")
            import :: c_int, c_ptr, c_double, hc_params
            type(hc_params), intent(in) :: p
            real(c_double), intent(in) :: dz(*)
            type(c_ptr), value :: u, v, w, out_dev, stream   ! device addresses, cudaStream_t
        end function

        ! ---- beyond the reference: body force, graph replay, ensemble, adjoint
        integer(c_int) function hc_set_body_force(h, fx, fy, fz) bind(C, name="hc_set_body_force")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: fx(*), fy(*), fz(*)    ! interior (nx,ny,nz) arrays
        end function
        integer(c_int) function hc_set_graph(h, enable) bind(C, name="hc_set_graph")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: enable
        end function
        integer(c_int) function hc_ensemble_create(members, n, e) bind(C, name="hc_ensemble_create")
            import :: c_int, c_ptr
            type(c_ptr), intent(in) :: members(*)
            integer(c_int), value :: n
            type(c_ptr), intent(out) :: e
        end function
        integer(c_int) function hc_ensemble_step(e, n) bind(C, name="hc_ensemble_step")
            import :: c_int, c_ptr
            type(c_ptr), value :: e
            integer(c_int), value :: n
        end function
        integer(c_int) function hc_ensemble_last_ms(e, ms, launches_per_step) bind(C, name="hc_ensemble_last_ms")
            import :: c_int, c_ptr, c_double, c_long_long
            type(c_ptr), value :: e
            real(c_double), intent(out) :: ms
            integer(c_long_long), intent(out) :: launches_per_step
        end function
        integer(c_int) function hc_ensemble_destroy(e) bind(C, name="hc_ensemble_destroy")
            import :: c_int, c_ptr
            type(c_ptr), value :: e
        end function
        integer(c_int) function hc_adjoint_forward(h, n, ckpt) bind(C, name="hc_adjoint_forward")
            import :: c_int, c_ptr
            type(c_ptr), value :: h
            integer(c_int), value :: n, ckpt
        end function
        integer(c_int) function hc_adjoint_reverse(h, lu, lv, lw, lp, gu, gv, gw, gp, gbf) &
                bind(C, name="hc_adjoint_reverse")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: lu(*), lv(*), lw(*), lp(*)      ! seeds dJ/d(field at step N)
            real(c_double), intent(out) :: gu(*), gv(*), gw(*), gp(*)     ! dJ/d(field at step 0)
            real(c_double), intent(out) :: gbf(*)                         ! dJ/d(body force), 3*nx*ny*nz
        end function
        integer(c_int) function hc_adjoint_reverse_t(h, lu, lv, lw, lp, lt, gu, gv, gw, gp, gt, gbf) &
                bind(C, name="hc_adjoint_reverse_t")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            real(c_double), intent(in) :: lu(*), lv(*), lw(*), lp(*), lt(*)   ! seeds, t included
            real(c_double), intent(out) :: gu(*), gv(*), gw(*), gp(*), gt(*)  ! gradients, t included
            real(c_double), intent(out) :: gbf(*)
        end function
        integer(c_int) function hc_adjoint(h, n, ckpt, lu, lv, lw, lp, gu, gv, gw, gp, gbf) &
                bind(C, name="hc_adjoint")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: h
            integer(c_int), value :: n, ckpt
            real(c_double), intent(in) :: lu(*), lv(*), lw(*), lp(*)
            real(c_double), intent(out) :: gu(*), gv(*), gw(*), gp(*), gbf(*)
        end function
        integer(c_int) function hc_adjoint_last_ms(h, forward_ms, reverse_ms, forward_launches, reverse_launches) &
                bind(C, name="hc_adjoint_last_ms")
            import :: c_int, c_ptr, c_double, c_long_long
            type(c_ptr), value :: h
            real(c_double), intent(out) :: forward_ms, reverse_ms
            integer(c_long_long), intent(out) :: forward_launches, reverse_launches
        end function
    end interface
end module module_gpu
