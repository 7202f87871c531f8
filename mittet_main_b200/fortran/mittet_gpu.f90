!-----------------------------------------------------------------------------
! mittet_gpu -- Fortran 2003 iso_c_binding interface to libmittet_b200.so
! (the C ABI of include/mittet.h), for the reference's ncver0027 driver.
!
! One call sequence replaces the per-shot time loop of ncver0027/cpu_main.f90
! (lines 99-143: read_source_3d, e_field_cpml4, CPML_E4, h_field_cpml4,
! CPML_H4, output_EH_J) and the DFT of f_to_d_e / f_to_d_h
! (cpu_f_to_d_e.f90:134-160, cpu_f_to_d_h.f90:141-167).  The driver keeps
! computing sig, myu, the source/receiver indices and the const_para scalars
! as before; sig(nx,ny,nz) column-major is exactly the x-fastest layout the
! C ABI takes, and 1-based (ix,iy,iz) positions are passed unchanged.
!
! No Fortran compiler was available where this build was made, so this
! module is provided as source.  Call sequence: mittet_phys_defaults,
! mittet_create, then mittet_set_model / mittet_set_sources /
! mittet_set_wavelet / mittet_set_receivers / mittet_set_freqs, then
! mittet_forward once per shot set, and mittet_destroy.
!-----------------------------------------------------------------------------
module mittet_gpu
    use iso_c_binding
    implicit none

    integer(c_int), parameter :: MITTET_OK = 0
    integer(c_int), parameter :: MITTET_FLAVOR_NCVER0027 = 0, MITTET_FLAVOR_SATAN_I = 1
    integer(c_int), parameter :: MITTET_FP32 = 0, MITTET_FP64 = 1
    integer(c_int), parameter :: MITTET_EX = 0, MITTET_EY = 1, MITTET_EZ = 2
    integer(c_int), parameter :: MITTET_HX = 3, MITTET_HY = 4, MITTET_HZ = 5
    integer(c_int), parameter :: MITTET_SRC_MAGNETIC = 0, MITTET_SRC_ELECTRIC = 1

    type, bind(c) :: mittet_grid
        integer(c_int32_t) :: nx, ny, nz
        real(c_double) :: dx, dy, dz
        integer(c_int32_t) :: ncpml
    end type

    type, bind(c) :: mittet_phys
        real(c_double) :: dt, omega0, cmax, mu0, c1, c2
        integer(c_int32_t) :: flavor, psi_hyx_typo, e_sign, h_sign
        real(c_double) :: cpml_nn, cpml_order, cpml_kappa_max, cpml_a_max, cpml_ma, cpml_rcoef, cpml_opt_to_max_x
        integer(c_int32_t) :: precision, device, check_cfl
    end type

    type, bind(c) :: mittet_point_source
        integer(c_int32_t) :: shot, ix, iy, iz, comp, kind
        real(c_double) :: amp
    end type

    type, bind(c) :: mittet_receiver
        integer(c_int32_t) :: ix, iy, iz, comp
    end type

    interface
        integer(c_int) function mittet_phys_defaults(flavor, phys) bind(c, name="mittet_phys_defaults")
            import :: c_int, c_int32_t, mittet_phys
            integer(c_int32_t), value :: flavor
            type(mittet_phys), intent(out) :: phys
        end function

        integer(c_int) function mittet_create(grid, phys, handle) bind(c, name="mittet_create")
            import :: c_int, c_ptr, mittet_grid, mittet_phys
            type(mittet_grid), intent(in) :: grid
            type(mittet_phys), intent(in) :: phys
            type(c_ptr), intent(out) :: handle
        end function

        subroutine mittet_destroy(handle) bind(c, name="mittet_destroy")
            import :: c_ptr
            type(c_ptr), value :: handle
        end subroutine

        integer(c_int) function mittet_set_model(handle, sigma, mu) bind(c, name="mittet_set_model")
            import :: c_int, c_ptr, c_double
            type(c_ptr), value :: handle
            real(c_double), intent(in) :: sigma(*)
            real(c_double), intent(in) :: mu(*)
        end function

        integer(c_int) function mittet_set_sources(handle, nshot, npoint, pts) bind(c, name="mittet_set_sources")
            import :: c_int, c_int32_t, c_ptr, mittet_point_source
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nshot, npoint
            type(mittet_point_source), intent(in) :: pts(*)
        end function

        integer(c_int) function mittet_set_wavelet(handle, nt, w) bind(c, name="mittet_set_wavelet")
            import :: c_int, c_int32_t, c_ptr, c_double
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nt
            real(c_double), intent(in) :: w(*)
        end function

        integer(c_int) function mittet_set_receivers(handle, nrec, rec) bind(c, name="mittet_set_receivers")
            import :: c_int, c_int32_t, c_ptr, mittet_receiver
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nrec
            type(mittet_receiver), intent(in) :: rec(*)
        end function

        integer(c_int) function mittet_set_freqs(handle, nf, omega, h_factor) bind(c, name="mittet_set_freqs")
            import :: c_int, c_int32_t, c_ptr, c_double
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nf, h_factor
            real(c_double), intent(in) :: omega(*)
        end function

        integer(c_int) function mittet_freq_grid_ref(nt, dt, nf, omega) bind(c, name="mittet_freq_grid_ref")
            import :: c_int, c_int32_t, c_double
            integer(c_int32_t), value :: nt, nf
            real(c_double), value :: dt
            real(c_double), intent(out) :: omega(*)
        end function

        ! rec_fd: complex(c_double_complex) rec_fd(nf, nrec, nshot); rec_td: real(c_double) rec_td(nt, nrec, nshot)
        integer(c_int) function mittet_forward(handle, nt, rec_fd, rec_td) bind(c, name="mittet_forward")
            import :: c_int, c_int32_t, c_ptr, c_double_complex, c_double
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nt
            complex(c_double_complex), intent(out) :: rec_fd(*)
            real(c_double), intent(out) :: rec_td(*)
        end function

        ! obs: complex(c_double_complex) obs(nf, nrec, nshot); grad(nx, ny, nz) (satan_i layout)
        integer(c_int) function mittet_gradient(handle, nt, obs, checkpoint_every, misfit, grad) &
                bind(c, name="mittet_gradient")
            import :: c_int, c_int32_t, c_ptr, c_double_complex, c_double
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nt, checkpoint_every
            complex(c_double_complex), intent(in) :: obs(*)
            real(c_double), intent(out) :: misfit
            real(c_double), intent(out) :: grad(*)
        end function

        ! frees the work buffers mittet_gradient keeps in the handle for its next call
        integer(c_int) function mittet_release_gradient_buffers(handle) &
                bind(c, name="mittet_release_gradient_buffers")
            import :: c_int, c_ptr
            type(c_ptr), value :: handle
        end function

        ! satan_i model update (calc_phi, trial forward, calc_alpha, update_para2):
        ! obs, ecal: complex(c_double_complex) (nf, nrec, nshot); grad, sigma: (nx, ny, nz);
        ! step(1) = scaler, step(2) = alpha; sigma is updated in place.
        integer(c_int) function mittet_fwi_update(handle, nt, obs, ecal, grad, iseabed, minval, maxval, sigma, step) &
                bind(c, name="mittet_fwi_update")
            import :: c_int, c_int32_t, c_ptr, c_double_complex, c_double
            type(c_ptr), value :: handle
            integer(c_int32_t), value :: nt, iseabed
            complex(c_double_complex), intent(in) :: obs(*), ecal(*)
            real(c_double), intent(in) :: grad(*)
            real(c_double), value :: minval, maxval
            real(c_double), intent(inout) :: sigma(*)
            real(c_double), intent(out) :: step(2)
        end function

        integer(c_int) function mittet_last_error(buf, len) bind(c, name="mittet_last_error")
            import :: c_int, c_char, c_size_t
            character(kind=c_char), intent(out) :: buf(*)
            integer(c_size_t), value :: len
        end function
    end interface
end module mittet_gpu
