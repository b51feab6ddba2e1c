! chemgen_m: the Fortran module a CFD solver uses to call getrates on the
! GPU, with the public interface of the reference's generated module
! (chemgen/templates/chemgen_mod.j2:1-166): init_chemgen(flag, ng) and
! getrates_gpu(P, T, ng, Y, wdot), bound to libchemgen_b200.so through
! ISO_C_BINDING.
!
! Build with the preprocessor (the .F90 suffix, or -cpp) and OpenMP offload,
! as the reference's module is built, and select the wrapper the same way:
! -DHIP_CHEM_v1 (default), -DHIP_CHEM_v2, -DHIP_CHEM_v3 or -DHIP_CHEM_v4.  All
! four wrappers run the same kernels here.  Link with
!   -L<dir> -lchemgen_b200 -Wl,-rpath,<dir>
! and, for the mechanism-specialised kernels, the module that
! generate_chemistry.py --language cuda --build wrote for the mechanism.
!
! Differences from the reference's module:
! * The mechanism comes from the blob file generate_chemistry.py writes
!   (named by the environment variable CHEMGEN_BLOB, else getrates.blob in
!   the working directory), where the reference's init_chemgen uploads arrays
!   compiled into its coef_m_v* modules (copyConstantsToDevice,
!   chemgen/constants.py:119-240).
! * The species count comes from the library (chemgen_global_num_species),
!   so Y and wdot are assumed-size in their second dimension.
! * A failing call prints the library's status and returns, as the
!   reference's HIP wrappers print and return (constants.py:7-24).
module chemgen_m
    use, intrinsic :: iso_c_binding
    implicit none
    private
    ! scratch the wrappers take (EG is unused here; C holds per-point state
    ! when a mechanism's state does not fit in shared memory)
    real(kind=8), allocatable, dimension(:,:) :: EG, C
    real(kind=8), allocatable, dimension(:) :: CTOT

    public :: init_chemgen
    public :: getrates_gpu

    interface
        subroutine getrates_hip_wrapper_v1(P, T, ng, Y, wdot, logEG, logC) bind(C, name="getrates_hip_wrapper_v1")
            import :: c_double, c_int
            real(c_double), intent(in) :: P(*)
            real(c_double), intent(in) :: T(*)
            integer(c_int), value, intent(in) :: ng
            real(c_double), intent(in) :: Y(*)
            real(c_double), intent(out) :: wdot(*)
            real(c_double), intent(in) :: logEG(*)
            real(c_double), intent(in) :: logC(*)
        end subroutine getrates_hip_wrapper_v1
        subroutine getrates_hip_wrapper_v2(P, T, ng, Y, wdot, logEG, logC) bind(C, name="getrates_hip_wrapper_v2")
            import :: c_double, c_int
            real(c_double), intent(in) :: P(*)
            real(c_double), intent(in) :: T(*)
            integer(c_int), value, intent(in) :: ng
            real(c_double), intent(in) :: Y(*)
            real(c_double), intent(out) :: wdot(*)
            real(c_double), intent(in) :: logEG(*)
            real(c_double), intent(in) :: logC(*)
        end subroutine getrates_hip_wrapper_v2
        subroutine getrates_hip_wrapper_v3(P, T, ng, Y, wdot, logEG, logC) bind(C, name="getrates_hip_wrapper_v3")
            import :: c_double, c_int
            real(c_double), intent(in) :: P(*)
            real(c_double), intent(in) :: T(*)
            integer(c_int), value, intent(in) :: ng
            real(c_double), intent(in) :: Y(*)
            real(c_double), intent(out) :: wdot(*)
            real(c_double), intent(in) :: logEG(*)
            real(c_double), intent(in) :: logC(*)
        end subroutine getrates_hip_wrapper_v3
        subroutine getrates_hip_wrapper_v4(P, T, ng, Y, wdot, logEG, logC) bind(C, name="getrates_hip_wrapper_v4")
            import :: c_double, c_int
            real(c_double), intent(in) :: P(*)
            real(c_double), intent(in) :: T(*)
            integer(c_int), value, intent(in) :: ng
            real(c_double), intent(in) :: Y(*)
            real(c_double), intent(out) :: wdot(*)
            real(c_double), intent(in) :: logEG(*)
            real(c_double), intent(in) :: logC(*)
        end subroutine getrates_hip_wrapper_v4
        subroutine allocate_intermediate_DeviceMemory(ng) bind(C, name="allocate_intermediate_DeviceMemory")
            import :: c_int
            integer(c_int), value, intent(in) :: ng
        end subroutine allocate_intermediate_DeviceMemory
        integer(c_int) function chemgen_init_constants_file(path) bind(C, name="chemgen_init_constants_file")
            import :: c_int, c_char
            character(kind=c_char), dimension(*), intent(in) :: path
        end function chemgen_init_constants_file
        integer(c_int) function chemgen_free_constants() bind(C, name="chemgen_free_constants")
            import :: c_int
        end function chemgen_free_constants
        integer(c_int) function chemgen_global_num_species() bind(C, name="chemgen_global_num_species")
            import :: c_int
        end function chemgen_global_num_species
        integer(c_int) function chemgen_last_wrapper_status() bind(C, name="chemgen_last_wrapper_status")
            import :: c_int
        end function chemgen_last_wrapper_status
    end interface

contains

!***************************************************************
! flag = 1: load the mechanism onto the current device and allocate the
! scratch for ng points; any other flag: release both.
subroutine init_chemgen(flag, ng)
    implicit none
    integer, intent(in) :: flag
    integer, intent(in) :: ng
    integer(c_int) :: ierr, ns
    if (flag .eq. 1) then
        ierr = chemgen_init_constants_file(c_null_char)
        if (ierr .ne. 0) then
            write(*, *) "chemgen_m: loading the mechanism blob failed, status ", ierr
            return
        endif
        ns = chemgen_global_num_species()
        allocate(EG(ng, ns))
        allocate(C(ng, ns))
        allocate(CTOT(ng))
!$omp target enter data map(alloc:EG,C,CTOT)
#ifdef HIP_CHEM_v4
        call allocate_intermediate_DeviceMemory(int(ng, c_int))
        if (chemgen_last_wrapper_status() .ne. 0) then
            write(*, *) "chemgen_m: reserving scratch failed, status ", chemgen_last_wrapper_status()
        endif
#endif
    else
        if (allocated(EG)) then
!$omp target exit data map(delete:EG,C,CTOT)
            deallocate(EG)
            deallocate(C)
            deallocate(CTOT)
        endif
        ierr = chemgen_free_constants()
    endif
end subroutine init_chemgen

!***************************************************************
! wdot(ng, ns) in mol/(cm^3 s) from P (dyne/cm^2), T (K) and mass fractions
! Y(ng, ns): the arrays are mapped to the device by the caller
! (!$omp target enter data), as the reference's mini app does.
subroutine getrates_gpu(P, T, ng, Y, wdot)
    implicit none
    integer, intent(in) :: ng
    real(kind=8), dimension(ng), intent(in) :: T, P
    real(kind=8), dimension(ng, *), intent(in) :: Y
    real(kind=8), dimension(ng, *), intent(out) :: wdot
    integer(c_int) :: ngc
    ngc = int(ng, c_int)
!$omp target data use_device_ptr(P, T, Y, wdot, EG, C)
#if defined(HIP_CHEM_v4)
    call getrates_hip_wrapper_v4(P, T, ngc, Y, wdot, EG, C)
#elif defined(HIP_CHEM_v3)
    call getrates_hip_wrapper_v3(P, T, ngc, Y, wdot, EG, C)
#elif defined(HIP_CHEM_v2)
    call getrates_hip_wrapper_v2(P, T, ngc, Y, wdot, EG, C)
#else
    call getrates_hip_wrapper_v1(P, T, ngc, Y, wdot, EG, C)
#endif
!$omp end target data
    if (chemgen_last_wrapper_status() .ne. 0) then
        write(*, *) "chemgen_m: getrates failed, status ", chemgen_last_wrapper_status()
    endif
end subroutine getrates_gpu

end module chemgen_m
