!-------------------------------------------------------------------------------
!> module mod_dg_gpu
!!
!! @par Description
!!      ISO_C_BINDING interface of the B200 DG advection library
!!      (libsdg_gpu.so, C ABI in include/sdg_gpu.h) for the Fortran driver of
!!      scale-dg-kernel-extraction.  It adds the "GPU" evaluation type next to
!!      GENERAL and OPT1: dg_gpu_setup uploads the operators and mesh tables
!!      once, dg_gpu_cal_tend replaces advect3d_eq_cal_tend
!!      (mod_advect3d_eq.f90:41-85) with identical arguments, and the
!!      resident calls (dg_gpu_set_state, dg_gpu_rk3_steps, dg_gpu_minmax,
!!      dg_gpu_get_state) run the whole time loop of main.f90:51-80 on the GPU.
!!
!!      Every C entry point returns an integer status; the wrappers stop with
!!      the library's message on failure (the reference aborts through the
!!      Fortran runtime on its own errors).
!!
!!      Note: no Fortran compiler exists in the image this library is built
!!      in, so this file is not compile-checked there.
!<
module mod_dg_gpu
  use, intrinsic :: iso_c_binding, only: &
    c_int, c_double, c_ptr, c_null_ptr, c_char, c_null_char, c_long_long, &
    c_associated
  implicit none
  private

  public :: dg_gpu_setup, dg_gpu_finalize, dg_gpu_cal_tend
  public :: dg_gpu_set_state, dg_gpu_get_state, dg_gpu_rk3_steps, dg_gpu_minmax
  public :: SDG_FLAG_EXACT, SDG_FLAG_ORDER_GENERAL, SDG_FLAG_MIXED
  public :: sdg_divlike_dev, sdg_gradlike_dev

  integer(c_int), parameter :: SDG_FLAG_EXACT = 1
  integer(c_int), parameter :: SDG_FLAG_ORDER_GENERAL = 2
  integer(c_int), parameter :: SDG_FLAG_MIXED = 4
  integer(c_int), parameter :: SDG_FIELD_Q = 0, SDG_FIELD_U = 1, &
                               SDG_FIELD_V = 2, SDG_FIELD_W = 3

  type(c_ptr), save :: handle = c_null_ptr

  interface
    integer(c_int) function sdg_last_error(buf, buflen) bind(C, name="sdg_last_error")
      import :: c_int, c_char
      character(kind=c_char), intent(out) :: buf(*)
      integer(c_int), value :: buflen
    end function
    integer(c_int) function sdg_init(h, Nq, Np, NfpTot, Ne, NeA, NhaloNode, &
        D1D, Lift_mat, VMapM, VMapP, halo_src_map, normal_fn, Escale, Fscale, &
        flags) bind(C, name="sdg_init")
      import :: c_int, c_double, c_ptr
      type(c_ptr), intent(out) :: h
      integer(c_int), value :: Nq, Np, NfpTot, Ne, NeA, NhaloNode, flags
      real(c_double), intent(in) :: D1D(*), Lift_mat(*), normal_fn(*), Escale(*), Fscale(*)
      integer(c_int), intent(in) :: VMapM(*), VMapP(*), halo_src_map(*)
    end function
    integer(c_int) function sdg_finalize(h) bind(C, name="sdg_finalize")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function sdg_cal_tend(h, dqdt, q, u, v, w) bind(C, name="sdg_cal_tend")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), intent(out) :: dqdt(*)
      real(c_double), intent(in) :: q(*), u(*), v(*), w(*)
    end function
    integer(c_int) function sdg_set_field(h, which, host) bind(C, name="sdg_set_field")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: which
      real(c_double), intent(in) :: host(*)
    end function
    integer(c_int) function sdg_get_field(h, which, host) bind(C, name="sdg_get_field")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: h
      integer(c_int), value :: which
      real(c_double), intent(out) :: host(*)
    end function
    integer(c_int) function sdg_rk3_steps(h, dt, nsteps) bind(C, name="sdg_rk3_steps")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function
    !> sdg_set_field(q) + sdg_rk3_steps + sdg_get_field(q) in one call, with
    !! the copies overlapping the stages chunk by chunk (q pinned for that).
    integer(c_int) function sdg_rk3_steps_host(h, q, dt, nsteps) &
        bind(C, name="sdg_rk3_steps_host")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), intent(inout) :: q(*)
      real(c_double), value :: dt
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function sdg_minmax(h, qmin, qmax) bind(C, name="sdg_minmax")
      import :: c_int, c_double, c_ptr
      type(c_ptr), value :: h
      real(c_double), intent(out) :: qmin, qmax
    end function
    !> x-, y- and z-derivatives of nvar fields per element, on device arrays
    !! (addresses from, e.g., an OpenACC host_data use_device region); replaces
    !! element_operation_kernel_matvec_divlike_dirXYZ_var5_P<p>
    !! (mod_dg_optr_kernel_opt1.F90.erb:347-465) over all elements at once.
    !! Array layout: vec_in_x(Np, nvar) of each element, stacked over elements.
    integer(c_int) function sdg_divlike_dev(Nq, nvar, Ne, D1D, in_x, in_y, in_z, &
        out_x, out_y, out_z, flags, stream) bind(C, name="sdg_divlike_dev")
      import :: c_int, c_long_long, c_double, c_ptr
      integer(c_int), value :: Nq, nvar
      integer(c_long_long), value :: Ne
      real(c_double), intent(in) :: D1D(*)
      type(c_ptr), value :: in_x, in_y, in_z, out_x, out_y, out_z
      integer(c_int), value :: flags
      type(c_ptr), value :: stream
    end function
    !> The three derivatives of one field per element; replaces
    !! element_operation_kernel_matvec_gradlike_dirXYZ_P<p> (erb:166-219).
    integer(c_int) function sdg_gradlike_dev(Nq, Ne, D1D, vec_in, out_x, out_y, out_z, &
        flags, stream) bind(C, name="sdg_gradlike_dev")
      import :: c_int, c_long_long, c_double, c_ptr
      integer(c_int), value :: Nq
      integer(c_long_long), value :: Ne
      real(c_double), intent(in) :: D1D(*)
      type(c_ptr), value :: vec_in, out_x, out_y, out_z
      integer(c_int), value :: flags
      type(c_ptr), value :: stream
    end function
  end interface

contains

  subroutine check(rc, what)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: what
    character(kind=c_char) :: buf(512)
    character(len=512) :: msg
    integer :: n, i
    if (rc == 0) return
    n = sdg_last_error(buf, 512_c_int)
    msg = ' '
    do i = 1, min(n, 511)
      msg(i:i) = buf(i)
    end do
    write(*,'(A,A,A,I0,A,A)') 'dg_gpu: ', what, ' failed (status ', rc, '): ', trim(msg)
    error stop 3
  end subroutine check

  !> Uploads the operators and mesh tables once ("GPU" evaluation type).
  !! flags: 0 = FMA kernels; SDG_FLAG_EXACT (+ SDG_FLAG_ORDER_GENERAL) =
  !! bit-for-bit OPT1 (GENERAL) rounding; SDG_FLAG_MIXED = FP32 tendency.
  subroutine dg_gpu_setup(D1D, Lift_mat, VMapM, VMapP, halo_src_map, &
      normal_fn, Escale, Fscale, Nq, Np, NfpTot, Ne, NeA, NhaloNode, flags)
    integer, intent(in) :: Nq, Np, NfpTot, Ne, NeA, NhaloNode, flags
    real(c_double), intent(in) :: D1D(Nq,Nq), Lift_mat(Nq,Nq,Nq,6)
    integer(c_int), intent(in) :: VMapM(NfpTot,Ne), VMapP(NfpTot,Ne)
    integer(c_int), intent(in) :: halo_src_map(NhaloNode)
    real(c_double), intent(in) :: normal_fn(NfpTot,Ne,3), Escale(Np,Ne,3), Fscale(NfpTot,Ne)
    if (c_associated(handle)) call check(sdg_finalize(handle), 'sdg_finalize')
    call check(sdg_init(handle, int(Nq,c_int), int(Np,c_int), int(NfpTot,c_int), &
      int(Ne,c_int), int(NeA,c_int), int(NhaloNode,c_int), D1D, Lift_mat, VMapM, &
      VMapP, halo_src_map, normal_fn, Escale, Fscale, int(flags,c_int)), 'sdg_init')
  end subroutine dg_gpu_setup

  subroutine dg_gpu_finalize()
    if (c_associated(handle)) call check(sdg_finalize(handle), 'sdg_finalize')
    handle = c_null_ptr
  end subroutine dg_gpu_finalize

  !> Same arguments as advect3d_eq_cal_tend (mod_advect3d_eq.f90:41-65); the
  !! mesh and operator arguments were uploaded by dg_gpu_setup and are unused.
  subroutine dg_gpu_cal_tend(dqdt, q, u, v, w, Np, NeA)
    integer, intent(in) :: Np, NeA
    real(c_double), intent(out) :: dqdt(Np,NeA)
    real(c_double), intent(in) :: q(Np,NeA), u(Np,NeA), v(Np,NeA), w(Np,NeA)
    call check(sdg_cal_tend(handle, dqdt, q, u, v, w), 'sdg_cal_tend')
  end subroutine dg_gpu_cal_tend

  subroutine dg_gpu_set_state(q, u, v, w, Np, NeA)
    integer, intent(in) :: Np, NeA
    real(c_double), intent(in) :: q(Np,NeA), u(Np,NeA), v(Np,NeA), w(Np,NeA)
    call check(sdg_set_field(handle, SDG_FIELD_Q, q), 'sdg_set_field(q)')
    call check(sdg_set_field(handle, SDG_FIELD_U, u), 'sdg_set_field(u)')
    call check(sdg_set_field(handle, SDG_FIELD_V, v), 'sdg_set_field(v)')
    call check(sdg_set_field(handle, SDG_FIELD_W, w), 'sdg_set_field(w)')
  end subroutine dg_gpu_set_state

  subroutine dg_gpu_get_state(q, Np, Ne)
    integer, intent(in) :: Np, Ne
    real(c_double), intent(out) :: q(Np,Ne)
    call check(sdg_get_field(handle, SDG_FIELD_Q, q), 'sdg_get_field')
  end subroutine dg_gpu_get_state

  subroutine dg_gpu_rk3_steps(dt, nsteps)
    real(c_double), intent(in) :: dt
    integer, intent(in) :: nsteps
    call check(sdg_rk3_steps(handle, dt, int(nsteps,c_int)), 'sdg_rk3_steps')
  end subroutine dg_gpu_rk3_steps

  subroutine dg_gpu_minmax(qmin, qmax)
    real(c_double), intent(out) :: qmin, qmax
    call check(sdg_minmax(handle, qmin, qmax), 'sdg_minmax')
  end subroutine dg_gpu_minmax

end module mod_dg_gpu
