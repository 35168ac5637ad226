! les_gpu_shim.f90 -- Fortran binding of libles_gpu.so (include/les_gpu.h, include/les_mlp.h).
!
! Replaces comp1.o comp2.o compadv1.o compsgs1.o compsgs3.o derivs1.o
! derivs2.o press.o tridv.o filter_fftw.o lowerbc.o upperbc.o complen.o in
! LESOBJS (Makefile:11-14) so that les.F90 keeps driving the stage loop
! (les.F90:254-285) with the same subroutine names and arguments, while the
! domain lives on one GPU.  The storage module stays the host copy used for
! restart files and statistics output.  Not compiled in this repository (no
! Fortran compiler in the build image); see INTEGRATION.md.
module les_gpu
  use iso_c_binding
  implicit none

  type, bind(C) :: les_config
     integer(c_int) :: nnx, nny, nnz, imodel, isurface, tke_production, precision, device
     real(c_double) :: xl, yl, zl, z0, dt, cb, skc, nu, ugal, vgal, ufree, emin, forcing
  end type les_config

  type(c_ptr), save :: les_h = c_null_ptr

  interface
     integer(c_int) function les_gpu_init(cfg, h) bind(C, name="les_gpu_init")
       import :: les_config, c_ptr, c_int
       type(les_config), intent(in) :: cfg
       type(c_ptr), intent(out) :: h
     end function
     subroutine les_gpu_finalize(h) bind(C, name="les_gpu_finalize")
       import :: c_ptr
       type(c_ptr), value :: h
     end subroutine
     integer(c_int) function les_gpu_upload(h, u, v, w, e, p, rb) bind(C, name="les_gpu_upload")
       import :: c_ptr, c_int
       type(c_ptr), value :: h, u, v, w, e, p
       integer(c_int), value :: rb
     end function
     integer(c_int) function les_gpu_download(h, u, v, w, e, p, rb) bind(C, name="les_gpu_download")
       import :: c_ptr, c_int
       type(c_ptr), value :: h, u, v, w, e, p
       integer(c_int), value :: rb
     end function
     ! redim.f90 on the device: dst's state := src's state on dst's grid
     integer(c_int) function les_gpu_regrid(dst, src) bind(C, name="les_gpu_regrid")
       import :: c_ptr, c_int
       type(c_ptr), value :: dst, src
     end function
     integer(c_int) function les_gpu_lower(h) bind(C, name="les_gpu_lower")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
     end function
     integer(c_int) function les_gpu_upper(h) bind(C, name="les_gpu_upper")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
     end function
     integer(c_int) function les_gpu_comp1(h, it, mnout, istage, dtab1, dtab2, xkmax) &
          bind(C, name="les_gpu_comp1")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h
       integer(c_int), value :: it, mnout, istage
       real(c_double), value :: dtab1, dtab2, xkmax
     end function
     integer(c_int) function les_gpu_comprhs(h, dtabm) bind(C, name="les_gpu_comprhs")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h
       real(c_double), value :: dtabm
     end function
     integer(c_int) function les_gpu_press(h) bind(C, name="les_gpu_press")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
     end function
     integer(c_int) function les_gpu_comp2(h, dtab1) bind(C, name="les_gpu_comp2")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h
       real(c_double), value :: dtab1
     end function
     integer(c_int) function les_gpu_stats(h, meanbuf, scalars) bind(C, name="les_gpu_stats")
       import :: c_ptr, c_int
       type(c_ptr), value :: h, meanbuf, scalars
     end function
     ! learned closure (include/les_mlp.h): create a network, load the
     ! parameters of a weights file (params(9478), norm(34) as real(c_float)),
     ! attach it to a handle configured with imodel = 5
     integer(c_int) function les_mlp_create(device, m) bind(C, name="les_mlp_create")
       import :: c_ptr, c_int
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: m
     end function
     integer(c_int) function les_mlp_set_params(m, params, norm) bind(C, name="les_mlp_set_params")
       import :: c_ptr, c_int
       type(c_ptr), value :: m, params, norm
     end function
     integer(c_int) function les_gpu_set_mlp(h, m, re_tau) bind(C, name="les_gpu_set_mlp")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h, m
       real(c_double), value :: re_tau
     end function
     integer(c_int) function les_gpu_learned_status(h, used, dissipation) bind(C, name="les_gpu_learned_status")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h
       integer(c_int), intent(out) :: used
       real(c_double), intent(out) :: dissipation
     end function
     ! second fallback test: factor against the Deardorff dissipation (<= 0: off)
     integer(c_int) function les_gpu_set_learned_guard(h, ratio) bind(C, name="les_gpu_set_learned_guard")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h
       real(c_double), value :: ratio
     end function
     subroutine les_mlp_destroy(m) bind(C, name="les_mlp_destroy")
       import :: c_ptr
       type(c_ptr), value :: m
     end subroutine
     type(c_ptr) function les_gpu_last_error(h) bind(C, name="les_gpu_last_error")
       import :: c_ptr
       type(c_ptr), value :: h
     end function
  end interface

contains

  subroutine les_check(rc)
    integer(c_int), intent(in) :: rc
    if (rc /= 0) call lesabort("les_gpu call failed")   ! abort.F90:1-17
  end subroutine les_check

  ! --- drop-in replacements with the reference's names and arguments ---
  subroutine lower(istart, np, nm)
    integer :: istart, np(7), nm(7)
    call les_check(les_gpu_lower(les_h))
  end subroutine lower

  subroutine upper(np)
    integer :: np(7)
    call les_check(les_gpu_upper(les_h))
  end subroutine upper

  subroutine comp1(it, mnout, istart, iend, nm, np, istage)
    use storage, only: dtab1, dtab2, xkmax
    integer :: it, istart, iend, nm(4), np(4), istage
    logical :: mnout
    call les_check(les_gpu_comp1(les_h, it, merge(1, 0, mnout), istage, &
         real(dtab1, c_double), real(dtab2, c_double), real(xkmax, c_double)))
  end subroutine comp1

  subroutine comprhs(istart, iend)
    use storage, only: dtabm
    integer :: istart, iend
    call les_check(les_gpu_comprhs(les_h, real(dtabm, c_double)))
  end subroutine comprhs

  subroutine press(istart, iend, procs, mynode, comm1d)
    integer :: istart, iend, procs, mynode, comm1d
    call les_check(les_gpu_press(les_h))
  end subroutine press

  subroutine comp2(istart, iend)
    use storage, only: dtab1
    integer :: istart, iend
    call les_check(les_gpu_comp2(les_h, real(dtab1, c_double)))
  end subroutine comp2

end module les_gpu
