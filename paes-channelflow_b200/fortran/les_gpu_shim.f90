! les_gpu_shim.f90 -- Fortran binding of libles_gpu.so (include/les_gpu.h, include/les_mlp.h).
!
! Replaces comp1.o comp2.o compadv1.o compsgs1.o compsgs3.o complen.o
! derivs1.o derivs2.o comprhs.o press.o tridv.o lowerbc.o upperbc.o and
! compmn.o in LESOBJS (Makefile:11-14) so that les.F90 keeps driving the
! stage loop (les.F90:254-285) with the same subroutine names and arguments
! while the domain lives on one GPU.  filter_fftw.o and FFTW 2.x stay in the
! link: the host still uses fft_init, deal, xderiv/yderiv (initvel,
! init.f90:95-96) and fft_finalize once, outside the stage loop
! (les.F90:149, 173, 185-190, 356).  The storage module stays the host copy
! of the state for restart files; three calls are added to les.F90:
!   les_gpu_attach  after the deal loop (les.F90:190): init + upload
!   les_gpu_fetch   before the restart write (les.F90:331): download
!   les_gpu_detach  before fft_finalize (les.F90:356)
! compmn (les.F90:288) is provided here and fills meanbuf, utau, utau_s,
! dudt and dvdt from the device.  Serial build only (no -DMPI: the GPU holds
! the whole domain).
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
     integer(c_int) function les_gpu_sync(h, timeout_s) bind(C, name="les_gpu_sync")
       import :: c_ptr, c_int, c_double
       type(c_ptr), value :: h
       real(c_double), value :: timeout_s
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

  ! bytes of the host's default real (4 as shipped, 8 with -fdefault-real-8)
  integer, save :: rbytes = 8

contains

  ! les.F90:190, after the restart read or initvel and the deal loop:
  ! les_gpu_init replaces setcombuf, allocate_arrays' device part, initwave
  ! and fft_init for the stage loop; the state is uploaded once.
  subroutine les_gpu_attach()
    use storage
    use parameters
    type(les_config), target :: gcfg
    gcfg%nnx = nnx; gcfg%nny = nny; gcfg%nnz = nnz
    gcfg%imodel = imodel; gcfg%isurface = isurface
    gcfg%tke_production = 0; gcfg%precision = 8; gcfg%device = 0
    gcfg%xl = xl; gcfg%yl = yl; gcfg%zl = zl; gcfg%z0 = z0; gcfg%dt = dt
    gcfg%cb = cb; gcfg%skc = skc; gcfg%nu = 0d0
    gcfg%ugal = ugal; gcfg%vgal = vgal; gcfg%ufree = 0d0
    gcfg%emin = emin; gcfg%forcing = 0.016d0
    rbytes = storage_size(u) / 8
    call les_check(les_gpu_init(gcfg, les_h))
    call les_check(les_gpu_upload(les_h, c_loc(u(1,1,1)), c_loc(v(1,1,1)), c_loc(w(1,1,1)), &
         c_loc(e(1,1,1)), c_null_ptr, int(rbytes, c_int)))
  end subroutine les_gpu_attach

  ! les.F90:331, before write_params / sav_field: the device state into the
  ! storage module (levels 1..nnz; p into p(1:nnx,:,:))
  subroutine les_gpu_fetch()
    use storage
    real, allocatable, target :: pr(:,:,:)
    allocate(pr(nnx, nny, nnz))
    call les_check(les_gpu_download(les_h, c_loc(u(1,1,1)), c_loc(v(1,1,1)), c_loc(w(1,1,1)), &
         c_loc(e(1,1,1)), c_loc(pr(1,1,1)), int(rbytes, c_int)))
    p(1:nnx, 1:nny, 1:nnz) = pr
    deallocate(pr)
  end subroutine les_gpu_fetch

  ! les.F90:356, before fft_finalize / deallocate_arrays
  subroutine les_gpu_detach()
    call les_check(les_gpu_sync(les_h, -1d0))
    call les_gpu_finalize(les_h)
    les_h = c_null_ptr
  end subroutine les_gpu_detach

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

  ! compmn (compmn.F90:1-64) from the device: meanbuf(19, nnz) in the
  ! allocate.f90:89-111 row order, and the wall-model scalars that
  ! output_profiles prints (les.F90:389-407)
  subroutine compmn(istart, iend)
    use storage
    integer :: istart, iend
    real(c_double), allocatable, target :: mb(:,:)
    real(c_double), target :: sc(5)
    allocate(mb(19, nnz))
    call les_check(les_gpu_stats(les_h, c_loc(mb(1,1)), c_loc(sc(1))))
    meanbuf(1:19, istart:iend) = mb(1:19, istart:iend)
    utau = sc(1); utau_s = sc(2); dudt = sc(3); dvdt = sc(4)
    deallocate(mb)
  end subroutine compmn

end module les_gpu
