! espec_gpu.f90 -- iso_c_binding shim between eSPec's Fortran driver and the
! GPU drop-ins of libespecgpu.so (declared in espec_gpu.h).
!
! The C entry points pspofft_, psodfft_, plnz_ and psod_ follow the gfortran
! calling convention (every argument by reference, one size_t length per
! CHARACTER*(*) argument appended in order), so a gfortran build can call
! them directly in place of the reference routines.  This module makes the
! call independent of that convention: each ESPEC_* subroutine below takes
! exactly the argument list of the reference routine it replaces (cited on
! each), converts the LOGICALs to C ints (0/1) and passes the CHARACTER
! lengths explicitly through a bind(C) interface.
!
! Use in espec.f: add "USE ESPEC_GPU" and replace
!   CALL PSPOFFT(...)  (espec.f:1474)   by  CALL ESPEC_PSPOFFT(...)
!   CALL PSODFFT(...)  (espec.f:1373)   by  CALL ESPEC_PSODFFT(...)
!   CALL PLNZ(...)     (espec.f:1499)   by  CALL ESPEC_PLNZ(...)
!   CALL PSOD(...)     (espec.f:1362)   by  CALL ESPEC_PSOD(...)
! and link with -L<dir> -lespecgpu -lcudart (INTEGRATION.md).  INFO keeps
! the reference's meaning (0 ok, 1 drift above TOL) and is 2 when the GPU
! path refused the case or failed (the message is on standard error).
module espec_gpu
  use iso_c_binding, only: c_int, c_double, c_char, c_size_t
  implicit none
  private
  public :: espec_pspofft, espec_psodfft, espec_plnz, espec_psod

  interface
    subroutine c_pspofft(absorb, dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, &
                         ti, tf, tol, np, shm, sh, sm, u1, v1, xi, xf, tc, vpot, vabc, lnzvc, &
                         wrk1, wrk2, var, dim_len, prtcrl_len, tpabsor_len) &
        bind(C, name="pspofft_")
      import :: c_int, c_double, c_char, c_size_t
      integer(c_int), intent(in) :: absorb
      character(kind=c_char), intent(in) :: dim(*), prtcrl(*), tpabsor(*)
      integer(c_int), intent(inout) :: info
      integer(c_int), intent(in) :: lc, mp, mpi, mpr, mxdct, n, np(*)
      real(c_double), intent(in) :: dt, ti, tf, tol, shm(*), sh(*), sm(*), xi(*), xf(*)
      real(c_double), intent(in) :: vpot(*), vabc(*), var(*)
      real(c_double), intent(inout) :: u1(*), v1(*), tc(*), lnzvc(*), wrk1(*), wrk2(*)
      integer(c_size_t), value :: dim_len, prtcrl_len, tpabsor_len
    end subroutine c_pspofft

    subroutine c_psodfft(absorb, dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, &
                         ti, tf, tol, np, shm, sh, sm, u1, u2, v1, v2, xi, xf, tc, vpot, vabc, &
                         wrkr, wrki, var, lnzvc, dim_len, prtcrl_len, tpabsor_len) &
        bind(C, name="psodfft_")
      import :: c_int, c_double, c_char, c_size_t
      integer(c_int), intent(in) :: absorb
      character(kind=c_char), intent(in) :: dim(*), prtcrl(*), tpabsor(*)
      integer(c_int), intent(inout) :: info
      integer(c_int), intent(in) :: lc, mp, mpi, mpr, mxdct, n, np(*)
      real(c_double), intent(in) :: dt, ti, tf, tol, shm(*), sh(*), sm(*), xi(*), xf(*)
      real(c_double), intent(in) :: vpot(*), vabc(*), var(*)
      real(c_double), intent(inout) :: u1(*), u2(*), v1(*), v2(*), tc(*), wrkr(*), wrki(*)
      real(c_double), intent(inout) :: lnzvc(*)
      integer(c_size_t), value :: dim_len, prtcrl_len, tpabsor_len
    end subroutine c_psodfft

    subroutine c_plnz(absorb, change, dim, prtcrl, tpabsor, info, lc, lmtreort, mp, mpi, mpr, &
                      mxdct, n, abstol, dt, ti, tf, tol, np, iwork, shm, vpot, vabc, u, v, xi, &
                      xf, wu, wv, wp, work, var, lnzvc, dim_len, prtcrl_len, tpabsor_len) &
        bind(C, name="plnz_")
      import :: c_int, c_double, c_char, c_size_t
      integer(c_int), intent(in) :: absorb, change
      character(kind=c_char), intent(in) :: dim(*), prtcrl(*), tpabsor(*)
      integer(c_int), intent(inout) :: info, mp, iwork(*)
      integer(c_int), intent(in) :: lc, lmtreort, mpi, mpr, mxdct, n, np(*)
      real(c_double), intent(in) :: abstol, dt, ti, tf, tol, shm(*), vpot(*), vabc(*)
      real(c_double), intent(in) :: xi(*), xf(*), var(*)
      real(c_double), intent(inout) :: u(*), v(*), wu(*), wv(*), wp(*), work(*), lnzvc(*)
      integer(c_size_t), value :: dim_len, prtcrl_len, tpabsor_len
    end subroutine c_plnz

    subroutine c_psod(absorb, dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, ti, &
                      tf, tol, np, shm, u1, u2, v1, v2, xi, xf, vpot, vabc, work, var, lnzvc, &
                      dim_len, prtcrl_len, tpabsor_len) &
        bind(C, name="psod_")
      import :: c_int, c_double, c_char, c_size_t
      integer(c_int), intent(in) :: absorb
      character(kind=c_char), intent(in) :: dim(*), prtcrl(*), tpabsor(*)
      integer(c_int), intent(inout) :: info
      integer(c_int), intent(in) :: lc, mp, mpi, mpr, mxdct, n, np(*)
      real(c_double), intent(in) :: dt, ti, tf, tol, shm(*), xi(*), xf(*), vpot(*), vabc(*)
      real(c_double), intent(in) :: var(*)
      real(c_double), intent(inout) :: u1(*), u2(*), v1(*), v2(*), work(*), lnzvc(*)
      integer(c_size_t), value :: dim_len, prtcrl_len, tpabsor_len
    end subroutine c_psod
  end interface

contains

  integer(c_int) function cbool(l)
    logical, intent(in) :: l
    cbool = 0
    if (l) cbool = 1
  end function cbool

  ! PSPOFFT (pspofft.f:1-15)
  subroutine espec_pspofft(absorb, dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, &
                           dt, ti, tf, tol, np, shm, sh, sm, u1, v1, xi, xf, tc, vpot, vabc, &
                           lnzvc, wrk1, wrk2, var)
    logical, intent(in) :: absorb
    character(len=*), intent(in) :: dim, prtcrl, tpabsor
    integer, intent(inout) :: info
    integer, intent(in) :: lc, mp, mpi, mpr, mxdct, n, np(*)
    real(8), intent(in) :: dt, ti, tf, tol, shm(*), sh(*), sm(*), xi(*), xf(*), vpot(*)
    real(8), intent(in) :: vabc(*), var(*)
    real(8), intent(inout) :: u1(*), v1(*), tc(*), wrk1(*), wrk2(*), lnzvc(mxdct, *)
    call c_pspofft(cbool(absorb), dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, &
                   ti, tf, tol, np, shm, sh, sm, u1, v1, xi, xf, tc, vpot, vabc, lnzvc, wrk1, &
                   wrk2, var, len(dim, c_size_t), len(prtcrl, c_size_t), len(tpabsor, c_size_t))
  end subroutine espec_pspofft

  ! PSODFFT (psodfft.f:1-14)
  subroutine espec_psodfft(absorb, dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, &
                           dt, ti, tf, tol, np, shm, sh, sm, u1, u2, v1, v2, xi, xf, tc, vpot, &
                           vabc, wrkr, wrki, var, lnzvc)
    logical, intent(in) :: absorb
    character(len=*), intent(in) :: dim, prtcrl, tpabsor
    integer, intent(inout) :: info
    integer, intent(in) :: lc, mp, mpi, mpr, mxdct, n, np(*)
    real(8), intent(in) :: dt, ti, tf, tol, shm(*), sh(*), sm(*), xi(*), xf(*), vpot(*)
    real(8), intent(in) :: vabc(*), var(*)
    real(8), intent(inout) :: u1(*), u2(*), v1(*), v2(*), tc(*), wrkr(*), wrki(*)
    real(8), intent(inout) :: lnzvc(mxdct, *)
    call c_psodfft(cbool(absorb), dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, &
                   ti, tf, tol, np, shm, sh, sm, u1, u2, v1, v2, xi, xf, tc, vpot, vabc, wrkr, &
                   wrki, var, lnzvc, len(dim, c_size_t), len(prtcrl, c_size_t), &
                   len(tpabsor, c_size_t))
  end subroutine espec_psodfft

  ! PLNZ (plnz.f:1-15); MP may be lowered to LMTREORT as LNZ does
  subroutine espec_plnz(absorb, change, dim, prtcrl, tpabsor, info, lc, lmtreort, mp, mpi, &
                        mpr, mxdct, n, abstol, dt, ti, tf, tol, np, iwork, shm, vpot, vabc, u, &
                        v, xi, xf, wu, wv, wp, work, var, lnzvc)
    logical, intent(in) :: absorb, change
    character(len=*), intent(in) :: dim, prtcrl, tpabsor
    integer, intent(inout) :: info, mp, iwork(*)
    integer, intent(in) :: lc, lmtreort, mpi, mpr, mxdct, n, np(*)
    real(8), intent(in) :: abstol, dt, ti, tf, tol, shm(*), vpot(*), vabc(*), xi(*), xf(*)
    real(8), intent(in) :: var(*)
    real(8), intent(inout) :: u(*), v(*), wu(*), wv(*), wp(*), work(*), lnzvc(mxdct, *)
    call c_plnz(cbool(absorb), cbool(change), dim, prtcrl, tpabsor, info, lc, lmtreort, mp, &
                mpi, mpr, mxdct, n, abstol, dt, ti, tf, tol, np, iwork, shm, vpot, vabc, u, v, &
                xi, xf, wu, wv, wp, work, var, lnzvc, len(dim, c_size_t), &
                len(prtcrl, c_size_t), len(tpabsor, c_size_t))
  end subroutine espec_plnz

  ! PSOD (psod.f:1-13)
  subroutine espec_psod(absorb, dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, &
                        ti, tf, tol, np, shm, u1, u2, v1, v2, xi, xf, vpot, vabc, work, var, &
                        lnzvc)
    logical, intent(in) :: absorb
    character(len=*), intent(in) :: dim, prtcrl, tpabsor
    integer, intent(inout) :: info
    integer, intent(in) :: lc, mp, mpi, mpr, mxdct, n, np(*)
    real(8), intent(in) :: dt, ti, tf, tol, shm(*), xi(*), xf(*), vpot(*), vabc(*), var(*)
    real(8), intent(inout) :: u1(*), u2(*), v1(*), v2(*), work(*), lnzvc(mxdct, *)
    call c_psod(cbool(absorb), dim, prtcrl, tpabsor, info, lc, mp, mpi, mpr, mxdct, n, dt, ti, &
                tf, tol, np, shm, u1, u2, v1, v2, xi, xf, vpot, vabc, work, var, lnzvc, &
                len(dim, c_size_t), len(prtcrl, c_size_t), len(tpabsor, c_size_t))
  end subroutine espec_psod

end module espec_gpu
