! parcel_b_iso.f90 -- ISO_C_BINDING drop-in for PARCEL's Fortran solver wrappers.
!
! Provides module PARCEL_wrapper with the subroutines parcel_dcg, parcel_dbicgstab,
! parcel_dgmres and parcel_dcagmres under the argument lists of the reference's CPU build
! (src/wrapper.f90:1813-2900), plus PARCEL_Init / PARCEL_Free
! (src/c_krylov_wrapper.f90:6-23).  Each routine forwards to the C ABI of libparcelb.so
! (include/parcel_b.h), which copies the host arrays to the B200, solves there and copies
! x and reshistory back.  A program written against the reference keeps its `use
! PARCEL_wrapper` and its calls, and links libparcelb.so instead of parcel_sparse.a.
!
! The icomm argument is accepted and ignored: one process per GPU, no MPI split of the
! matrix (n must equal gn).  iret follows the reference (0 converged, 1 iteration limit);
! a negative iret reports an error the reference would have stopped on.
module parcel_b_c_interface
  use iso_c_binding
  implicit none
  interface
     subroutine c_parcel_init(myrank) bind(c, name="parcel_init_c_")
       import :: c_int
       integer(c_int) :: myrank
     end subroutine c_parcel_init
     subroutine c_parcel_free() bind(c, name="parcel_free_c_")
     end subroutine c_parcel_free
     subroutine c_parcel_dcg(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, iret) bind(c, name="parcel_dcg_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm
       real(c_double) :: vecx(*), vecb(*), crsa(*), reshistory(*)
       integer(c_int32_t) :: n, gn, nnz, istart, crsrow_ptr(*), crscol(*)
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, iret
       real(c_double) :: rtolmax
     end subroutine c_parcel_dcg
     subroutine c_parcel_dbicgstab(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, iret) bind(c, name="parcel_dbicgstab_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm
       real(c_double) :: vecx(*), vecb(*), crsa(*), reshistory(*)
       integer(c_int32_t) :: n, gn, nnz, istart, crsrow_ptr(*), crscol(*)
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, iret
       real(c_double) :: rtolmax
     end subroutine c_parcel_dbicgstab
     subroutine c_parcel_dgmres(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, restart, gmres_gsflag, iret) &
          bind(c, name="parcel_dgmres_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm
       real(c_double) :: vecx(*), vecb(*), crsa(*), reshistory(*)
       integer(c_int32_t) :: n, gn, nnz, istart, crsrow_ptr(*), crscol(*)
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, restart, gmres_gsflag, iret
       real(c_double) :: rtolmax
     end subroutine c_parcel_dgmres
     subroutine c_parcel_dcagmres(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, sstep, tstep, basis, qrflag, iret) &
          bind(c, name="parcel_dcagmres_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm
       real(c_double) :: vecx(*), vecb(*), crsa(*), reshistory(*)
       integer(c_int32_t) :: n, gn, nnz, istart, crsrow_ptr(*), crscol(*)
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, sstep, tstep, basis, qrflag, iret
       real(c_double) :: rtolmax
     end subroutine c_parcel_dcagmres
  end interface
end module parcel_b_c_interface

module PARCEL_wrapper
  use iso_c_binding
  use parcel_b_c_interface
  implicit none
contains
  subroutine PARCEL_Init(myrank)
    integer :: myrank
    integer(c_int) :: r
    r = myrank
    call c_parcel_init(r)
  end subroutine PARCEL_Init

  subroutine PARCEL_Free()
    call c_parcel_free()
  end subroutine PARCEL_Free

  ! parcel_dcg (src/wrapper.f90:1995): itrmax is in/out (iterations used on return).
  subroutine parcel_dcg(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    call c_parcel_dcg(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dcg

  ! parcel_dbicgstab (src/wrapper.f90:1813)
  subroutine parcel_dbicgstab(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    call c_parcel_dbicgstab(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dbicgstab

  ! parcel_dgmres (src/wrapper.f90:2179)
  subroutine parcel_dgmres(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    call c_parcel_dgmres(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret)
  end subroutine parcel_dgmres

  ! parcel_dcagmres (src/wrapper.f90:2807)
  subroutine parcel_dcagmres(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
       CAGMRES_basis, CAGMRES_QRflag, iret)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer :: CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    call c_parcel_dcagmres(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
         CAGMRES_basis, CAGMRES_QRflag, iret)
  end subroutine parcel_dcagmres
end module PARCEL_wrapper
