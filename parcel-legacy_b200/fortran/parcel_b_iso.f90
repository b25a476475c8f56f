! parcel_b_iso.f90 -- ISO_C_BINDING drop-in for PARCEL's Fortran solver wrappers.
!
! Provides module PARCEL_wrapper with the subroutines parcel_dcg, parcel_dbicgstab,
! parcel_dgmres and parcel_dcagmres under the argument lists of the reference's CPU build
! (src/wrapper.f90:1813-2900), their DIA forms parcel_d*_dia (src/wrapper.f90:1905-3134),
! the double-double parcel_ddcg, parcel_ddbicgstab, parcel_ddgmres and their DIA forms
! (src/ddwrapper.f90:4-565), plus PARCEL_Init / PARCEL_Free
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
     subroutine c_parcel_ddcg(icomm, vecx, vecx_lo, vecb, vecb_lo, n, gn, nnz, istart, crsA, &
          crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, &
          reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, &
          PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) bind(c, name="parcel_ddcg_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
            PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int32_t) :: crsRow_ptr(*), crsCol(*)
       real(c_double) :: vecx(*), vecx_lo(*), vecb(*), vecb_lo(*), crsA(*), crsA_lo(*), &
            reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddcg
     subroutine c_parcel_ddbicgstab(icomm, vecx, vecx_lo, vecb, vecb_lo, n, gn, nnz, istart, &
          crsA, crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, niter, &
          rtolmax, reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, &
          PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) bind(c, &
          name="parcel_ddbicgstab_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
            PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int32_t) :: crsRow_ptr(*), crsCol(*)
       real(c_double) :: vecx(*), vecx_lo(*), vecb(*), vecb_lo(*), crsA(*), crsA_lo(*), &
            reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddbicgstab
     subroutine c_parcel_ddgmres(icomm, vecx, vecx_lo, vecb, vecb_lo, n, gn, nnz, istart, crsA, &
          crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, &
          reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, restart, &
          gmres_gsflag, PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) &
          bind(c, name="parcel_ddgmres_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, restart, gmres_gsflag, &
            PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int32_t) :: crsRow_ptr(*), crsCol(*)
       real(c_double) :: vecx(*), vecx_lo(*), vecb(*), vecb_lo(*), crsA(*), crsA_lo(*), &
            reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddgmres
     subroutine c_parcel_dcg_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
          ILU_method, addL, iflagAS, niter, rtolmax, reshistory, iovlflag, precon_thblock, &
          Neuman_itr, independ_nvec, nBlock, iret) bind(c, name="parcel_dcg_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dcg_dia
     subroutine c_parcel_dbicgstab_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, &
          ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, Neuman_itr, independ_nvec, nBlock, iret) bind(c, &
          name="parcel_dbicgstab_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dbicgstab_dia
     subroutine c_parcel_dgmres_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, &
          ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, Neuman_itr, independ_nvec, nBlock, restart, gmres_gsflag, iret) &
          bind(c, name="parcel_dgmres_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, restart, gmres_gsflag, iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dgmres_dia
     subroutine c_parcel_dcagmres_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, &
          ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, Neuman_itr, independ_nvec, nBlock, sstep, tstep, basis, qrflag, iret) &
          bind(c, name="parcel_dcagmres_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, sstep, tstep, basis, qrflag, &
            iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dcagmres_dia
     subroutine c_parcel_ddcg_dia(icomm, vecx, vecx_lo, vecb, vecb_lo, n, gn, istart, diaA, &
          diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, reshistory, &
          iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
          PRECISION_x, PRECISION_PRECONDITION, iret) bind(c, name="parcel_ddcg_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
            PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecx_lo(*), vecb(*), vecb_lo(*), diaA(*), diaA_lo(*), &
            reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddcg_dia
     subroutine c_parcel_ddbicgstab_dia(icomm, vecx, vecx_lo, vecb, vecb_lo, n, gn, istart, &
          diaA, diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, &
          reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, &
          PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) bind(c, &
          name="parcel_ddbicgstab_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
            PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecx_lo(*), vecb(*), vecb_lo(*), diaA(*), diaA_lo(*), &
            reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddbicgstab_dia
     subroutine c_parcel_ddgmres_dia(icomm, vecx, vecx_lo, vecb, vecb_lo, n, gn, istart, diaA, &
          diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, niter, rtolmax, reshistory, &
          iovlflag, precon_thblock, independ_nvec, nBlock, restart, gmres_gsflag, PRECISION_A, &
          PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) bind(c, &
          name="parcel_ddgmres_dia_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, niter, iovlflag, &
            precon_thblock, independ_nvec, nBlock, restart, gmres_gsflag, PRECISION_A, &
            PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int32_t) :: n, gn, istart, nnd
       integer(c_int32_t) :: offset(*)
       real(c_double) :: vecx(*), vecx_lo(*), vecb(*), vecb_lo(*), diaA(*), diaA_lo(*), &
            reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddgmres_dia
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

  ! parcel_ddbicgstab (src/ddwrapper.f90:4-92)
  subroutine parcel_ddbicgstab(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, &
       crsA_hi, crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, &
       rtolmax, reshistory, iovlflag, precon_thblock, independ_nvec, nBlock, PRECISION_A, &
       PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
         PRECISION_PRECONDITION, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    integer(c_int32_t) :: crsRow_ptr(*), crsCol(*)
    real(c_double) :: vecx_hi(*), vecx_lo(*), vecb_hi(*), vecb_lo(*), crsA_hi(*), &
         crsA_lo(*), reshistory(*)
    real(c_double) :: rtolmax
    integer(c_int) :: neuman
    neuman = 1
    call c_parcel_ddbicgstab(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, &
         crsA_hi, crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, &
         rtolmax, reshistory, iovlflag, precon_thblock, neuman, independ_nvec, nBlock, &
         PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddbicgstab

  ! parcel_ddcg (src/ddwrapper.f90:184-279)
  subroutine parcel_ddcg(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, crsA_hi, &
       crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, &
       reshistory, iovlflag, precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
       PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
         PRECISION_PRECONDITION, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    integer(c_int32_t) :: crsRow_ptr(*), crsCol(*)
    real(c_double) :: vecx_hi(*), vecx_lo(*), vecb_hi(*), vecb_lo(*), crsA_hi(*), &
         crsA_lo(*), reshistory(*)
    real(c_double) :: rtolmax
    integer(c_int) :: neuman
    neuman = 1
    call c_parcel_ddcg(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, crsA_hi, &
         crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, &
         reshistory, iovlflag, precon_thblock, neuman, independ_nvec, nBlock, PRECISION_A, &
         PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddcg

  ! parcel_ddgmres (src/ddwrapper.f90:376-471)
  subroutine parcel_ddgmres(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, &
       crsA_hi, crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, &
       rtolmax, reshistory, iovlflag, precon_thblock, independ_nvec, nBlock, GMRES_m, &
       GMRES_GSflag, PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, PRECISION_A, &
         PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    integer(c_int32_t) :: crsRow_ptr(*), crsCol(*)
    real(c_double) :: vecx_hi(*), vecx_lo(*), vecb_hi(*), vecb_lo(*), crsA_hi(*), &
         crsA_lo(*), reshistory(*)
    real(c_double) :: rtolmax
    integer(c_int) :: neuman
    neuman = 1
    call c_parcel_ddgmres(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, &
         crsA_hi, crsA_lo, crsRow_ptr, crsCol, ipreflag, ILU_method, addL, iflagAS, itrmax, &
         rtolmax, reshistory, iovlflag, precon_thblock, neuman, independ_nvec, nBlock, GMRES_m, &
         GMRES_GSflag, PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddgmres

  ! parcel_dbicgstab_dia (src/wrapper.f90:1905); machineflag is accepted and ignored
  subroutine parcel_dbicgstab_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
       ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
       Neuman_itr, independ_nvec, nBlock, iret, machineflag)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
    real(c_double) :: rtolmax
    integer, optional :: machineflag
    call c_parcel_dbicgstab_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
         ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
         Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dbicgstab_dia

  ! parcel_dcg_dia (src/wrapper.f90:2086); machineflag is accepted and ignored
  subroutine parcel_dcg_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
       ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
       Neuman_itr, independ_nvec, nBlock, iret, machineflag)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
    real(c_double) :: rtolmax
    integer, optional :: machineflag
    call c_parcel_dcg_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
         ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
         Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dcg_dia

  ! parcel_dgmres_dia (src/wrapper.f90:2273); machineflag is accepted and ignored
  subroutine parcel_dgmres_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
       ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
       Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret, machineflag)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
    real(c_double) :: rtolmax
    integer, optional :: machineflag
    call c_parcel_dgmres_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
         ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
         Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret)
  end subroutine parcel_dgmres_dia

  ! parcel_dcagmres_dia (src/wrapper.f90:2909); machineflag is accepted and ignored
  subroutine parcel_dcagmres_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
       ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
       Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, &
       CAGMRES_QRflag, iret, machineflag)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
         CAGMRES_basis, CAGMRES_QRflag, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx(*), vecb(*), diaA(*), reshistory(*)
    real(c_double) :: rtolmax
    integer, optional :: machineflag
    call c_parcel_dcagmres_dia(icomm, vecx, vecb, n, gn, istart, diaA, offset, nnd, ipreflag, &
         ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
         Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, &
         CAGMRES_QRflag, iret)
  end subroutine parcel_dcagmres_dia

  ! parcel_ddbicgstab_dia (src/ddwrapper.f90:94-181)
  subroutine parcel_ddbicgstab_dia(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, istart, &
       diaA_hi, diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, &
       reshistory, iovlflag, precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
       PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
         PRECISION_PRECONDITION, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx_hi(*), vecx_lo(*), vecb_hi(*), vecb_lo(*), diaA_hi(*), &
         diaA_lo(*), reshistory(*)
    real(c_double) :: rtolmax
    integer(c_int) :: neuman
    neuman = 1
    call c_parcel_ddbicgstab_dia(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, istart, &
         diaA_hi, diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, &
         reshistory, iovlflag, precon_thblock, neuman, independ_nvec, nBlock, PRECISION_A, &
         PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddbicgstab_dia

  ! parcel_ddcg_dia (src/ddwrapper.f90:282-374)
  subroutine parcel_ddcg_dia(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, istart, diaA_hi, &
       diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, &
       iovlflag, precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
       PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
         PRECISION_PRECONDITION, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx_hi(*), vecx_lo(*), vecb_hi(*), vecb_lo(*), diaA_hi(*), &
         diaA_lo(*), reshistory(*)
    real(c_double) :: rtolmax
    integer(c_int) :: neuman
    neuman = 1
    call c_parcel_ddcg_dia(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, istart, diaA_hi, &
         diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, &
         iovlflag, precon_thblock, neuman, independ_nvec, nBlock, PRECISION_A, PRECISION_b, &
         PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddcg_dia

  ! parcel_ddgmres_dia (src/ddwrapper.f90:473-565)
  subroutine parcel_ddgmres_dia(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, istart, &
       diaA_hi, diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, &
       reshistory, iovlflag, precon_thblock, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, &
       PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag, &
         precon_thblock, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, PRECISION_A, &
         PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret
    integer(c_int32_t) :: n, gn, istart, nnd
    integer(c_int32_t) :: offset(*)
    real(c_double) :: vecx_hi(*), vecx_lo(*), vecb_hi(*), vecb_lo(*), diaA_hi(*), &
         diaA_lo(*), reshistory(*)
    real(c_double) :: rtolmax
    call c_parcel_ddgmres_dia(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, istart, diaA_hi, &
         diaA_lo, offset, nnd, ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, &
         iovlflag, precon_thblock, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, PRECISION_A, &
         PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddgmres_dia
end module PARCEL_wrapper
