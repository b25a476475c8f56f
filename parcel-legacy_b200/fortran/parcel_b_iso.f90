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
! Also provided: modules PARCEL_integer, PARCEL_define and krylov with the reference's
! integer kind, option constants and a C-interoperable KSP_INPUT_PARAM; INIT_PARCEL_INPUT
! and the generic PARCEL_KSP_CRS (src/wrapper.f90:5-222), PARCEL_ddKSP_CRS
! (src/ddwrapper.f90:569-614); and the CUDA build's forms of parcel_dcg, parcel_dbicgstab,
! parcel_dgmres and parcel_dcagmres, whose arrays are device addresses (type(c_ptr),
! src/wrapper.f90:362-1454): the generic names resolve to the host or the device form by
! the type of vecx.
!
! The icomm argument is accepted and ignored: one process per GPU, no MPI split of the
! matrix (n must equal gn).  iret follows the reference (0 converged, 1 iteration limit);
! a negative iret reports an error the reference would have stopped on.
! The reference's integer kind (src/define.f90:133-164, PARCEL_INT int32 by default).
module PARCEL_integer
  use iso_c_binding
  implicit none
  integer, parameter :: intType = c_int32_t
end module PARCEL_integer

! The constants of src/define.f90 (module PARCEL_define) that the hot path's options use;
! the values are the reference's, so existing callers pass the same numbers.
module PARCEL_define
  implicit none
  integer, parameter :: MATRIX_FORMAT_CRS = 1, MATRIX_FORMAT_DIA = 2, MATRIX_FORMAT_DDM = 3
  integer, parameter :: KSP_DOUBLE_PRECISION = 1, KSP_DOUBLE_DOUBLE_PRECISION = 2
  integer, parameter :: KSP_SOLVER_CG = 1, KSP_SOLVER_BiCG = 2, KSP_SOLVER_GMRES = 3, &
       KSP_SOLVER_CAGMRES = 4, KSP_SOLVER_CBCG = 5
  integer, parameter :: KSP_SPMV_OVL_NONE = 0, KSP_SPMV_OVL_CORE = 1, KSP_SPMV_OVL_RANK = 2
  integer, parameter :: KSP_PRECONDITION_NONE = 0, KSP_PRECONDITION_POINTJACOBI = 1, &
       KSP_PRECONDITION_BLOCKJACOBI = 2, KSP_PRECONDITION_ADDITIVESCHWARZ = 3, &
       KSP_PRECONDITION_NEUMANN = 4, KSP_PRECONDITION_NEUMANN_LOCAL = 5
  integer, parameter :: KSP_PRECONDITION_NEUMANN_TRUE_COMM = 1
  integer, parameter :: KSP_PRECONDITION_ILU = 0, KSP_PRECONDITION_ILUD = 1, KSP_PRECONDITION_MLUD = 2
  integer, parameter :: KSP_ADDITIVESCHWARZ_TYPE_BASIC = 1, KSP_ADDITIVESCHWARZ_TYPE_RESTRICT = 2, &
       KSP_ADDITIVESCHWARZ_TYPE_INTERPOLATE = 3, KSP_ADDITIVESCHWARZ_TYPE_NONE = 4
  integer, parameter :: KSP_QRDECOMPOSITION_MGS = 1, KSP_QRDECOMPOSITION_CGS = 2, &
       KSP_QRDECOMPOSITION_TSQR = 3, KSP_QRDECOMPOSITION_CHOLESKYQR = 4, KSP_QRDECOMPOSITION_CHOLESKYQR2 = 5
  integer, parameter :: KSP_GMRES_GS_TYPE_MGS = KSP_QRDECOMPOSITION_MGS, &
       KSP_GMRES_GS_TYPE_CGS = KSP_QRDECOMPOSITION_CGS
  integer, parameter :: KSP_CAGMRES_QR_TYPE_MGS = KSP_QRDECOMPOSITION_MGS, &
       KSP_CAGMRES_QR_TYPE_CGS = KSP_QRDECOMPOSITION_CGS, KSP_CAGMRES_QR_TYPE_TSQR = KSP_QRDECOMPOSITION_TSQR, &
       KSP_CAGMRES_QR_TYPE_CHOLESKYQR = KSP_QRDECOMPOSITION_CHOLESKYQR, &
       KSP_CAGMRES_QR_TYPE_CHOLESKYQR2 = KSP_QRDECOMPOSITION_CHOLESKYQR2
  integer, parameter :: KSP_MPK_MONOMIAL_BASIS = 0, KSP_MPK_NEWTON_BASIS = 1
  integer, parameter :: PARCEL_RETURNCODE_NORMAL = 0, PARCEL_RETURNCODE_MAXITERATION = 1
  integer, parameter :: PARCEL_CPU_FLAG_ON = 1, PARCEL_GPU_FLAG_ON = 2
  integer, parameter :: PARCEL_MACHINE_FLAG_DEFAULT = PARCEL_GPU_FLAG_ON
end module PARCEL_define

! KSP_INPUT_PARAM (src/type.f90:907-946) as a C-interoperable type: the reference's fields
! in the reference's order, then the extensions, member for member the C struct
! parcel_b_input of include/parcel_b.h.  A program that says `use krylov` and fills a
! type(KSP_INPUT_PARAM) passes it to PARCEL_KSP_CRS unchanged.
module krylov
  use iso_c_binding
  use PARCEL_define
  implicit none
  type, bind(c) :: KSP_INPUT_PARAM
     integer(c_int) :: ipreflag
     integer(c_int) :: ILU_method
     integer(c_int) :: addL
     integer(c_int) :: iflagAS
     integer(c_int) :: solver
     integer(c_int) :: iovlflag
     integer(c_int) :: GMRES_m
     integer(c_int) :: GMRES_GSflag
     integer(c_int) :: CAGMRES_sstep
     integer(c_int) :: CAGMRES_tstep
     integer(c_int) :: CAGMRES_basis
     integer(c_int) :: CAGMRES_QRflag
     integer(c_int) :: CBCG_kstep
     integer(c_int) :: CBCG_Eigenflag
     integer(c_int) :: power_method_itrmax
     integer(c_int) :: CAARNOLDI_sstep
     integer(c_int) :: CAARNOLDI_tstep
     integer(c_int) :: CAARNOLDI_basis
     integer(c_int) :: CAARNOLDI_QRflag
     integer(c_int) :: machineflag
     integer(c_int) :: dataflag
     integer(c_int) :: calcflag
     integer(c_int) :: Neuman_itr
     integer(c_int) :: Neuman_local
     integer(c_int) :: itrmax
     real(c_double) :: rtolmax
     real(c_double) :: abstolmax
     integer(c_int) :: independ_nvec
     integer(c_int) :: precon_thblock
     integer(c_int) :: nBlock
     integer(c_int) :: PRECISION_A
     integer(c_int) :: PRECISION_b
     integer(c_int) :: PRECISION_x
     integer(c_int) :: PRECISION_PRECONDITION
     integer(c_int) :: inner_precision
     integer(c_int) :: residual_dd
     real(c_double) :: inner_rtol
     integer(c_int) :: max_refine
     integer(c_int) :: reserved(7)
  end type KSP_INPUT_PARAM
end module krylov

module parcel_b_c_interface
  use iso_c_binding
  use krylov, only: KSP_INPUT_PARAM
  implicit none
  ! parcel_b_crs of include/parcel_b.h
  type, bind(c) :: parcel_b_crs_t
     integer(c_int32_t) :: n, gn
     integer(c_int64_t) :: nnz
     integer(c_int32_t) :: istart
     type(c_ptr) :: rowptr, col, val
  end type parcel_b_crs_t
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
     ! ---- generic entries (include/parcel_b.h): the CRS matrix struct holds raw
     ! pointers, host or device; arrays are passed as c_loc of TARGET arrays or as the
     ! device addresses themselves
     subroutine c_parcel_b_input_init(prm) bind(c, name="parcel_b_input_init")
       import :: KSP_INPUT_PARAM
       type(KSP_INPUT_PARAM) :: prm
     end subroutine c_parcel_b_input_init
     integer(c_int) function c_parcel_b_solve(prm, a, b, x, reshistory, niter, iret) &
          bind(c, name="parcel_b_solve")
       import :: c_int, c_ptr, KSP_INPUT_PARAM, parcel_b_crs_t
       type(KSP_INPUT_PARAM) :: prm
       type(parcel_b_crs_t) :: a
       type(c_ptr), value :: b, x, reshistory
       integer(c_int) :: niter, iret
     end function c_parcel_b_solve
     integer(c_int) function c_parcel_b_ddcg(prm, a, val_lo, precision_a, precision_b, precision_x, &
          precision_precondition, b_hi, b_lo, x_hi, x_lo, reshistory, niter, iret) bind(c, name="parcel_b_ddcg")
       import :: c_int, c_ptr, KSP_INPUT_PARAM, parcel_b_crs_t
       type(KSP_INPUT_PARAM) :: prm
       type(parcel_b_crs_t) :: a
       type(c_ptr), value :: val_lo, b_hi, b_lo, x_hi, x_lo, reshistory
       integer(c_int), value :: precision_a, precision_b, precision_x, precision_precondition
       integer(c_int) :: niter, iret
     end function c_parcel_b_ddcg
     integer(c_int) function c_parcel_b_ddbicgstab(prm, a, val_lo, precision_a, precision_b, precision_x, &
          precision_precondition, b_hi, b_lo, x_hi, x_lo, reshistory, niter, iret) &
          bind(c, name="parcel_b_ddbicgstab")
       import :: c_int, c_ptr, KSP_INPUT_PARAM, parcel_b_crs_t
       type(KSP_INPUT_PARAM) :: prm
       type(parcel_b_crs_t) :: a
       type(c_ptr), value :: val_lo, b_hi, b_lo, x_hi, x_lo, reshistory
       integer(c_int), value :: precision_a, precision_b, precision_x, precision_precondition
       integer(c_int) :: niter, iret
     end function c_parcel_b_ddbicgstab
     integer(c_int) function c_parcel_b_ddgmres(prm, a, val_lo, precision_a, precision_b, precision_x, &
          precision_precondition, b_hi, b_lo, x_hi, x_lo, reshistory, niter, iret) &
          bind(c, name="parcel_b_ddgmres")
       import :: c_int, c_ptr, KSP_INPUT_PARAM, parcel_b_crs_t
       type(KSP_INPUT_PARAM) :: prm
       type(parcel_b_crs_t) :: a
       type(c_ptr), value :: val_lo, b_hi, b_lo, x_hi, x_lo, reshistory
       integer(c_int), value :: precision_a, precision_b, precision_x, precision_precondition
       integer(c_int) :: niter, iret
     end function c_parcel_b_ddgmres
     ! ---- CUDA-build shims: vecx, vecb and the CRS arrays are device addresses
     ! (type(c_ptr), passed by reference as the reference's GPU build passes them)
     subroutine c_parcel_dcg_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, iret) bind(c, name="parcel_dcg_gpu_c_")
       import :: c_int, c_int32_t, c_double, c_ptr
       integer(c_int) :: icomm
       type(c_ptr) :: vecx, vecb, crsa, crsrow_ptr, crscol
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, iret
       real(c_double) :: rtolmax, reshistory(*)
     end subroutine c_parcel_dcg_gpu
     subroutine c_parcel_dbicgstab_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, iret) bind(c, name="parcel_dbicgstab_gpu_c_")
       import :: c_int, c_int32_t, c_double, c_ptr
       integer(c_int) :: icomm
       type(c_ptr) :: vecx, vecb, crsa, crsrow_ptr, crscol
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, iret
       real(c_double) :: rtolmax, reshistory(*)
     end subroutine c_parcel_dbicgstab_gpu
     subroutine c_parcel_dgmres_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, restart, gmres_gsflag, iret) &
          bind(c, name="parcel_dgmres_gpu_c_")
       import :: c_int, c_int32_t, c_double, c_ptr
       integer(c_int) :: icomm
       type(c_ptr) :: vecx, vecb, crsa, crsrow_ptr, crscol
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, restart, gmres_gsflag, iret
       real(c_double) :: rtolmax, reshistory(*)
     end subroutine c_parcel_dgmres_gpu
     subroutine c_parcel_dcagmres_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, &
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, &
          precon_thblock, neuman_itr, independ_nvec, nblock, cagmres_sstep, cagmres_tstep, cagmres_basis, &
          cagmres_qrflag, iret) bind(c, name="parcel_dcagmres_gpu_c_")
       import :: c_int, c_int32_t, c_double, c_ptr
       integer(c_int) :: icomm
       type(c_ptr) :: vecx, vecb, crsa, crsrow_ptr, crscol
       integer(c_int32_t) :: n, gn, nnz, istart
       integer(c_int) :: ipreflag, ilu_method, addl, iflagas, niter, iovlflag, precon_thblock
       integer(c_int) :: neuman_itr, independ_nvec, nblock, cagmres_sstep, cagmres_tstep, cagmres_basis
       integer(c_int) :: cagmres_qrflag, iret
       real(c_double) :: rtolmax, reshistory(*)
     end subroutine c_parcel_dcagmres_gpu
  end interface
end module parcel_b_c_interface

module PARCEL_wrapper
  use iso_c_binding
  use PARCEL_define
  use krylov
  use parcel_b_c_interface
  implicit none
  private :: parcel_ksp_crs_host, parcel_ksp_crs_dev, parcel_dcg_host, parcel_dcg_dev, &
       parcel_dbicgstab_host, parcel_dbicgstab_dev, parcel_dgmres_host, parcel_dgmres_dev, &
       parcel_dcagmres_host, parcel_dcagmres_dev
  ! generic names: the host (CPU-build) or device (CUDA-build) form by the type of vecx
  interface PARCEL_KSP_CRS
     module procedure parcel_ksp_crs_host, parcel_ksp_crs_dev
  end interface PARCEL_KSP_CRS
  interface parcel_dcg
     module procedure parcel_dcg_host, parcel_dcg_dev
  end interface parcel_dcg
  interface parcel_dbicgstab
     module procedure parcel_dbicgstab_host, parcel_dbicgstab_dev
  end interface parcel_dbicgstab
  interface parcel_dgmres
     module procedure parcel_dgmres_host, parcel_dgmres_dev
  end interface parcel_dgmres
  interface parcel_dcagmres
     module procedure parcel_dcagmres_host, parcel_dcagmres_dev
  end interface parcel_dcagmres
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
  subroutine parcel_dcg_host(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    integer, optional :: machineflag   ! accepted and ignored, as in the reference
    call c_parcel_dcg(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dcg_host

  ! parcel_dbicgstab (src/wrapper.f90:1813)
  subroutine parcel_dbicgstab_host(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    integer, optional :: machineflag   ! accepted and ignored, as in the reference
    call c_parcel_dbicgstab(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dbicgstab_host

  ! parcel_dgmres (src/wrapper.f90:2179)
  subroutine parcel_dgmres_host(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    integer, optional :: machineflag   ! accepted and ignored, as in the reference
    call c_parcel_dgmres(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret)
  end subroutine parcel_dgmres_host

  ! parcel_dcagmres (src/wrapper.f90:2807)
  subroutine parcel_dcagmres_host(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
       CAGMRES_basis, CAGMRES_QRflag, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer :: CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double) :: vecx(n), vecb(n), crsA(nnz), rtolmax, reshistory(itrmax)
    integer(c_int32_t) :: crsRow_ptr(n+1), crsCol(nnz)
    integer, optional :: machineflag   ! accepted and ignored, as in the reference
    call c_parcel_dcagmres(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
         CAGMRES_basis, CAGMRES_QRflag, iret)
  end subroutine parcel_dcagmres_host

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

  ! INIT_PARCEL_INPUT (src/wrapper.f90:5-45): every field -1 (the extensions get their
  ! defaults), through parcel_b_input_init.
  subroutine INIT_PARCEL_INPUT(PARCEL_INPUT)
    type(KSP_INPUT_PARAM) :: PARCEL_INPUT
    call c_parcel_b_input_init(PARCEL_INPUT)
  end subroutine INIT_PARCEL_INPUT

  ! PARCEL_KSP_CRS, CPU-build form (src/wrapper.f90:147-221): host arrays.  The eigenvalue
  ! outputs of the reference's CA-Arnoldi belong to its eigensolvers, which this library
  ! does not provide: passing them returns iret = -5 (PARCEL_B_E_UNSUPPORTED).
  subroutine parcel_ksp_crs_host(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       PARCEL_INPUT, niter, reshistory, iret, EigenValueReal, EigenValueImag, EigenVector, &
       EigenErrorNorm, MaxEigenID, MinEigenID)
    integer :: icomm
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double), target :: vecx(n), vecb(n), crsA(nnz)
    integer(c_int32_t), target :: crsRow_ptr(n+1), crsCol(nnz)
    type(KSP_INPUT_PARAM) :: PARCEL_INPUT
    integer(c_int) :: niter, iret
    real(c_double), target :: reshistory(PARCEL_INPUT%itrmax)
    real(c_double), optional :: EigenValueReal(*), EigenValueImag(*), EigenVector(*), EigenErrorNorm(*)
    integer, optional :: MaxEigenID, MinEigenID
    type(parcel_b_crs_t) :: a
    integer(c_int) :: rc
    if (present(EigenValueReal) .or. present(MinEigenID)) then
       iret = -5
       return
    end if
    a = parcel_b_crs_t(n, gn, int(nnz, c_int64_t), istart, c_loc(crsRow_ptr), c_loc(crsCol), c_loc(crsA))
    rc = c_parcel_b_solve(PARCEL_INPUT, a, c_loc(vecb), c_loc(vecx), c_loc(reshistory), niter, iret)
    if (rc < 0) iret = rc
  end subroutine parcel_ksp_crs_host

  ! PARCEL_KSP_CRS, CUDA-build form (src/wrapper.f90:48-145): vecx, vecb and the CRS
  ! arrays are device addresses.
  subroutine parcel_ksp_crs_dev(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       PARCEL_INPUT, niter, reshistory, iret, EigenValueReal, EigenValueImag, EigenVector, &
       EigenErrorNorm, MaxEigenID, MinEigenID)
    integer :: icomm
    integer(c_int32_t) :: n, gn, nnz, istart
    type(c_ptr) :: vecx, vecb, crsA, crsRow_ptr, crsCol
    type(KSP_INPUT_PARAM) :: PARCEL_INPUT
    integer(c_int) :: niter, iret
    real(c_double), target :: reshistory(PARCEL_INPUT%itrmax)
    real(c_double), optional :: EigenValueReal(*), EigenValueImag(*), EigenVector(*), EigenErrorNorm(*)
    integer, optional :: MaxEigenID, MinEigenID
    type(parcel_b_crs_t) :: a
    integer(c_int) :: rc
    if (present(EigenValueReal) .or. present(MinEigenID)) then
       iret = -5
       return
    end if
    a = parcel_b_crs_t(n, gn, int(nnz, c_int64_t), istart, crsRow_ptr, crsCol, crsA)
    rc = c_parcel_b_solve(PARCEL_INPUT, a, vecb, vecx, c_loc(reshistory), niter, iret)
    if (rc < 0) iret = rc
  end subroutine parcel_ksp_crs_dev

  ! PARCEL_ddKSP_CRS (src/ddwrapper.f90:569-614): the double-double CG, BiCGStab or GMRES
  ! selected by PARCEL_INPUT%solver, with PARCEL_INPUT's PRECISION_* flags; host arrays.
  subroutine PARCEL_ddKSP_CRS(icomm, vecx_hi, vecx_lo, vecb_hi, vecb_lo, n, gn, nnz, istart, &
       crsA_hi, crsA_lo, crsRow_ptr, crsCol, PARCEL_INPUT, niter, reshistory, iret)
    integer :: icomm
    integer(c_int32_t) :: n, gn, nnz, istart
    real(c_double), target :: vecx_hi(n), vecx_lo(n), vecb_hi(n), vecb_lo(n), crsA_hi(nnz), crsA_lo(nnz)
    integer(c_int32_t), target :: crsRow_ptr(n+1), crsCol(nnz)
    type(KSP_INPUT_PARAM) :: PARCEL_INPUT
    integer(c_int) :: niter, iret
    real(c_double), target :: reshistory(PARCEL_INPUT%itrmax)
    type(parcel_b_crs_t) :: a
    integer(c_int) :: rc
    a = parcel_b_crs_t(n, gn, int(nnz, c_int64_t), istart, c_loc(crsRow_ptr), c_loc(crsCol), c_loc(crsA_hi))
    select case (PARCEL_INPUT%solver)
    case (KSP_SOLVER_CG)
       rc = c_parcel_b_ddcg(PARCEL_INPUT, a, c_loc(crsA_lo), PARCEL_INPUT%PRECISION_A, PARCEL_INPUT%PRECISION_b, &
            PARCEL_INPUT%PRECISION_x, PARCEL_INPUT%PRECISION_PRECONDITION, c_loc(vecb_hi), c_loc(vecb_lo), &
            c_loc(vecx_hi), c_loc(vecx_lo), c_loc(reshistory), niter, iret)
    case (KSP_SOLVER_BiCG)
       rc = c_parcel_b_ddbicgstab(PARCEL_INPUT, a, c_loc(crsA_lo), PARCEL_INPUT%PRECISION_A, &
            PARCEL_INPUT%PRECISION_b, PARCEL_INPUT%PRECISION_x, PARCEL_INPUT%PRECISION_PRECONDITION, &
            c_loc(vecb_hi), c_loc(vecb_lo), c_loc(vecx_hi), c_loc(vecx_lo), c_loc(reshistory), niter, iret)
    case (KSP_SOLVER_GMRES)
       rc = c_parcel_b_ddgmres(PARCEL_INPUT, a, c_loc(crsA_lo), PARCEL_INPUT%PRECISION_A, &
            PARCEL_INPUT%PRECISION_b, PARCEL_INPUT%PRECISION_x, PARCEL_INPUT%PRECISION_PRECONDITION, &
            c_loc(vecb_hi), c_loc(vecb_lo), c_loc(vecx_hi), c_loc(vecx_lo), c_loc(reshistory), niter, iret)
    case default
       rc = -5
    end select
    if (rc < 0) iret = rc
  end subroutine PARCEL_ddKSP_CRS

  ! parcel_dcg, CUDA-build form (src/wrapper.f90:544): device addresses.
  subroutine parcel_dcg_dev(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    type(c_ptr) :: vecx, vecb, crsA, crsRow_ptr, crsCol
    real(c_double) :: rtolmax, reshistory(itrmax)
    integer, optional :: machineflag
    call c_parcel_dcg_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dcg_dev

  ! parcel_dbicgstab, CUDA-build form (src/wrapper.f90:362)
  subroutine parcel_dbicgstab_dev(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    type(c_ptr) :: vecx, vecb, crsA, crsRow_ptr, crsCol
    real(c_double) :: rtolmax, reshistory(itrmax)
    integer, optional :: machineflag
    call c_parcel_dbicgstab_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dbicgstab_dev

  ! parcel_dgmres, CUDA-build form (src/wrapper.f90:727)
  subroutine parcel_dgmres_dev(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret
    integer(c_int32_t) :: n, gn, nnz, istart
    type(c_ptr) :: vecx, vecb, crsA, crsRow_ptr, crsCol
    real(c_double) :: rtolmax, reshistory(itrmax)
    integer, optional :: machineflag
    call c_parcel_dgmres_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret)
  end subroutine parcel_dgmres_dev

  ! parcel_dcagmres, CUDA-build form (src/wrapper.f90:1355)
  subroutine parcel_dcagmres_dev(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
       ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
       precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
       CAGMRES_basis, CAGMRES_QRflag, iret, machineflag)
    integer :: icomm, ipreflag, ILU_method, addL, iflagAS, itrmax, iovlflag
    integer :: precon_thblock, Neuman_itr, independ_nvec, nBlock, iret
    integer :: CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag
    integer(c_int32_t) :: n, gn, nnz, istart
    type(c_ptr) :: vecx, vecb, crsA, crsRow_ptr, crsCol
    real(c_double) :: rtolmax, reshistory(itrmax)
    integer, optional :: machineflag
    call c_parcel_dcagmres_gpu(icomm, vecx, vecb, n, gn, nnz, istart, crsA, crsRow_ptr, crsCol, &
         ipreflag, ILU_method, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, &
         CAGMRES_basis, CAGMRES_QRflag, iret)
  end subroutine parcel_dcagmres_dev
end module PARCEL_wrapper

! Module ddm_wrapper: the DDM stencil-format solvers under the argument lists of the
! reference's CPU build (src/src_DDM/ddm_kernel.f90:1906-3279, used by
! src/example/main_ddm.f90 through `use ddm_wrapper`).  x and b are the process's padded box
! (nrow = m cells); the block-Jacobi D-ILU runs on precon_thblock slabs along div_direc_th,
! as the CPU build's OpenMP threads cut them.  One process: ndiv_grids all 1 and no
! neighbour ranks (a box split over processes runs through the Python package's
! parcel_b.ddm on torch.distributed); anything else returns iret = -5.
module ddm_wrapper
  use iso_c_binding
  implicit none
  private
  public :: parcel_dcg_ddm, parcel_dbicgstab_ddm, parcel_dgmres_ddm, parcel_dcagmres_ddm, parcel_ddcg_ddm, parcel_ddbicgstab_ddm, parcel_ddgmres_ddm

  interface
     subroutine c_parcel_dcg_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
          num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
          ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
          iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, iret) &
          bind(c, name="parcel_dcg_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dcg_ddm
     subroutine c_parcel_dbicgstab_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
          num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
          ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
          iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, iret) &
          bind(c, name="parcel_dbicgstab_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dbicgstab_ddm
     subroutine c_parcel_dgmres_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
          num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
          ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
          iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, &
          GMRES_GSflag, iret) &
          bind(c, name="parcel_dgmres_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dgmres_ddm
     subroutine c_parcel_dcagmres_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
          num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
          ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
          iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, &
          CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag, iret) &
          bind(c, name="parcel_dcagmres_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, &
            CAGMRES_QRflag, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_dcagmres_ddm
     subroutine c_parcel_ddcg_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
          val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
          num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
          reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, &
          PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) &
          bind(c, name="parcel_ddcg_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
            PRECISION_PRECONDITION, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*), x_lo(*), b_lo(*), &
            val_dia_lo(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddcg_ddm
     subroutine c_parcel_ddbicgstab_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, &
          val_dia, val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, &
          ndiv_grids, num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, &
          rtolmax, reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, &
          PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) &
          bind(c, name="parcel_ddbicgstab_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
            PRECISION_PRECONDITION, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*), x_lo(*), b_lo(*), &
            val_dia_lo(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddbicgstab_ddm
     subroutine c_parcel_ddgmres_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
          val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
          num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
          reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, &
          GMRES_GSflag, PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret) &
          bind(c, name="parcel_ddgmres_ddm_c_")
       import :: c_int, c_int32_t, c_double
       integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
            ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
            independ_nvec, nBlock, GMRES_m, GMRES_GSflag, PRECISION_A, PRECISION_b, &
            PRECISION_x, PRECISION_PRECONDITION, iret
       integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
       integer(c_int32_t) :: nrow
       integer(c_int32_t) :: ioff_dia(*)
       real(c_double) :: x(*), b(*), val_dia(*), reshistory(*), x_lo(*), b_lo(*), &
            val_dia_lo(*)
       real(c_double) :: rtolmax
     end subroutine c_parcel_ddgmres_ddm
  end interface

contains

  ! parcel_dcg_ddm (src/src_DDM/ddm_kernel.f90:2893-2986), CPU build: host arrays, one process
  subroutine parcel_dcg_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, num_neighbor_ranks, &
       neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, ioff_grids, div_direc_th, &
       ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, precon_thblock, &
       Neuman_itr, independ_nvec, nBlock, iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
    real(c_double) :: rtolmax
    call c_parcel_dcg_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, num_neighbor_ranks, &
         neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, ioff_grids, &
         div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dcg_ddm

  ! parcel_dbicgstab_ddm (src/src_DDM/ddm_kernel.f90:2988-3080), CPU build: host arrays, one process
  subroutine parcel_dbicgstab_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
       num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
       ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
       iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
    real(c_double) :: rtolmax
    call c_parcel_dbicgstab_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
         num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
         ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
         iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, iret)
  end subroutine parcel_dbicgstab_ddm

  ! parcel_dgmres_ddm (src/src_DDM/ddm_kernel.f90:3082-3178), CPU build: host arrays, one process
  subroutine parcel_dgmres_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
       num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
       ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
       iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, &
       iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
    real(c_double) :: rtolmax
    call c_parcel_dgmres_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, num_neighbor_ranks, &
         neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, ioff_grids, &
         div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, iovlflag, &
         precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, GMRES_GSflag, iret)
  end subroutine parcel_dgmres_ddm

  ! parcel_dcagmres_ddm (src/src_DDM/ddm_kernel.f90:3180-3279), CPU build: host arrays, one process
  subroutine parcel_dcagmres_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
       num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
       ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
       iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, &
       CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag, iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, CAGMRES_sstep, CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag, &
         iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*)
    real(c_double) :: rtolmax
    call c_parcel_dcagmres_ddm(icomm, x, b, nrow, nnd, ioff_dia, val_dia, &
         num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, num_grids, &
         ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, reshistory, &
         iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, CAGMRES_sstep, &
         CAGMRES_tstep, CAGMRES_basis, CAGMRES_QRflag, iret)
  end subroutine parcel_dcagmres_ddm

  ! parcel_ddcg_ddm (src/src_DDM/ddm_kernel.f90:1906-2023), CPU build: host arrays, one process
  subroutine parcel_ddcg_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
       val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
       num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
       reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, &
       PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
         PRECISION_PRECONDITION, iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*), x_lo(*), b_lo(*), val_dia_lo(*)
    real(c_double) :: rtolmax
    call c_parcel_ddcg_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
         val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
         num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
         reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, &
         PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddcg_ddm

  ! parcel_ddbicgstab_ddm (src/src_DDM/ddm_kernel.f90:2025-2141), CPU build: host arrays, one process
  subroutine parcel_ddbicgstab_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
       val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
       num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
       reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, PRECISION_A, &
       PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, PRECISION_A, PRECISION_b, PRECISION_x, &
         PRECISION_PRECONDITION, iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*), x_lo(*), b_lo(*), val_dia_lo(*)
    real(c_double) :: rtolmax
    call c_parcel_ddbicgstab_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
         val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
         num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
         reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, &
         PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddbicgstab_ddm

  ! parcel_ddgmres_ddm (src/src_DDM/ddm_kernel.f90:2143-2263), CPU build: host arrays, one process
  subroutine parcel_ddgmres_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
       val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
       num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
       reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, &
       GMRES_GSflag, PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
    integer(c_int) :: icomm, nnd, num_neighbor_ranks, margin, ncomp_grids, div_direc_th, &
         ipreflag, addL, iflagAS, itrmax, iovlflag, precon_thblock, Neuman_itr, &
         independ_nvec, nBlock, GMRES_m, GMRES_GSflag, PRECISION_A, PRECISION_b, &
         PRECISION_x, PRECISION_PRECONDITION, iret
    integer(c_int) :: ioff_grids(*), ndiv_grids(*), neighbor_ranks(*), num_grids(*)
    integer(c_int32_t) :: nrow
    integer(c_int32_t) :: ioff_dia(*)
    real(c_double) :: x(*), b(*), val_dia(*), reshistory(*), x_lo(*), b_lo(*), val_dia_lo(*)
    real(c_double) :: rtolmax
    call c_parcel_ddgmres_ddm(icomm, x, x_lo, b, b_lo, nrow, nnd, ioff_dia, val_dia, &
         val_dia_lo, num_neighbor_ranks, neighbor_ranks, margin, ncomp_grids, ndiv_grids, &
         num_grids, ioff_grids, div_direc_th, ipreflag, addL, iflagAS, itrmax, rtolmax, &
         reshistory, iovlflag, precon_thblock, Neuman_itr, independ_nvec, nBlock, GMRES_m, &
         GMRES_GSflag, PRECISION_A, PRECISION_b, PRECISION_x, PRECISION_PRECONDITION, iret)
  end subroutine parcel_ddgmres_ddm

end module ddm_wrapper
