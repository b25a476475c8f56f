/* parcel_b.h -- C ABI of libparcelb, a B200 (sm_100a) implementation of PARCEL-legacy's
 * single-process preconditioned Krylov solve on CRS matrices.
 *
 * Every entry point is `extern "C"` with plain pointers and sizes.  Two families:
 *
 *  1. Drop-in shims with the reference's C-callable signatures (every argument by
 *     reference, CRS 1-based with global column ids, int32 indices, real*8 values):
 *       parcel_init_c_, parcel_free_c_, parcel_dcg_c_, parcel_dbicgstab_c_,
 *       parcel_dgmres_c_, parcel_dcagmres_c_          (host arrays: the CPU-build ABI)
 *       parcel_d*_gpu_c_                              (device pointers: the GPU-build ABI)
 *  2. The native API: parcel_b_solve (PARCEL_KSP_CRS with the KSP_INPUT_PARAM struct),
 *     the split setup/solve handle API, and kernel-level entries used by tests.
 *
 * Pointer arguments of parcel_b_solve and the split API may be host or device memory;
 * the library detects which (cudaPointerGetAttributes) and copies host data in and out.
 *
 * Return convention: `iret` 0 = converged, 1 = iteration limit reached, as in the
 * reference (src/define.f90:101-102).  Where the reference stops the process
 * (zero pivot, matrix.f90:8018-8021; allocation failure, cu_common.h:119-124), this
 * library returns a negative PARCEL_B_E_* code in iret instead.
 */
#ifndef PARCEL_B_H
#define PARCEL_B_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------- */
#define PARCEL_B_OK 0
#define PARCEL_B_MAXITER 1
#define PARCEL_B_E_ZERO_PIVOT (-1)   /* reference: `stop` in ILU / D-ILU setup        */
#define PARCEL_B_E_ARG (-2)          /* invalid argument                               */
#define PARCEL_B_E_CUDA (-3)         /* CUDA runtime error                             */
#define PARCEL_B_E_BREAKDOWN (-4)    /* NaN / Inf in the iteration                     */
#define PARCEL_B_E_UNSUPPORTED (-5)  /* option this single-GPU build does not provide  */
#define PARCEL_B_E_NOMEM (-6)        /* device allocation failed                       */
#define PARCEL_B_E_NOT_INIT (-7)

/* ---- constants of src/define.f90:14-102 ------------------------------------------ */
#define PARCEL_B_SOLVER_CG 1
#define PARCEL_B_SOLVER_BICG 2
#define PARCEL_B_SOLVER_GMRES 3
#define PARCEL_B_SOLVER_CAGMRES 4
#define PARCEL_B_PRECON_NONE 0
#define PARCEL_B_PRECON_POINTJACOBI 1
#define PARCEL_B_PRECON_BLOCKJACOBI 2
#define PARCEL_B_PRECON_ADDITIVESCHWARZ 3
#define PARCEL_B_ILU0 0
#define PARCEL_B_ILUD 1
#define PARCEL_B_MLUD 2
#define PARCEL_B_GS_MGS 1
#define PARCEL_B_GS_CGS 2
#define PARCEL_B_BASIS_MONOMIAL 0
#define PARCEL_B_BASIS_NEWTON 1
#define PARCEL_B_QR_MGS 1
#define PARCEL_B_QR_CGS 2
#define PARCEL_B_QR_TSQR 3
#define PARCEL_B_QR_CHOLQR 4
#define PARCEL_B_QR_CHOLQR2 5

/* Inner arithmetic of the Krylov iteration (extension; the reference is FP64 only). */
#define PARCEL_B_INNER_FP64 0
#define PARCEL_B_INNER_FP32_REFINE 1 /* FP32 Krylov + FP32 preconditioner inside an
                                        FP64 / double-double iterative refinement loop */

/* KSP_INPUT_PARAM (src/type.f90:907-946), field for field and in the same order, followed
 * by this library's extensions.  A value of -1 selects the reference default
 * (PARCEL_KSP_Default_Setting, type.f90:949-1132; INIT_PARCEL_INPUT, wrapper.f90:5-45). */
typedef struct parcel_b_input {
  int ipreflag;
  int ILU_method;
  int addL;
  int iflagAS;
  int solver;
  int iovlflag;
  int GMRES_m;
  int GMRES_GSflag;
  int CAGMRES_sstep;
  int CAGMRES_tstep;
  int CAGMRES_basis;
  int CAGMRES_QRflag;
  int CBCG_kstep;
  int CBCG_Eigenflag;
  int power_method_itrmax;
  int CAARNOLDI_sstep;
  int CAARNOLDI_tstep;
  int CAARNOLDI_basis;
  int CAARNOLDI_QRflag;
  int machineflag;
  int dataflag;
  int calcflag;
  int Neuman_itr;
  int Neuman_local;
  int itrmax;
  double rtolmax;
  double abstolmax;
  int independ_nvec;
  int precon_thblock;
  int nBlock;
  int PRECISION_A;
  int PRECISION_b;
  int PRECISION_x;
  int PRECISION_PRECONDITION;
  /* ---- extensions ---- */
  int inner_precision;    /* PARCEL_B_INNER_*                                     */
  int residual_dd;        /* 1: outer residual b - A x in double-double            */
  double inner_rtol;      /* relative tolerance of each inner solve (FP32 path)     */
  int max_refine;         /* outer refinement steps (FP32 path)                     */
  int reserved[7];
} parcel_b_input;

/* Fills every field with -1 / defaults (INIT_PARCEL_INPUT, wrapper.f90:5-45). */
void parcel_b_input_init(parcel_b_input* p);

/* CRS matrix of one process, reference layout: rowptr has n+1 entries with
 * rowptr[0] = 1, col holds 1-based global column ids sorted within each row, istart is
 * the 1-based global id of the first row (1 on one process). */
typedef struct parcel_b_crs {
  int32_t n;
  int32_t gn;
  int64_t nnz;
  int32_t istart;
  const int32_t* rowptr;
  const int32_t* col;
  const double* val;
} parcel_b_crs;

/* Matrix in DIA format (PARCEL_KSP_DIA, src/wrapper.f90:224-357): val[j*n + k] is the entry
 * of row k (0-based) on diagonal j, whose 1-based global column is k + istart + offset[j];
 * nnd distinct offsets.  Entries equal to zero, and entries whose column falls outside rows
 * 1..n, are not part of the matrix. */
typedef struct parcel_b_dia {
  int32_t n;
  int32_t gn;
  int32_t istart;
  int32_t nnd;
  const double* val;
  const int32_t* offset;
} parcel_b_dia;

/* DDM stencil format (src/src_DDM; argument list of parcel_dcg_ddm_c,
 * src/example/c2fortran_kernel.f90:2964-3064): one process's box of a structured grid,
 * padded by `margin` cells on both sides of each of the ndim axes, x fastest, so the box
 * holds m = prod(n_grids[d] + 2 margin) cells (set_grids_decompostion,
 * src/example/ddm_setup.f90).  Stencil point k couples interior cell j with cell
 * j + offset[k], offset[k] = sum_d offset_dim[k + nnd d] * stride_d, with the value
 * val[k m + j] (diaA); margin cells carry no unknowns.  b and x hold m entries (the
 * interior cells are used; x's margin is left as it is). */
#define PARCEL_B_DDM_BOXES_THREADS 0   /* CPU build: precon_thblock slabs along div_direc_th */
#define PARCEL_B_DDM_BOXES_CUBES   1   /* GPU build (DDM_CUDA_BJ): n_d / 4 boxes per axis    */
typedef struct parcel_b_ddm {
  int32_t ndim;                /* 1..3                                                      */
  int32_t n_grids[3];          /* interior cells per axis (entries beyond ndim ignored)     */
  int32_t margin;              /* padding cells per side, >= the largest |offset_dim|       */
  int64_t m;                   /* padded cells (n of parcel_dcg_ddm_c)                       */
  int32_t nnd;                 /* stencil points, at most 32                                 */
  const int32_t* offset;       /* nnd linear offsets                                         */
  const int32_t* offset_dim;   /* nnd x ndim per-axis offsets, column-major (offset_dim)     */
  const double* val;           /* nnd x m values (diaA)                                      */
  int32_t div_direc_th;        /* thread-slab axis: 1 x, 2 y, 3 z                            */
  int32_t boxes;               /* PARCEL_B_DDM_BOXES_*                                       */
} parcel_b_ddm;

/* Per-solve statistics (extension). */
typedef struct parcel_b_stats {
  double setup_s;           /* preconditioner + layout setup, wall seconds           */
  double solve_s;           /* Krylov iteration, wall seconds                        */
  double total_s;
  double true_relres;       /* ||b - A x|| / ||b|| in FP64 at exit                   */
  double true_relres_dd;    /* same, residual computed in double-double (if asked)   */
  int niter;
  int iret;
  int refine_steps;         /* FP32 path: outer refinement steps                     */
  int kernel_launches;      /* kernels this library launched for the solve           */
  int ilu_levels_max;       /* longest wavefront (levels) of any block-Jacobi block  */
  int ilu_nblocks;
  int fallback;             /* learned solve: right-hand sides the plain PGMRES finished */
  int spmv_diagonals;       /* > 0: the SpMV ran on a diagonal (DIA) copy with this many
                               diagonals (natural layout: no or point-Jacobi preconditioner) */
  int reserved[4];
} parcel_b_stats;

/* ---- lifecycle: PARCEL_Init / PARCEL_Free (src/c_krylov_wrapper.f90:6-23,
 *      src/example/c2fortran_kernel.f90:1-10) -------------------------------------- */
void parcel_init_c_(int* myrank);
void parcel_free_c_(void);
/* Selects the CUDA stream the library launches on (NULL: a private non-blocking stream). */
int parcel_b_set_stream(void* cuda_stream);
void* parcel_b_get_stream(void);
/* Last error message and code of this thread's most recent failing call. */
int parcel_b_last_error(char* buf, int buflen);
/* Statistics of the most recent solve. */
int parcel_b_last_stats(parcel_b_stats* out);

/* ---- generic entry: PARCEL_KSP_CRS (src/wrapper.f90:47-222) ------------------------
 * x holds x0 on entry and the solution on exit; reshistory has itrmax entries;
 * niter returns the iterations used; iret as described above. */
int parcel_b_solve(const parcel_b_input* prm, const parcel_b_crs* A, const double* b,
                   double* x, double* reshistory, int* niter, int* iret);

/* PARCEL_KSP_DIA: as parcel_b_solve for a DIA matrix (host or device arrays).  The DIA
 * arrays become CRS once, on the GPU (each row's nonzero entries in ascending column
 * order, as dia2crs, src/matrix.f90:7536-7576, gives them for ascending offsets), and the
 * CRS solve runs on that; the conversion time is part of the setup statistics. */
int parcel_b_solve_dia(const parcel_b_input* prm, const parcel_b_dia* A, const double* b,
                       double* x, double* reshistory, int* niter, int* iret);
/* PARCEL_ddKSP_DIA: the double-double CG / BiCGStab / GMRES (prm->solver 1, 2 or 3) on a
 * DIA matrix, with the arguments of parcel_b_ddcg (val_lo: the low parts, laid out as
 * A->val). */
int parcel_b_ddsolve_dia(const parcel_b_input* prm, const parcel_b_dia* A, const double* val_lo,
                         int precision_A, int precision_b, int precision_x, int precision_precondition,
                         const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                         double* reshistory, int* niter, int* iret);

/* parcel_ddm_main (src/src_DDM/ddm_kernel.f90:463-1756) on one process: CG / BiCGStab /
 * GMRES / CA-GMRES (prm->solver) on the interior cells of a DDM box (host or device arrays).
 * ipreflag 0 none, 1 point Jacobi, 2 block-Jacobi D-ILU on the boxes A->boxes selects
 * (precon_thblock slabs for PARCEL_B_DDM_BOXES_THREADS); ILU_method is not used (the DDM
 * preconditioner is D-ILU).  Not provided: additive Schwarz (ipreflag 3), the Neumann
 * series (4) and the x-line-independent D-ILU (independ_nvec = 1), each refused with
 * PARCEL_B_E_UNSUPPORTED.  The cells are renumbered box by box, each box's cells in
 * lexicographic order, and the CRS solvers run on that matrix with the boxes as the
 * block-Jacobi blocks; the renumbering time is part of the setup statistics. */
int parcel_b_solve_ddm(const parcel_b_input* prm, const parcel_b_ddm* A, const double* b, double* x,
                       double* reshistory, int* niter, int* iret);
/* parcel_ddm_main_dd (ddm_kernel.f90:1758-1899): the double-double CG / BiCGStab / GMRES
 * (prm->solver 1, 2 or 3) on a DDM box, with the arguments of parcel_b_ddcg (val_lo: the
 * low parts, laid out as A->val; b_lo / x_lo: m entries or NULL). */
int parcel_b_ddsolve_ddm(const parcel_b_input* prm, const parcel_b_ddm* A, const double* val_lo,
                         int precision_A, int precision_b, int precision_x, int precision_precondition,
                         const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                         double* reshistory, int* niter, int* iret);
/* The renumbering of a DDM box: perm[r] (0-based padded cell of row r, for the interior
 * cells) and the rows at which the boxes start (starts[0] = 0, starts[nb] = interior
 * cells).  *nblocks: in, the capacity of starts minus one; out, the number of boxes (the
 * call fails with PARCEL_B_E_ARG, having set it, when the capacity is too small).  perm may
 * be NULL. */
int parcel_b_ddm_order(const parcel_b_ddm* A, int precon_thblock, int32_t* perm, int32_t* starts,
                       int32_t* nblocks);

/* ---- drop-in shims, CPU-build ABI (host arrays; src/example/c2fortran_kernel.f90) ----
 * parcel_dcg_c       : c2fortran_kernel.f90:334-432  -> parcel_dcg (wrapper.f90:1995)
 * parcel_dbicgstab_c : c2fortran_kernel.f90:434-521  -> parcel_dbicgstab (wrapper.f90:1813)
 * parcel_dgmres_c    : c2fortran_kernel.f90:523-618  -> parcel_dgmres (wrapper.f90:2179)
 * parcel_dcagmres_c  : c2fortran_kernel.f90:901-1004 -> parcel_dcagmres (wrapper.f90:2807)
 * niter: in = itrmax, out = iterations used (wrapper.f90:630). */
void parcel_dcg_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                   int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                   int32_t* crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                   int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                   int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                   int* iret);
void parcel_dbicgstab_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                         int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                         int32_t* crscol, int* ipreflag, int* ilu_method, int* addl,
                         int* iflagas, int* niter, double* rtolmax, double* reshistory,
                         int* iovlflag, int* precon_thblock, int* neuman_itr,
                         int* independ_nvec, int* nblock, int* iret);
void parcel_dgmres_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                      int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                      int32_t* crscol, int* ipreflag, int* ilu_method, int* addl,
                      int* iflagas, int* niter, double* rtolmax, double* reshistory,
                      int* iovlflag, int* precon_thblock, int* neuman_itr,
                      int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag,
                      int* iret);
void parcel_dcagmres_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                        int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                        int32_t* crscol, int* ipreflag, int* ilu_method, int* addl,
                        int* iflagas, int* niter, double* rtolmax, double* reshistory,
                        int* iovlflag, int* precon_thblock, int* neuman_itr,
                        int* independ_nvec, int* nblock, int* cagmres_sstep,
                        int* cagmres_tstep, int* cagmres_basis, int* cagmres_qrflag,
                        int* iret);

/* ---- drop-in shims, GPU-build ABI: vecx, vecb, crsa, crsrow_ptr and crscol are passed
 * as `devicemem*` (src/CUDA/src/cu_common.h:37-42), whose first member is the device
 * pointer; a `void**` pointing at the device pointer is the same thing. ------------- */
/* parcel_ddcg_c (src/example/c2fortran_kernel.f90:620-708): the double-double CG with the
 * reference's argument order; host arrays; niter in = itrmax, out = iterations. */
void parcel_ddcg_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                    int32_t* gn, int32_t* nnz, int32_t* istart, double* crsa, double* crsa_lo,
                    int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag, int* ilu_method, int* addl,
                    int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                    int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                    int* precision_a, int* precision_b, int* precision_x, int* precision_precondition,
                    int* iret);
/* parcel_ddbicgstab_c (src/example/c2fortran_kernel.f90:710-799): same argument list. */
void parcel_ddbicgstab_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                          int32_t* gn, int32_t* nnz, int32_t* istart, double* crsa, double* crsa_lo,
                          int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag, int* ilu_method, int* addl,
                          int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                          int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                          int* precision_a, int* precision_b, int* precision_x, int* precision_precondition,
                          int* iret);
/* parcel_ddgmres_c (src/example/c2fortran_kernel.f90:801-898): the same list with the
 * restart length and the Gram-Schmidt flag after nblock. */
void parcel_ddgmres_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                       int32_t* gn, int32_t* nnz, int32_t* istart, double* crsa, double* crsa_lo,
                       int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag, int* ilu_method, int* addl,
                       int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                       int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* restart,
                       int* gmres_gsflag, int* precision_a, int* precision_b, int* precision_x,
                       int* precision_precondition, int* iret);
/* DIA shims (src/example/c2fortran_kernel.f90:1228-1872): the CRS lists with n, gn, istart,
 * diaA, offset, nnd in place of n, gn, nnz, istart, crsa, crsrow_ptr, crscol. */
void parcel_dcg_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                       double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                       int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                       int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* iret);
void parcel_dbicgstab_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                             double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                             int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                             int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* iret);
void parcel_dgmres_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                          double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                          int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                          int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* restart,
                          int* gmres_gsflag, int* iret);
void parcel_dcagmres_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                            double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                            int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                            int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                            int* cagmres_sstep, int* cagmres_tstep, int* cagmres_basis, int* cagmres_qrflag,
                            int* iret);
void parcel_ddcg_dia_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                        int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset, int32_t* nnd,
                        int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                        double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                        int* independ_nvec, int* nblock, int* precision_a, int* precision_b, int* precision_x,
                        int* precision_precondition, int* iret);
void parcel_ddbicgstab_dia_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                              int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset,
                              int32_t* nnd, int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter,
                              double* rtolmax, double* reshistory, int* iovlflag, int* precon_thblock,
                              int* neuman_itr, int* independ_nvec, int* nblock, int* precision_a, int* precision_b,
                              int* precision_x, int* precision_precondition, int* iret);
/* parcel_ddgmres_dia_c has no Neuman_itr argument (c2fortran_kernel.f90:1681-1773). */
void parcel_ddgmres_dia_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                           int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset,
                           int32_t* nnd, int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter,
                           double* rtolmax, double* reshistory, int* iovlflag, int* precon_thblock,
                           int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag, int* precision_a,
                           int* precision_b, int* precision_x, int* precision_precondition, int* iret);
void parcel_dcg_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                       int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                       void** crscol, int* ipreflag, int* ilu_method, int* addl,
                       int* iflagas, int* niter, double* rtolmax, double* reshistory,
                       int* iovlflag, int* precon_thblock, int* neuman_itr,
                       int* independ_nvec, int* nblock, int* iret);
void parcel_dbicgstab_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                             int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                             void** crscol, int* ipreflag, int* ilu_method, int* addl,
                             int* iflagas, int* niter, double* rtolmax, double* reshistory,
                             int* iovlflag, int* precon_thblock, int* neuman_itr,
                             int* independ_nvec, int* nblock, int* iret);
void parcel_dgmres_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                          int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                          void** crscol, int* ipreflag, int* ilu_method, int* addl,
                          int* iflagas, int* niter, double* rtolmax, double* reshistory,
                          int* iovlflag, int* precon_thblock, int* neuman_itr,
                          int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag,
                          int* iret);
void parcel_dcagmres_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                            int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                            void** crscol, int* ipreflag, int* ilu_method, int* addl,
                            int* iflagas, int* niter, double* rtolmax, double* reshistory,
                            int* iovlflag, int* precon_thblock, int* neuman_itr,
                            int* independ_nvec, int* nblock, int* cagmres_sstep,
                            int* cagmres_tstep, int* cagmres_basis, int* cagmres_qrflag,
                            int* iret);
/* DIA shims of the CUDA build: vecx, vecb, diaA and offset as device pointers passed by
 * reference (type(c_ptr) arguments). */
void parcel_dcg_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                           void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                           int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                           int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* iret);
void parcel_dbicgstab_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                                 void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method,
                                 int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                                 int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                                 int* nblock, int* iret);
void parcel_dgmres_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                              void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                              int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                              int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* restart,
                              int* gmres_gsflag, int* iret);
void parcel_dcagmres_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                                void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method,
                                int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                                int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                                int* nblock, int* cagmres_sstep, int* cagmres_tstep, int* cagmres_basis,
                                int* cagmres_qrflag, int* iret);

/* ---- DDM drop-in shims (src/example/c2fortran_kernel.f90:2964-3691) -----------------
 * parcel_dcg_ddm_c 2964-3064, parcel_dbicgstab_ddm_c 3066-3164, parcel_dgmres_ddm_c
 * 3166-3270, parcel_ddcg_ddm_c 3272-3371, parcel_ddbicgstab_ddm_c 3373-3472,
 * parcel_ddgmres_ddm_c 3474-3578, parcel_dcagmres_ddm_c 3580-3691.  n = m padded cells;
 * one process (npe_dim all 1, no neighbour ranks; a box split over processes runs through
 * parcel_b.ddm on torch.distributed).  The CPU-build forms (host arrays) cut the boxes as
 * the CPU build does (precon_thblock slabs along div_direc_th), the _gpu_ forms (device
 * arrays behind devicemem handles, as the CUDA build passes them) as the CUDA build does
 * (n_d / 4 boxes per axis).  niter: in = itrmax, out = iterations used. */
void parcel_dcg_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                       double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim,
                       int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag,
                       int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                       int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                       int* iret);
void parcel_dbicgstab_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                             double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                             int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                             int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                             double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                             int* independ_nvec, int* nblock, int* iret);
void parcel_dgmres_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                          double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                          int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                          int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                          double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                          int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag, int* iret);
void parcel_dcagmres_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                            double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                            int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                            int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                            double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                            int* independ_nvec, int* nblock, int* cagmres_sstep, int* cagmres_tstep,
                            int* cagmres_basis, int* cagmres_qrflag, int* iret);
void parcel_ddcg_ddm_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                        int32_t* n, int* nnd, int32_t* offset, double* diaA, double* diaA_lo,
                        int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim, int* npe_dim,
                        int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag, int* addl,
                        int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                        int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                        int* precision_A, int* precision_b, int* precision_x, int* precision_precondition,
                        int* iret);
void parcel_ddbicgstab_ddm_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                              int32_t* n, int* nnd, int32_t* offset, double* diaA, double* diaA_lo,
                              int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim,
                              int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag,
                              int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                              int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                              int* nblock, int* precision_A, int* precision_b, int* precision_x,
                              int* precision_precondition, int* iret);
void parcel_ddgmres_ddm_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                           int32_t* n, int* nnd, int32_t* offset, double* diaA, double* diaA_lo,
                           int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim,
                           int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag,
                           int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                           int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                           int* nblock, int* restart, int* gmres_gsflag, int* precision_A, int* precision_b,
                           int* precision_x, int* precision_precondition, int* iret);
void parcel_dcg_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                           void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                           int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                           int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                           double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                           int* independ_nvec, int* nblock, int* iret);
void parcel_dbicgstab_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                                 void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                                 int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                                 int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                                 double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                                 int* independ_nvec, int* nblock, int* iret);
void parcel_dgmres_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                              void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                              int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                              int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                              double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                              int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag, int* iret);
void parcel_dcagmres_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                                void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                                int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                                int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                                double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                                int* independ_nvec, int* nblock, int* cagmres_sstep, int* cagmres_tstep,
                                int* cagmres_basis, int* cagmres_qrflag, int* iret);

/* ---- split setup / solve (set_ksp_crs_c, start_ksp_solver_crs_c, get_vecx_ksp_crs_c,
 *      get_reshistory_ksp_crs_c: src/example/c2fortran_kernel.f90:2855-2961) ----------
 * A handle keeps the matrix layout and preconditioner on the device between solves. */
typedef struct parcel_b_handle_s* parcel_b_handle;
int parcel_b_setup(const parcel_b_input* prm, const parcel_b_crs* A, parcel_b_handle* out);
int parcel_b_start(parcel_b_handle h, const double* b, double* x, double* reshistory,
                   int* niter, int* iret);
int parcel_b_release(parcel_b_handle h);

/* ---- kernel-level entries (tests and benchmarks) ---------------------------------- */
/* y = A x with the library's CRS SpMV (MatVec_crs, matrix.f90:1348-1512); device arrays. */
int parcel_b_spmv(const parcel_b_crs* A, const double* x, double* y);
/* y = A x in FP32 values and vectors (the mixed-precision inner SpMV); device arrays. */
int parcel_b_spmv_f32(int32_t n, int64_t nnz, int32_t istart, const int32_t* rowptr,
                      const int32_t* col, const float* val, const float* x, float* y);
/* s = M^-1 r for the preconditioner described by prm (setup + one application);
 * host or device arrays. */
int parcel_b_precon_apply(const parcel_b_input* prm, const parcel_b_crs* A, const double* r,
                          double* s);
/* Deterministic dot product of two device vectors. */
int parcel_b_dot(int64_t n, const double* x, const double* y, double* out_host);
/* Dot product of two device vectors that allocates nothing (no counterpart in the
 * reference).  For callers that may not allocate device memory while they run (their
 * own memory pool owns the GPU, or a cudaMalloc would synchronise a pipeline): scratch
 * is a fixed file-scope device array, the kernel runs on `stream` (a cudaStream_t, NULL
 * for the legacy default stream) and writes *result_dev (device memory) without a host
 * synchronisation.  Same result as parcel_b_dot up to rounding (different block size).
 *   - n <= 67,108,864 (one partial per 16,384 elements, 4,096 partials); larger n
 *     returns PARCEL_B_E_ARG;
 *   - one scratch array per device shared by all calls: calls that overlap on the GPU
 *     race; serialise them;
 *   - the first call on a device resolves the array's address on the current device:
 *     make it before any stream capture. */
int parcel_b_dot_noalloc(int64_t n, const double* x, const double* y, double* result_dev,
                         void* stream);
/* r = b - A x in double-double with the reference's dd add / mul order
 * (dd_func.f90:5-98); A values, b and x given as (hi, lo) pairs, lo may be NULL. Device
 * arrays; returns r as (r_hi, r_lo). */
int parcel_b_residual_dd(const parcel_b_crs* A, const double* x_hi, const double* x_lo,
                         const double* b_hi, const double* b_lo, double* r_hi, double* r_lo);

/* Double-double preconditioned CG (ddKSP_pCG, src/ddpcg.f90:247-563, called through
 * PARCEL_ddKSP_CRS's precision flags, src/ddwrapper.f90:184-280).  Each of A, b, x and
 * the preconditioner is in double (1) or double-double (2): a low-part array (val_lo,
 * b_lo, x_lo) is used when its flag is 2 and may be NULL otherwise (or to mean zero).
 * prm->solver is ignored (CG); ipreflag 0 (none), 1 (point Jacobi) or 2/3 (block-Jacobi
 * D-ILU, ILU_method 1 or 2; ILU(0) returns PARCEL_B_E_UNSUPPORTED).  x_hi (and x_lo when
 * precision_x is 2) in/out.  Host or device arrays.  The reference runs this solver on
 * the CPU only; here it runs on the GPU with the reference's dd operation order
 * (dd_func.f90) and a fixed dot-product split, bit-for-bit reproducible. */
int parcel_b_ddcg(const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo, int precision_A,
                  int precision_b, int precision_x, int precision_precondition, const double* b_hi,
                  const double* b_lo, double* x_hi, double* x_lo, double* reshistory, int* niter, int* iret);
/* Double-double BiCGStab (ddKSP_pBiCG, src/ddpbicg.f90:496-875), right-preconditioned,
 * with the same arguments and preconditioners as parcel_b_ddcg; the history entry is the
 * high part of the dd quotient rnorm / bnorm, as in the reference. */
int parcel_b_ddbicgstab(const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo, int precision_A,
                        int precision_b, int precision_x, int precision_precondition, const double* b_hi,
                        const double* b_lo, double* x_hi, double* x_lo, double* reshistory, int* niter, int* iret);
/* Double-double GMRES(m) (ddKSP_pGMRES, src/ddpgmres.f90:254-713), right-preconditioned,
 * with the same arguments and preconditioners as parcel_b_ddcg; the restart length is
 * prm->GMRES_m and the orthogonalisation prm->GMRES_GSflag (MGS or CGS, as in
 * ddQRDecomposition.f90:4-121).  niter and the history follow the reference: entry 1 is
 * the starting residual and entry k + 1 the residual after iteration k. */
int parcel_b_ddgmres(const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo, int precision_A,
                     int precision_b, int precision_x, int precision_precondition, const double* b_hi,
                     const double* b_lo, double* x_hi, double* x_lo, double* reshistory, int* niter, int* iret);

/* Kernel timing for benchmarks: builds the solver layout and preconditioner described by
 * prm (setup excluded from the timing), then launches `reps` back-to-back SpMVs and `reps`
 * preconditioner applications on the library stream and returns the mean milliseconds per
 * launch of each, measured with CUDA events on that stream.  Host or device matrix.  With
 * prm->inner_precision = 1 it times the FP32 system of the mixed-precision path. */
int parcel_b_bench_kernels(const parcel_b_input* prm, const parcel_b_crs* A, int reps,
                           double* ms_spmv, double* ms_precon);
/* As parcel_b_bench_kernels for a DDM box: the renumbered system and its boxes as the
 * block-Jacobi blocks, as parcel_b_solve_ddm builds them. */
int parcel_b_bench_kernels_ddm(const parcel_b_input* prm, const parcel_b_ddm* A, int reps, double* ms_spmv,
                               double* ms_precon);

/* ---- one process's share of a row-distributed system ---------------------------------
 * The GPU side of the multi-process solve (parcel_b/dist.py), which mirrors the reference's
 * MPI decomposition: contiguous rows per process (src/krylov.f90:447-470), the halo of x
 * exchanged before every product (src/comm.f90:528-597), block-Jacobi blocks inside each
 * process (src/matrix.f90:8074-8134).  A holds this process's n rows with local column ids:
 * 1..n for owned rows, n+1..n_ext for halo values (istart = 1; host or device arrays).  The
 * preconditioner of prm (none, point Jacobi or block-Jacobi ILU / D-ILU over the owned rows,
 * precon_thblock blocks) is built on the owned-owned submatrix. */
typedef struct parcel_b_local_s* parcel_b_local;
int parcel_b_local_create(const parcel_b_input* prm, const parcel_b_crs* A, int n_ext, parcel_b_local* out);
/* As parcel_b_local_create, with explicit block-Jacobi blocks: the owned rows
 * [starts[b], starts[b+1]) for b < nblocks (starts[0] = 0, starts[nblocks] = n; the boxes of
 * a DDM process, parcel_b_ddm_order). */
int parcel_b_local_create_blocks(const parcel_b_input* prm, const parcel_b_crs* A, int n_ext, int nblocks,
                                 const int32_t* starts, parcel_b_local* out);
/* y[n] = A x_ext[n_ext], device arrays. */
int parcel_b_local_spmv(parcel_b_local h, const double* x_ext, double* y);
/* z[n] = M^-1 r[n], device arrays. */
int parcel_b_local_precon(parcel_b_local h, const double* r, double* z);
int parcel_b_local_destroy(parcel_b_local h);

/* ---- learned two-level preconditioner stage (no counterpart in the reference) --------
 * Flexible GMRES with the additive two-level preconditioner
 *   z = M^-1 v + P y,   y ~ A_c^-1 P^T v,   A_c = P^T A P  (Galerkin, 27-point),
 * on a structured nx x ny x nz grid (natural row = (z ny + y) nx + x) coarsened by an even
 * factor c: P = cell-centred trilinear interpolation clamped at the boundary.  y comes from
 * coarse_steps Jacobi-preconditioned CG iterations on A_c, started from the network's
 * prediction of the coarse error (scaled by the A_c-optimal gamma) or from zero.
 * Net: six BF16 3x3x3 convolutions, 2 -> 32 -> 32 -> 32 -> 32 -> 32 -> 1 channels, ReLU
 * between, zero padding, FP32 sums; inputs [P^T v / rms, dhat], dhat = normalised coarse
 * log|diag A|.  Parameters (FP32): for layer l = 0..5, W_l[27][C_in][C_out]
 * (tap 9(dz+1)+3(dy+1)+(dx+1)) then b_l[C_out]. */
typedef struct parcel_b_learned_s* parcel_b_learned;
int parcel_b_learned_create(int nx, int ny, int nz, int coarsen, uint64_t seed, parcel_b_learned* out);
int parcel_b_learned_destroy(parcel_b_learned h);
int64_t parcel_b_learned_num_params(void);
/* FP32 master parameters (host or device array of num_params) and the target scale s. */
int parcel_b_learned_get_params(parcel_b_learned h, float* params, double* target_scale);
/* params may be NULL (keep); target_scale <= 0 keeps the current one. */
int parcel_b_learned_set_params(parcel_b_learned h, const float* params, double target_scale);
/* The network alone on `batch` coarse grids: u [batch][V][2] FP32 (rounded to BF16 on
 * entry), y [batch][V]; V = (nx ny nz) / coarsen^3; host or device arrays. */
int parcel_b_learned_forward(parcel_b_learned h, int batch, const float* u, float* y);
/* loss = 1/(2 M) sum (y - target)^2 over the M = batch V outputs and its gradient with
 * respect to every parameter (FP32, parameter layout), kept for parcel_b_learned_adam. */
int parcel_b_learned_grad(parcel_b_learned h, int batch, const float* u, const float* target,
                          double* loss, float* grad);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) with the last gradient. */
int parcel_b_learned_adam(parcel_b_learned h, double lr);
/* Solves A x = b with the plain GMRES of prm (x0 = 0) and appends up to max_pairs
 * training pairs, one per residual r = b - A x_k after each restart cycle (x_0 = 0
 * included): input [P^T r / sigma, dhat], target y / sigma with A_c y = P^T r (400 coarse
 * PCG iterations), sigma = rms(P^T r).  Needs an even coarsening factor. */
int parcel_b_learned_collect(parcel_b_learned h, const parcel_b_input* prm, const parcel_b_crs* A,
                             const double* b, int max_pairs, int* npairs);
int parcel_b_learned_num_pairs(parcel_b_learned h);
/* Adam over the collected pairs: `steps` steps of `batch` pairs drawn with `seed`. */
int parcel_b_learned_train(parcel_b_learned h, int steps, int batch, double lr, uint64_t seed,
                           double* first_loss, double* last_loss);
/* Coarse solve of the stage: coarse_steps >= 0 Jacobi-PCG iterations, started from the
 * network's guess (use_net 1) or from zero (use_net 0).  Defaults: 8 and 1. */
int parcel_b_learned_set_stage(parcel_b_learned h, int coarse_steps, int use_net);
/* The stage's Galerkin operator for A on the handle's grid: ac[27][Vc] FP64, tap
 * t = 9(dz+1)+3(dy+1)+(dx+1), zero where the neighbour lies outside the coarse grid. */
int parcel_b_learned_galerkin(parcel_b_learned h, const parcel_b_crs* A, double* ac);
/* The stage's coarse solve on its own: `steps` Jacobi-PCG iterations on A_c y = rc (FP32,
 * one thread-block cluster), from zero (g0 NULL) or from gamma g0. */
int parcel_b_learned_coarse_solve(parcel_b_learned h, const parcel_b_crs* A, const float* rc, const float* g0,
                                  int steps, float* y);
/* Grid transfers in the natural layout: to_coarse 1: out[Vc] = P^T in[n]; 0: out[n] = P in[Vc]
 * (computed in FP32). */
int parcel_b_learned_transfer(parcel_b_learned h, int to_coarse, const double* in, double* out);
/* Flexible GMRES(GMRES_m) with M from prm and the learned stage (h NULL: M alone), FP64
 * or, with inner_precision = 1, FP32 inside the FP64 refinement loop.  If the FP64 true
 * residual misses rtolmax, plain PGMRES with M continues from x (stats.fallback = 1). */
int parcel_b_solve_learned(const parcel_b_input* prm, const parcel_b_crs* A, parcel_b_learned h,
                           const double* b, double* x, double* reshistory, int* niter, int* iret);
/* nrhs systems A x_k = b_k with one set-up (layout, ILU factors, learned stage), solved one
 * after the other on the device: b and x hold nrhs vectors of n entries each, niter and
 * iret nrhs entries.  Statistics: setup_s once, solve_s for all, true_relres the worst. */
int parcel_b_solve_learned_many(const parcel_b_input* prm, const parcel_b_crs* A, parcel_b_learned h,
                                int nrhs, const double* b, double* x, int* niter, int* iret);

#ifdef __cplusplus
}
#endif
#endif /* PARCEL_B_H */
