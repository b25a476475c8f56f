// pb_dia.cu -- DIA-format input: PARCEL_KSP_DIA / PARCEL_ddKSP_DIA and the parcel_d*_dia shims.
//
// Reference: PARCEL_KSP_DIA (src/wrapper.f90:224-357) -> KSP_DIA and set_KSP_DIA
// (src/krylov.f90:159-445, 845-905).  The DIA arrays hold diaA(k + (j-1) n) = A(Row, Row +
// offset(j)) with Row = k - 1 + istart; the reference takes the entries whose magnitude
// exceeds minReal8 = 0 as the matrix (get_nnz_dia and dia2crs, src/matrix.f90:7536-7607;
// src/type.f90:445), and its DIA solve follows its CRS solve (template_cpu/STDOUT_run prints
// the same CG history for both).  Here the DIA arrays are converted once, on the device,
// into CRS: each row keeps its nonzero entries with the diagonals walked in ascending offset
// order, so the columns come out sorted, and the CRS solver runs on that.  An entry whose
// column falls outside this process's rows multiplies a halo value in the reference (zero
// on one process) and is left out here.  The iteration matrix and the preconditioner are
// then the CRS path's (sliced ELLPACK in the block-Jacobi level order, where the diagonals
// of the stencil are no longer diagonals).
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>
#include <numeric>
#include <vector>

#include "pb_api.cuh"

namespace pb {
namespace {

constexpr int kDiaThreads = 256;

inline int dia_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kDiaThreads - 1) / kDiaThreads, 8LL * num_sms()));
}

__device__ __forceinline__ bool dia_keep(const double* vh, const double* vl, int64_t q) {
  return fabs(vh[q]) > 0.0 || (vl != nullptr && fabs(vl[q]) > 0.0);
}

// Entries kept in row k (0-based): nonzero, column inside [0, n).  cnt[k] = count.
__global__ void k_dia_count(int n, int nnd, const double* __restrict__ vh, const double* __restrict__ vl,
                            const int* __restrict__ ord, const int* __restrict__ off, int* __restrict__ cnt) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    int c = 0;
    for (int jj = 0; jj < nnd; ++jj) {
      const int j = ord[jj];
      const int64_t col = k + off[j];
      if (col >= 0 && col < n && dia_keep(vh, vl, (int64_t)j * n + k)) ++c;
    }
    cnt[k] = c;
  }
}

// Row k's entries in ascending offset order: 1-based global columns, values (and low parts).
// rp holds the 0-based row starts; it is turned into the 1-based CRS row pointer afterwards.
__global__ void k_dia_fill(int n, int nnd, int istart, const double* __restrict__ vh, const double* __restrict__ vl,
                           const int* __restrict__ ord, const int* __restrict__ off, const int* __restrict__ rp,
                           int* __restrict__ col_out, double* __restrict__ vh_out, double* __restrict__ vl_out) {
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    int p = rp[k];
    for (int jj = 0; jj < nnd; ++jj) {
      const int j = ord[jj];
      const int64_t col = k + off[j];
      const int64_t q = (int64_t)j * n + k;
      if (col >= 0 && col < n && dia_keep(vh, vl, q)) {
        col_out[p] = (int)(col + istart);
        vh_out[p] = vh[q];
        if (vl_out) vl_out[p] = vl ? vl[q] : 0.0;
        ++p;
      }
    }
  }
}

__global__ void k_add_one(int64_t m, int* __restrict__ a) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
    a[i] += 1;
}

// CRS arrays built from a DIA matrix, on the device.
struct DiaCrs {
  DBuf rowptr, col, vh, vl;
  parcel_b_crs crs;
  const double* lo() const { return vl.p ? dp<double>(vl) : nullptr; }
};

// Converts A (host or device arrays; val_lo may be null) into device CRS.
void dia_to_crs(const parcel_b_dia* A, const double* val_lo, DiaCrs& out) {
  PB_CHECK(A != nullptr, PARCEL_B_E_ARG, "matrix is NULL");
  PB_CHECK(A->n > 0, PARCEL_B_E_ARG, "n = %d", A->n);
  PB_CHECK(A->nnd > 0, PARCEL_B_E_ARG, "nnd = %d", A->nnd);
  PB_CHECK(A->val && A->offset, PARCEL_B_E_ARG, "DIA arrays must not be NULL");
  PB_CHECK(A->gn <= 0 || A->gn == A->n, PARCEL_B_E_UNSUPPORTED,
           "n=%d != gn=%d: a matrix split over processes needs the MPI halo exchange, "
           "which this single-GPU build does not provide", A->n, A->gn);
  PB_CHECK(A->istart == 1, PARCEL_B_E_UNSUPPORTED, "istart=%d: one process owns rows 1..n", A->istart);
  PB_CHECK((int64_t)A->nnd * A->n < (int64_t)INT32_MAX, PARCEL_B_E_UNSUPPORTED,
           "nnd x n = %lld entries: the CRS built from them is indexed by int32",
           (long long)A->nnd * A->n);
  cudaStream_t st = stream();
  const int n = A->n, nnd = A->nnd;
  const size_t nv = (size_t)nnd * (size_t)n;
  // offsets: ascending order of the diagonals (distinct offsets required)
  std::vector<int> off(nnd);
  if (is_device_ptr(A->offset)) d2h(off.data(), A->offset, sizeof(int) * nnd);
  else std::memcpy(off.data(), A->offset, sizeof(int) * nnd);
  std::vector<int> ord(nnd);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return off[a] < off[b]; });
  for (int i = 1; i < nnd; ++i)
    PB_CHECK(off[ord[i]] != off[ord[i - 1]], PARCEL_B_E_ARG, "offset %d appears twice in the DIA offsets",
             off[ord[i]]);
  DBuf doff(sizeof(int) * nnd), dord(sizeof(int) * nnd);
  h2d(doff.p, off.data(), sizeof(int) * nnd);
  h2d(dord.p, ord.data(), sizeof(int) * nnd);
  DBuf hv, lv;
  const double* vh = A->val;
  const double* vl = val_lo;
  if (!is_device_ptr(vh)) {
    hv.alloc(sizeof(double) * nv);
    h2d(hv.p, vh, sizeof(double) * nv);
    vh = dp<double>(hv);
  }
  if (vl && !is_device_ptr(vl)) {
    lv.alloc(sizeof(double) * nv);
    h2d(lv.p, vl, sizeof(double) * nv);
    vl = dp<double>(lv);
  }
  out.rowptr.alloc(sizeof(int) * ((size_t)n + 1));   // zero-filled: rowptr[0] = 0
  int* rp = dp<int>(out.rowptr);
  const int g = dia_grid(n);
  DBuf cnt(sizeof(int) * (size_t)n);
  k_dia_count<<<g, kDiaThreads, 0, st>>>(n, nnd, vh, vl, dp<int>(dord), dp<int>(doff), dp<int>(cnt));
  PB_CUDA(cudaGetLastError());
  size_t tmp_bytes = 0;
  PB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, dp<int>(cnt), rp + 1, n, st));
  DBuf tmp(std::max<size_t>(tmp_bytes, 16));
  PB_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmp_bytes, dp<int>(cnt), rp + 1, n, st));
  int nnz = 0;
  PB_CUDA(cudaMemcpyAsync(&nnz, rp + n, sizeof(int), cudaMemcpyDeviceToHost, st));
  sync();
  PB_CHECK(nnz > 0, PARCEL_B_E_ARG, "the DIA matrix has no nonzero entry inside rows 1..n");
  out.col.alloc(sizeof(int) * (size_t)nnz);
  out.vh.alloc(sizeof(double) * (size_t)nnz);
  if (val_lo) out.vl.alloc(sizeof(double) * (size_t)nnz);
  k_dia_fill<<<g, kDiaThreads, 0, st>>>(n, nnd, A->istart, vh, vl, dp<int>(dord), dp<int>(doff), rp,
                                        dp<int>(out.col), dp<double>(out.vh),
                                        val_lo ? dp<double>(out.vl) : nullptr);
  k_add_one<<<dia_grid(n + 1), kDiaThreads, 0, st>>>((int64_t)n + 1, rp);
  PB_CUDA(cudaGetLastError());
  sync();   // the uploaded DIA arrays are released on return
  out.crs.n = n;
  out.crs.gn = n;
  out.crs.nnz = nnz;
  out.crs.istart = A->istart;
  out.crs.rowptr = rp;
  out.crs.col = dp<int>(out.col);
  out.crs.val = dp<double>(out.vh);
}

// Adds the conversion time to the statistics of the solve that followed it.
void add_setup_time(double secs) {
  parcel_b_stats s;
  if (parcel_b_last_stats(&s) != 0) return;
  s.setup_s += secs;
  s.total_s += secs;
  set_stats(s);
}

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" int parcel_b_solve_dia(const parcel_b_input* prm, const parcel_b_dia* A, const double* b, double* x,
                                  double* reshistory, int* niter, int* iret) {
  DiaCrs C;
  double t0 = 0.0, conv = 0.0;
  int rc = guarded([&]() -> int {
    ensure_init();
    t0 = now_s();
    dia_to_crs(A, nullptr, C);
    conv = now_s() - t0;
    return 0;
  });
  if (rc < 0) {
    if (iret) *iret = rc;
    if (niter) *niter = 0;
    return rc;
  }
  rc = parcel_b_solve(prm, &C.crs, b, x, reshistory, niter, iret);
  add_setup_time(conv);
  return rc;
}

extern "C" int parcel_b_ddsolve_dia(const parcel_b_input* prm, const parcel_b_dia* A, const double* val_lo,
                                    int precision_A, int precision_b, int precision_x, int precision_precondition,
                                    const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                                    double* reshistory, int* niter, int* iret) {
  DiaCrs C;
  int solver = prm && prm->solver > 0 ? prm->solver : PARCEL_B_SOLVER_CG;
  int rc = guarded([&]() -> int {
    ensure_init();
    PB_CHECK(solver == PARCEL_B_SOLVER_CG || solver == PARCEL_B_SOLVER_BICG || solver == PARCEL_B_SOLVER_GMRES,
             PARCEL_B_E_UNSUPPORTED, "solver=%d: the dd solvers are CG (1), BiCGStab (2) and GMRES (3)", solver);
    dia_to_crs(A, precision_A == 2 ? val_lo : nullptr, C);
    return 0;
  });
  if (rc < 0) {
    if (iret) *iret = rc;
    if (niter) *niter = 0;
    return rc;
  }
  auto fn = solver == PARCEL_B_SOLVER_BICG ? parcel_b_ddbicgstab
                                           : (solver == PARCEL_B_SOLVER_GMRES ? parcel_b_ddgmres : parcel_b_ddcg);
  return fn(prm, &C.crs, C.lo(), precision_A, precision_b, precision_x, precision_precondition, b_hi, b_lo, x_hi,
            x_lo, reshistory, niter, iret);
}

// ---- drop-in shims (src/example/c2fortran_kernel.f90:1228-1872), CPU-build ABI ----------
namespace {

void dia_common(parcel_b_input* p, int solver, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                int* niter, double* rtolmax, int* iovlflag, int* precon_thblock, int* neuman_itr,
                int* independ_nvec, int* nblock) {
  parcel_b_input_init(p);
  p->solver = solver;
  p->ipreflag = *ipreflag;
  p->ILU_method = *ilu_method;
  p->addL = *addl;
  p->iflagAS = *iflagas;
  p->itrmax = *niter;
  p->rtolmax = *rtolmax;
  p->abstolmax = 0.0;
  p->iovlflag = *iovlflag;
  p->precon_thblock = *precon_thblock;
  if (neuman_itr) p->Neuman_itr = *neuman_itr;
  p->independ_nvec = *independ_nvec;
  p->nBlock = *nblock;
}

void dia_run(parcel_b_input* p, int32_t* n, int32_t* gn, int32_t* istart, double* diaA, int32_t* offset,
             int32_t* nnd, double* vecb, double* vecx, double* reshistory, int* niter, int* iret) {
  parcel_b_dia A;
  A.n = *n; A.gn = *gn; A.istart = *istart; A.nnd = *nnd;
  A.val = diaA; A.offset = offset;
  int used = 0, ir = 0;
  parcel_b_solve_dia(p, &A, vecb, vecx, reshistory, &used, &ir);
  *niter = used;
  *iret = ir;
}

void dd_dia_run(parcel_b_input* p, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset, int32_t* nnd,
                double* reshistory, int* pa, int* pb, int* px, int* pm, int* niter, int* iret) {
  parcel_b_dia A;
  A.n = *n; A.gn = *gn; A.istart = *istart; A.nnd = *nnd;
  A.val = diaA; A.offset = offset;
  int used = 0, ir = 0;
  parcel_b_ddsolve_dia(p, &A, diaA_lo, *pa, *pb, *px, *pm, vecb, vecb_lo, vecx, vecx_lo, reshistory, &used, &ir);
  *niter = used;
  *iret = ir;
}

}  // namespace

extern "C" {

void parcel_dcg_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                       double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                       int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                       int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_CG, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  dia_run(&p, n, gn, istart, diaA, offset, nnd, vecb, vecx, reshistory, niter, iret);
}

void parcel_dbicgstab_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                             double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                             int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                             int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_BICG, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag,
             precon_thblock, neuman_itr, independ_nvec, nblock);
  dia_run(&p, n, gn, istart, diaA, offset, nnd, vecb, vecx, reshistory, niter, iret);
}

void parcel_dgmres_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                          double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                          int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                          int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* restart,
                          int* gmres_gsflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_GMRES, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag,
             precon_thblock, neuman_itr, independ_nvec, nblock);
  p.GMRES_m = *restart;
  p.GMRES_GSflag = *gmres_gsflag;
  dia_run(&p, n, gn, istart, diaA, offset, nnd, vecb, vecx, reshistory, niter, iret);
}

void parcel_dcagmres_dia_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* istart,
                            double* diaA, int32_t* offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                            int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                            int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                            int* cagmres_sstep, int* cagmres_tstep, int* cagmres_basis, int* cagmres_qrflag,
                            int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_CAGMRES, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag,
             precon_thblock, neuman_itr, independ_nvec, nblock);
  p.CAGMRES_sstep = *cagmres_sstep;
  p.CAGMRES_tstep = *cagmres_tstep;
  p.CAGMRES_basis = *cagmres_basis;
  p.CAGMRES_QRflag = *cagmres_qrflag;
  dia_run(&p, n, gn, istart, diaA, offset, nnd, vecb, vecx, reshistory, niter, iret);
}

void parcel_ddcg_dia_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                        int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset, int32_t* nnd,
                        int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                        double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                        int* independ_nvec, int* nblock, int* precision_a, int* precision_b, int* precision_x,
                        int* precision_precondition, int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_CG, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  dd_dia_run(&p, vecx, vecx_lo, vecb, vecb_lo, n, gn, istart, diaA, diaA_lo, offset, nnd, reshistory, precision_a,
             precision_b, precision_x, precision_precondition, niter, iret);
}

void parcel_ddbicgstab_dia_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                              int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset,
                              int32_t* nnd, int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter,
                              double* rtolmax, double* reshistory, int* iovlflag, int* precon_thblock,
                              int* neuman_itr, int* independ_nvec, int* nblock, int* precision_a, int* precision_b,
                              int* precision_x, int* precision_precondition, int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_BICG, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag,
             precon_thblock, neuman_itr, independ_nvec, nblock);
  dd_dia_run(&p, vecx, vecx_lo, vecb, vecb_lo, n, gn, istart, diaA, diaA_lo, offset, nnd, reshistory, precision_a,
             precision_b, precision_x, precision_precondition, niter, iret);
}

// parcel_ddgmres_dia_c has no Neuman_itr argument (c2fortran_kernel.f90:1681-1773).
void parcel_ddgmres_dia_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                           int32_t* gn, int32_t* istart, double* diaA, double* diaA_lo, int32_t* offset,
                           int32_t* nnd, int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter,
                           double* rtolmax, double* reshistory, int* iovlflag, int* precon_thblock,
                           int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag, int* precision_a,
                           int* precision_b, int* precision_x, int* precision_precondition, int* iret) {
  (void)icomm;
  parcel_b_input p;
  dia_common(&p, PARCEL_B_SOLVER_GMRES, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag,
             precon_thblock, nullptr, independ_nvec, nblock);
  p.GMRES_m = *restart;
  p.GMRES_GSflag = *gmres_gsflag;
  dd_dia_run(&p, vecx, vecx_lo, vecb, vecb_lo, n, gn, istart, diaA, diaA_lo, offset, nnd, reshistory, precision_a,
             precision_b, precision_x, precision_precondition, niter, iret);
}

// CUDA-build ABI: vecx, vecb, diaA and offset are device pointers passed by reference
// (type(c_ptr) arguments of the CUDA_SOLVER build of the same shims).
void parcel_dcg_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                           void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                           int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                           int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* iret) {
  parcel_dcg_dia_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, istart, (double*)*diaA, (int32_t*)*offset, nnd,
                    ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, precon_thblock,
                    neuman_itr, independ_nvec, nblock, iret);
}

void parcel_dbicgstab_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                                 void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method,
                                 int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                                 int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                                 int* nblock, int* iret) {
  parcel_dbicgstab_dia_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, istart, (double*)*diaA, (int32_t*)*offset,
                          nnd, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag,
                          precon_thblock, neuman_itr, independ_nvec, nblock, iret);
}

void parcel_dgmres_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                              void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method, int* addl,
                              int* iflagas, int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                              int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock, int* restart,
                              int* gmres_gsflag, int* iret) {
  parcel_dgmres_dia_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, istart, (double*)*diaA, (int32_t*)*offset,
                       nnd, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag,
                       precon_thblock, neuman_itr, independ_nvec, nblock, restart, gmres_gsflag, iret);
}

void parcel_dcagmres_dia_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* istart,
                                void** diaA, void** offset, int32_t* nnd, int* ipreflag, int* ilu_method,
                                int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                                int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                                int* nblock, int* cagmres_sstep, int* cagmres_tstep, int* cagmres_basis,
                                int* cagmres_qrflag, int* iret) {
  parcel_dcagmres_dia_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, istart, (double*)*diaA, (int32_t*)*offset,
                         nnd, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag,
                         precon_thblock, neuman_itr, independ_nvec, nblock, cagmres_sstep, cagmres_tstep,
                         cagmres_basis, cagmres_qrflag, iret);
}

}  // extern "C"
