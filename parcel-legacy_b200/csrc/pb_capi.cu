// pb_capi.cu -- the C ABI of libparcelb (declared in include/parcel_b.h).
//
// Mirrors the reference's entry points: PARCEL_KSP_CRS (src/wrapper.f90:47-222), the
// parcel_d{cg,bicgstab,gmres,cagmres} wrappers (wrapper.f90:362-1455 GPU build,
// 1813-2900 CPU build) and their C-callable forms (src/example/c2fortran_kernel.f90).
// Like KSP_CRS (src/krylov.f90:447-735) every call is self-contained: it copies what it
// needs, solves, writes x and reshistory back and frees its memory.  Errors come back as
// status codes instead of `stop`.
#include <cmath>
#include <memory>
#include <mutex>

#include "pb_api.cuh"

namespace pb {

namespace {
std::mutex g_stats_mu;
parcel_b_stats g_stats;
}  // namespace

void set_stats(const parcel_b_stats& s) {
  std::lock_guard<std::mutex> lk(g_stats_mu);
  g_stats = s;
}

void validate(const parcel_b_crs* A) {
  PB_CHECK(A != nullptr, PARCEL_B_E_ARG, "matrix is NULL");
  PB_CHECK(A->n > 0, PARCEL_B_E_ARG, "n = %d", A->n);
  PB_CHECK(A->nnz >= 0 && A->nnz < (int64_t)INT32_MAX, PARCEL_B_E_ARG, "nnz = %lld out of int32 range",
           (long long)A->nnz);
  PB_CHECK(A->rowptr && A->col && A->val, PARCEL_B_E_ARG, "CRS arrays must not be NULL");
  PB_CHECK(A->gn <= 0 || A->gn == A->n, PARCEL_B_E_UNSUPPORTED,
           "n=%d != gn=%d: a matrix split over processes needs the MPI halo exchange, "
           "which this single-GPU build does not provide", A->n, A->gn);
  PB_CHECK(A->istart == 1, PARCEL_B_E_UNSUPPORTED,
           "istart=%d: one process owns rows 1..n", A->istart);
}

// Deterministic dot of two device vectors, result on the host.
template <class T>
double dev_dot(int64_t n, const T* x, const T* y) {
  Workspace W;
  W.init();
  DBuf out(sizeof(double));
  Red rr = W.red(EPI_STORE);
  rr.ea.out = dp<double>(out);
  DotSel sel;
  sel.a[0] = 1; sel.b[0] = 2;
  lincomb_dot<T>(n, nullptr, x, cimm(0), y, cimm(0), nullptr, cimm(0), nullptr, nullptr, sel, 1, rr,
                 nullptr, stream());
  double h;
  d2h(&h, out.p, sizeof(double));
  return h;
}
template double dev_dot<double>(int64_t, const double*, const double*);
template double dev_dot<float>(int64_t, const float*, const float*);

// ||b - A x|| / ||b|| in FP64, natural layout, device arrays.
double true_relres(const DevMat<double>& A, const double* b, const double* x) {
  DBuf r(sizeof(double) * A.n);
  spmv<double, double>(A, x, dp<double>(r), SPMV_RES, b, nullptr, stream());
  double rr = dev_dot<double>(A.n, dp<double>(r), dp<double>(r));
  double bb = dev_dot<double>(A.n, b, b);
  return std::sqrt(rr) / std::sqrt(bb);
}

// One FP64 solve on a built system.  b, x natural-layout device arrays; x in/out.
SolveOut solve_on_system(const Options& o, System<double>& S, const double* b_dev, double* x_dev,
                         std::vector<double>& hist_out, double* setup_t) {
  cudaStream_t st = stream();
  const int np = S.np;
  DBuf bb, xb;
  const double* bi = b_dev;
  double* xi = x_dev;
  if (S.permuted) {
    bb.alloc(sizeof(double) * np);
    xb.alloc(sizeof(double) * np);
    PB_CUDA(cudaMemsetAsync(bb.p, 0, sizeof(double) * np, st));
    PB_CUDA(cudaMemsetAsync(xb.p, 0, sizeof(double) * np, st));
    scatter_perm<double>(S.n, dp<double>(bb), b_dev, dp<int>(S.pos), st);
    scatter_perm<double>(S.n, dp<double>(xb), x_dev, dp<int>(S.pos), st);
    bi = dp<double>(bb);
    xi = dp<double>(xb);
  }
  DBuf hist(sizeof(double) * (o.itrmax + 2));
  PB_CUDA(cudaMemsetAsync(hist.p, 0, sizeof(double) * (o.itrmax + 2), st));
  sync();
  if (setup_t) *setup_t = now_s();
  SolveOut so = run_krylov<double>(o, S, bi, xi, dp<double>(hist));
  if (S.permuted) gather_perm<double>(S.n, x_dev, xi, dp<int>(S.pos), st);
  hist_out.assign(std::max(so.niter, 0), 0.0);
  if (so.niter > 0) d2h(hist_out.data(), hist.p, sizeof(double) * so.niter);
  sync();
  return so;
}

struct Handle {
  Options o;
  parcel_b_crs A;
  bool dev = false;
  std::unique_ptr<System<double>> S;
};

}  // namespace pb

using namespace pb;

extern "C" {

void parcel_b_input_init(parcel_b_input* p) {
  if (!p) return;
  int* ip = reinterpret_cast<int*>(p);
  (void)ip;
  p->ipreflag = p->ILU_method = p->addL = p->iflagAS = p->solver = p->iovlflag = -1;
  p->GMRES_m = p->GMRES_GSflag = -1;
  p->CAGMRES_sstep = p->CAGMRES_tstep = p->CAGMRES_basis = p->CAGMRES_QRflag = -1;
  p->CBCG_kstep = p->CBCG_Eigenflag = p->power_method_itrmax = -1;
  p->CAARNOLDI_sstep = p->CAARNOLDI_tstep = p->CAARNOLDI_basis = p->CAARNOLDI_QRflag = -1;
  p->machineflag = p->dataflag = p->calcflag = -1;
  p->Neuman_itr = p->Neuman_local = -1;
  p->itrmax = -1;
  p->rtolmax = -1.0;
  p->abstolmax = -1.0;
  p->independ_nvec = p->precon_thblock = p->nBlock = -1;
  p->PRECISION_A = p->PRECISION_b = p->PRECISION_x = p->PRECISION_PRECONDITION = -1;
  p->inner_precision = 0;
  p->residual_dd = 0;
  p->inner_rtol = -1.0;
  p->max_refine = -1;
  for (int i = 0; i < 7; ++i) p->reserved[i] = 0;
}

int parcel_b_last_stats(parcel_b_stats* out) {
  if (!out) return PARCEL_B_E_ARG;
  std::lock_guard<std::mutex> lk(g_stats_mu);
  *out = g_stats;
  return 0;
}

int parcel_b_solve(const parcel_b_input* prm, const parcel_b_crs* A, const double* b, double* x,
                   double* reshistory, int* niter, int* iret) {
  int rc = guarded([&]() -> int {
    ensure_init();
    validate(A);
    PB_CHECK(b && x, PARCEL_B_E_ARG, "b and x must not be NULL");
    Options o = resolve_options(prm);
    PB_CHECK(o.independ_nvec == 1, PARCEL_B_E_UNSUPPORTED,
             "independ_nvec=%d: only 1 (the reference default) is provided", o.independ_nvec);
    PB_CHECK(o.precon >= 0 && o.precon <= 2, PARCEL_B_E_UNSUPPORTED,
             "ipreflag=%d (Neumann series) is not provided by this build", o.precon);
    const double t0 = now_s();
    const bool dev = is_device_ptr(A->val);
    const bool bdev = is_device_ptr(b), xdev = is_device_ptr(x);
    parcel_b_stats stt;
    memset(&stt, 0, sizeof(stt));
    NatVec bv(b, A->n, bdev), xv(x, A->n, xdev);
    std::vector<double> hist;
    SolveOut so;
    double t1 = t0;
    if (o.solver == PARCEL_B_SOLVER_CAGMRES) {
      System<double> S;
      build_system<double>(o, *A, dev, S);
      so = solve_cagmres(o, S, bv.p, xv.p, hist, &t1);
      stt.ilu_levels_max = S.ilu_levels_max;
      stt.ilu_nblocks = S.ilu_nblocks;
      stt.spmv_diagonals = S.spmv_diagonals;
      stt.true_relres = true_relres(S.Anat, bv.p, xv.p);
    } else if (o.inner == PARCEL_B_INNER_FP32_REFINE) {
      MixedResult mr = solve_mixed(o, *A, dev, bv.p, xv.p, hist, &t1);
      so.niter = mr.niter;
      so.iret = mr.iret;
      so.launches = mr.launches;
      stt.refine_steps = mr.refine_steps;
      stt.true_relres = mr.true_relres;
      stt.true_relres_dd = mr.true_relres_dd;
      stt.ilu_levels_max = mr.ilu_levels_max;
      stt.ilu_nblocks = mr.ilu_nblocks;
    } else {
      System<double> S;
      build_system<double>(o, *A, dev, S);
      so = solve_on_system(o, S, bv.p, xv.p, hist, &t1);
      stt.ilu_levels_max = S.ilu_levels_max;
      stt.ilu_nblocks = S.ilu_nblocks;
      stt.spmv_diagonals = S.spmv_diagonals;
      stt.true_relres = true_relres(S.Anat, bv.p, xv.p);
    }
    const double t2 = now_s();
    if (!xdev) d2h(x, xv.p, sizeof(double) * A->n);
    if (reshistory && !hist.empty()) {
      size_t cnt = std::min<size_t>(hist.size(), (size_t)std::max(o.itrmax, 0));
      if (is_device_ptr(reshistory)) { h2d(reshistory, hist.data(), sizeof(double) * cnt); sync(); }
      else memcpy(reshistory, hist.data(), sizeof(double) * cnt);
    }
    if (niter) *niter = so.niter;
    if (iret) *iret = so.iret;
    stt.setup_s = t1 - t0;
    stt.solve_s = t2 - t1;
    stt.total_s = now_s() - t0;
    stt.niter = so.niter;
    stt.iret = so.iret;
    stt.kernel_launches = so.launches;
    set_stats(stt);
    return so.iret < 0 ? so.iret : 0;
  });
  if (rc < 0 && iret) *iret = rc;
  return rc;
}

// ---- drop-in shims ----------------------------------------------------------------
static void fill_common(parcel_b_input* p, int solver, int* ipreflag, int* ilu_method, int* addl,
                        int* iflagas, int* niter, double* rtolmax, int* iovlflag, int* precon_thblock,
                        int* neuman_itr, int* independ_nvec, int* nblock) {
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
  p->Neuman_itr = *neuman_itr;
  p->independ_nvec = *independ_nvec;
  p->nBlock = *nblock;
}

static void run_shim(parcel_b_input* p, int32_t* n, int32_t* gn, int32_t* nnz, int32_t* istart,
                     const double* crsa, const int32_t* rp, const int32_t* ci, const double* b,
                     double* x, double* hist, int* niter, int* iret) {
  parcel_b_crs A;
  A.n = *n; A.gn = *gn; A.nnz = *nnz; A.istart = *istart;
  A.rowptr = rp; A.col = ci; A.val = crsa;
  int used = 0, ir = 0;
  parcel_b_solve(p, &A, b, x, hist, &used, &ir);
  *niter = used;
  *iret = ir;
}

void parcel_dcg_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn, int32_t* nnz,
                   int32_t* istart, double* crsa, int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag,
                   int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                   double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                   int* independ_nvec, int* nblock, int* iret) {
  (void)icomm;
  parcel_b_input p;
  fill_common(&p, PARCEL_B_SOLVER_CG, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, iovlflag,
              precon_thblock, neuman_itr, independ_nvec, nblock);
  run_shim(&p, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, vecb, vecx, reshistory, niter, iret);
}

void parcel_dbicgstab_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                         int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                         int32_t* crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                         int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                         int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                         int* iret) {
  (void)icomm;
  parcel_b_input p;
  fill_common(&p, PARCEL_B_SOLVER_BICG, ipreflag, ilu_method, addl, iflagas, niter, rtolmax,
              iovlflag, precon_thblock, neuman_itr, independ_nvec, nblock);
  run_shim(&p, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, vecb, vecx, reshistory, niter, iret);
}

void parcel_dgmres_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                      int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                      int32_t* crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                      int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                      int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                      int* restart, int* gmres_gsflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  fill_common(&p, PARCEL_B_SOLVER_GMRES, ipreflag, ilu_method, addl, iflagas, niter, rtolmax,
              iovlflag, precon_thblock, neuman_itr, independ_nvec, nblock);
  p.GMRES_m = *restart;
  p.GMRES_GSflag = *gmres_gsflag;
  run_shim(&p, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, vecb, vecx, reshistory, niter, iret);
}

void parcel_dcagmres_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int32_t* gn,
                        int32_t* nnz, int32_t* istart, double* crsa, int32_t* crsrow_ptr,
                        int32_t* crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                        int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                        int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                        int* cagmres_sstep, int* cagmres_tstep, int* cagmres_basis,
                        int* cagmres_qrflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  fill_common(&p, PARCEL_B_SOLVER_CAGMRES, ipreflag, ilu_method, addl, iflagas, niter, rtolmax,
              iovlflag, precon_thblock, neuman_itr, independ_nvec, nblock);
  p.CAGMRES_sstep = *cagmres_sstep;
  p.CAGMRES_tstep = *cagmres_tstep;
  p.CAGMRES_basis = *cagmres_basis;
  p.CAGMRES_QRflag = *cagmres_qrflag;
  run_shim(&p, n, gn, nnz, istart, crsa, crsrow_ptr, crscol, vecb, vecx, reshistory, niter, iret);
}

void parcel_dcg_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn, int32_t* nnz,
                       int32_t* istart, void** crsa, void** crsrow_ptr, void** crscol, int* ipreflag,
                       int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                       double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                       int* independ_nvec, int* nblock, int* iret) {
  parcel_dcg_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, nnz, istart, (double*)*crsa,
                (int32_t*)*crsrow_ptr, (int32_t*)*crscol, ipreflag, ilu_method, addl, iflagas, niter,
                rtolmax, reshistory, iovlflag, precon_thblock, neuman_itr, independ_nvec, nblock, iret);
}

void parcel_dbicgstab_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                             int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                             void** crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                             int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                             int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                             int* iret) {
  parcel_dbicgstab_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, nnz, istart, (double*)*crsa,
                      (int32_t*)*crsrow_ptr, (int32_t*)*crscol, ipreflag, ilu_method, addl, iflagas,
                      niter, rtolmax, reshistory, iovlflag, precon_thblock, neuman_itr,
                      independ_nvec, nblock, iret);
}

void parcel_dgmres_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                          int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                          void** crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                          int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                          int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                          int* restart, int* gmres_gsflag, int* iret) {
  parcel_dgmres_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, nnz, istart, (double*)*crsa,
                   (int32_t*)*crsrow_ptr, (int32_t*)*crscol, ipreflag, ilu_method, addl, iflagas, niter,
                   rtolmax, reshistory, iovlflag, precon_thblock, neuman_itr, independ_nvec, nblock,
                   restart, gmres_gsflag, iret);
}

void parcel_dcagmres_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int32_t* gn,
                            int32_t* nnz, int32_t* istart, void** crsa, void** crsrow_ptr,
                            void** crscol, int* ipreflag, int* ilu_method, int* addl, int* iflagas,
                            int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                            int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                            int* cagmres_sstep, int* cagmres_tstep, int* cagmres_basis,
                            int* cagmres_qrflag, int* iret) {
  parcel_dcagmres_c_(icomm, (double*)*vecx, (double*)*vecb, n, gn, nnz, istart, (double*)*crsa,
                     (int32_t*)*crsrow_ptr, (int32_t*)*crscol, ipreflag, ilu_method, addl, iflagas,
                     niter, rtolmax, reshistory, iovlflag, precon_thblock, neuman_itr, independ_nvec,
                     nblock, cagmres_sstep, cagmres_tstep, cagmres_basis, cagmres_qrflag, iret);
}

// ---- split setup / solve ----------------------------------------------------------
struct parcel_b_handle_s {
  pb::Handle h;
};

int parcel_b_setup(const parcel_b_input* prm, const parcel_b_crs* A, parcel_b_handle* out) {
  return guarded([&]() -> int {
    ensure_init();
    validate(A);
    PB_CHECK(out != nullptr, PARCEL_B_E_ARG, "handle pointer is NULL");
    auto* H = new parcel_b_handle_s();
    H->h.o = resolve_options(prm);
    PB_CHECK(H->h.o.inner == PARCEL_B_INNER_FP64 && H->h.o.solver != PARCEL_B_SOLVER_CAGMRES,
             PARCEL_B_E_UNSUPPORTED, "the split API runs the FP64 CG / BiCGStab / GMRES solvers");
    H->h.A = *A;
    H->h.dev = is_device_ptr(A->val);
    H->h.S.reset(new System<double>());
    try {
      build_system<double>(H->h.o, *A, H->h.dev, *H->h.S);
    } catch (...) {
      delete H;
      throw;
    }
    sync();
    *out = H;
    return 0;
  });
}

int parcel_b_start(parcel_b_handle h, const double* b, double* x, double* reshistory, int* niter,
                   int* iret) {
  int rc = guarded([&]() -> int {
    PB_CHECK(h != nullptr, PARCEL_B_E_ARG, "handle is NULL");
    const Options& o = h->h.o;
    const int n = h->h.A.n;
    const double t0 = now_s();
    const bool xdev = is_device_ptr(x);
    NatVec bv(b, n, is_device_ptr(b)), xv(x, n, xdev);
    std::vector<double> hist;
    double t1 = t0;
    SolveOut so = solve_on_system(o, *h->h.S, bv.p, xv.p, hist, &t1);
    const double t2 = now_s();
    if (!xdev) d2h(x, xv.p, sizeof(double) * n);
    if (reshistory && !hist.empty()) {
      size_t cnt = std::min<size_t>(hist.size(), (size_t)o.itrmax);
      if (is_device_ptr(reshistory)) { h2d(reshistory, hist.data(), sizeof(double) * cnt); sync(); }
      else memcpy(reshistory, hist.data(), sizeof(double) * cnt);
    }
    if (niter) *niter = so.niter;
    if (iret) *iret = so.iret;
    parcel_b_stats stt;
    memset(&stt, 0, sizeof(stt));
    stt.setup_s = t1 - t0;
    stt.solve_s = t2 - t1;
    stt.total_s = now_s() - t0;
    stt.niter = so.niter;
    stt.iret = so.iret;
    stt.kernel_launches = so.launches;
    stt.ilu_levels_max = h->h.S->ilu_levels_max;
    stt.ilu_nblocks = h->h.S->ilu_nblocks;
    stt.spmv_diagonals = h->h.S->spmv_diagonals;
    set_stats(stt);
    return so.iret < 0 ? so.iret : 0;
  });
  if (rc < 0 && iret) *iret = rc;
  return rc;
}

int parcel_b_release(parcel_b_handle h) {
  return guarded([&]() -> int {
    if (h) { sync(); delete h; }
    return 0;
  });
}

// ---- kernel-level entries ----------------------------------------------------------
int parcel_b_spmv(const parcel_b_crs* A, const double* x, double* y) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(A && x && y, PARCEL_B_E_ARG, "NULL argument");
    DevMat<double> M;
    M.n = A->n; M.nnz = A->nnz; M.rowptr = A->rowptr; M.col = A->col; M.val = A->val;
    M.rbase = 1; M.cbase = A->istart;
    spmv<double, double>(M, x, y, SPMV_Y, nullptr, nullptr, stream());
    sync();
    return 0;
  });
}

int parcel_b_spmv_f32(int32_t n, int64_t nnz, int32_t istart, const int32_t* rowptr, const int32_t* col,
                      const float* val, const float* x, float* y) {
  return guarded([&]() -> int {
    ensure_init();
    DevMat<float> M;
    M.n = n; M.nnz = nnz; M.rowptr = rowptr; M.col = col; M.val = val; M.rbase = 1; M.cbase = istart;
    spmv<float, float>(M, x, y, SPMV_Y, nullptr, nullptr, stream());
    sync();
    return 0;
  });
}

int parcel_b_precon_apply(const parcel_b_input* prm, const parcel_b_crs* A, const double* r, double* s) {
  return guarded([&]() -> int {
    ensure_init();
    validate(A);
    Options o = resolve_options(prm);
    PB_CHECK(o.precon >= 0 && o.precon <= 2, PARCEL_B_E_UNSUPPORTED, "ipreflag=%d", o.precon);
    const bool dev = is_device_ptr(A->val);
    System<double> S;
    build_system<double>(o, *A, dev, S);
    const int n = A->n;
    const bool sdev = is_device_ptr(s);
    NatVec rv(r, n, is_device_ptr(r));
    DBuf sown;
    double* sp = s;
    if (!sdev) { sown.alloc(sizeof(double) * n); sp = dp<double>(sown); }
    cudaStream_t st = stream();
    if (S.permuted) {
      DBuf rp(sizeof(double) * S.np), spp(sizeof(double) * S.np);
      PB_CUDA(cudaMemsetAsync(rp.p, 0, sizeof(double) * S.np, st));
      scatter_perm<double>(n, dp<double>(rp), rv.p, dp<int>(S.pos), st);
      S.M.apply(S.np, dp<double>(rp), dp<double>(spp), nullptr, st);
      gather_perm<double>(n, sp, dp<double>(spp), dp<int>(S.pos), st);
      sync();
    } else {
      S.M.apply(n, rv.p, sp, nullptr, st);
    }
    int err = 0;
    if (S.permuted) d2h(&err, S.M.ilu.err.p, sizeof(int));
    PB_CHECK(err == 0, PARCEL_B_E_CUDA, "ILU sweep kernel reported wait timeout %d", err);
    if (!sdev) d2h(s, sp, sizeof(double) * n);
    sync();
    return 0;
  });
}

int parcel_b_dot(int64_t n, const double* x, const double* y, double* out_host) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(out_host, PARCEL_B_E_ARG, "NULL output");
    *out_host = dev_dot<double>(n, x, y);
    return 0;
  });
}

int parcel_b_residual_dd(const parcel_b_crs* A, const double* x_hi, const double* x_lo,
                         const double* b_hi, const double* b_lo, double* r_hi, double* r_lo) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(A && x_hi && b_hi && r_hi && r_lo, PARCEL_B_E_ARG, "NULL argument");
    DevMat<double> M;
    M.n = A->n; M.nnz = A->nnz; M.rowptr = A->rowptr; M.col = A->col; M.val = A->val;
    M.rbase = 1; M.cbase = A->istart;
    residual_dd(M, nullptr, x_hi, x_lo, b_hi, b_lo, r_hi, r_lo, stream());
    sync();
    return 0;
  });
}

int parcel_b_bench_kernels(const parcel_b_input* prm, const parcel_b_crs* A, int reps, double* ms_spmv,
                           double* ms_precon) {
  return guarded([&]() -> int {
    ensure_init();
    validate(A);
    PB_CHECK(reps > 0 && ms_spmv && ms_precon, PARCEL_B_E_ARG, "bad arguments");
    Options o = resolve_options(prm);
    auto run = [&](auto tag) {
      using T = decltype(tag);
      System<T> S;
      build_system<T>(o, *A, is_device_ptr(A->val), S);
      cudaStream_t st = stream();
      const int np = S.np;
      DBuf x(sizeof(T) * np), y(sizeof(T) * np);
      if constexpr (sizeof(T) == sizeof(double)) {
        fill(np, dp<double>(x), 1.0, st);
      } else {
        DBuf one(sizeof(double) * np);
        fill(np, dp<double>(one), 1.0, st);
        convert<T, double>(np, dp<T>(x), dp<double>(one), st);
      }
      PB_CUDA(cudaMemsetAsync(y.p, 0, sizeof(T) * np, st));
      cudaEvent_t e0, e1;
      PB_CUDA(cudaEventCreate(&e0));
      PB_CUDA(cudaEventCreate(&e1));
      for (int i = 0; i < 3; ++i) spmv<T, T>(S.A, dp<T>(x), dp<T>(y), SPMV_Y, nullptr, nullptr, st);
      PB_CUDA(cudaEventRecord(e0, st));
      for (int i = 0; i < reps; ++i) spmv<T, T>(S.A, dp<T>(x), dp<T>(y), SPMV_Y, nullptr, nullptr, st);
      PB_CUDA(cudaEventRecord(e1, st));
      PB_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      PB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      *ms_spmv = ms / reps;
      for (int i = 0; i < 3; ++i) S.M.apply(np, dp<T>(y), dp<T>(x), nullptr, st);
      PB_CUDA(cudaEventRecord(e0, st));
      for (int i = 0; i < reps; ++i) S.M.apply(np, dp<T>(y), dp<T>(x), nullptr, st);
      PB_CUDA(cudaEventRecord(e1, st));
      PB_CUDA(cudaEventSynchronize(e1));
      PB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      *ms_precon = ms / reps;
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
    };
    // inner_precision = 1 times the FP32 system of the mixed-precision path
    if (o.inner == PARCEL_B_INNER_FP32_REFINE) run(float(0)); else run(double(0));
    return 0;
  });
}

}  // extern "C"
