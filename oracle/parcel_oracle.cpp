// parcel_oracle.cpp -- CPU oracle for the PARCEL-legacy preconditioned Krylov path.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, in plain C++/OpenMP, the reference's
// CPU algorithms for the single-process CRS solve so that the GPU library can be checked
// against it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// it.  The product library (libparcelb.so) never links or calls it.
//
// Parity is pinned against the reference's own stored output
// (src/example/template_cpu/STDOUT_run: CG + block-Jacobi D-ILU, 80 blocks, 160^3 Poisson,
// 291 iterations) by tests/test_oracle_golden.py.
//
// Conventions follow the reference: CRS arrays are 1-based with global column ids
// (crsRow_ptr(1) = 1), values real*8, indices int32 (define.f90:133-164).  One process,
// so istart = 1 and n = gn unless the caller says otherwise; columns outside
// [istart, istart+n-1] are halo columns, which a single process never has.
//
// Reductions: the reference uses OpenMP REDUCTION clauses followed by MPI_Allreduce
// (vec.f90:1027-1048), whose summation order depends on the thread count.  The oracle
// uses a fixed chunked order (ORC_NCHUNK chunks, summed in chunk order) so that its
// results do not depend on the number of threads it runs on.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// ---------------------------------------------------------------------------------
// Constants mirrored from src/define.f90:14-102.
enum {
  ORC_SOLVER_CG = 1, ORC_SOLVER_BICG = 2, ORC_SOLVER_GMRES = 3, ORC_SOLVER_CAGMRES = 4,
  ORC_PRECON_NONE = 0, ORC_PRECON_PJ = 1, ORC_PRECON_BJ = 2, ORC_PRECON_AS = 3,
  ORC_ILU0 = 0, ORC_ILUD = 1, ORC_MLUD = 2,
  ORC_GS_MGS = 1, ORC_GS_CGS = 2,
};
// Status codes: 0 normal, 1 max iterations (define.f90:101-102); negative = error that the
// reference handles with `stop` (matrix.f90:8018-8021, 3540-3543).
enum { ORC_E_ZERO_PIVOT = -1, ORC_E_ARG = -2, ORC_E_UNSUPPORTED = -5 };

struct OrcMat {           // one process's rows of a CRS matrix, reference layout
  int n;                  // local rows
  int nnz;
  int istart;             // 1-based global id of the first local row
  const int* rowptr;      // n+1, 1-based
  const int* col;         // nnz, 1-based global columns
  const double* val;      // nnz
};

struct OrcParams {        // subset of KSP_INPUT_PARAM (type.f90:907-946)
  int solver;
  int ipreflag;
  int ILU_method;
  int precon_thblock;     // number of block-Jacobi blocks (the reference ties it to threads)
  int itrmax;
  double rtolmax;
  int GMRES_m;
  int GMRES_GSflag;
  int CAGMRES_sstep;
  int CAGMRES_tstep;
  int CAGMRES_basis;
  int CAGMRES_QRflag;
};

}  // extern "C"

namespace {

constexpr int ORC_NCHUNK = 256;

// divide_region (common.f90:125-182): contiguous split of [idown, iup] into np parts,
// the first mod(len, np) parts one row longer.  Returns 1-based inclusive bounds.
void divide_region(int r, int np, long idown, long iup, long* lo, long* hi) {
  if (iup == idown) { *lo = idown; *hi = iup; return; }
  long region = iup - idown + 1;
  long blk = region / np;
  long over = region % np;
  if (r < over) { *lo = idown + blk * r + r; *hi = *lo + blk; }
  else { *lo = idown + blk * r + over; *hi = *lo + blk - 1; }
}

// Deterministic dot: fixed chunk order, independent of thread count.
template <class F>
double chunked_sum(long n, F term) {
  double part[ORC_NCHUNK];
  long nch = std::min<long>(ORC_NCHUNK, std::max<long>(1, n));
#pragma omp parallel for schedule(static)
  for (long c = 0; c < nch; ++c) {
    long lo = n * c / nch, hi = n * (c + 1) / nch;
    double s = 0.0;
    for (long i = lo; i < hi; ++i) s += term(i);
    part[c] = s;
  }
  double s = 0.0;
  for (long c = 0; c < nch; ++c) s += part[c];
  return s;
}

double dot(long n, const double* x, const double* y) {
  return chunked_sum(n, [&](long i) { return x[i] * y[i]; });
}

// MatVec_crs (matrix.f90:1348-1512), single process: y(i) = sum_j a_ij x(col_j - istart + 1).
void spmv(const OrcMat& A, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < A.n; ++i) {
    double t = 0.0;
    for (long j = A.rowptr[i] - 1; j < A.rowptr[i + 1] - 1; ++j)
      t += A.val[j] * x[A.col[j] - A.istart];
    y[i] = t;
  }
}

// calc_res: r = b - A x
void residual(const OrcMat& A, const double* x, const double* b, double* r) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < A.n; ++i) {
    double t = 0.0;
    for (long j = A.rowptr[i] - 1; j < A.rowptr[i + 1] - 1; ++j)
      t += A.val[j] * x[A.col[j] - A.istart];
    r[i] = b[i] - t;
  }
}

// ---------------------------------------------------------------------------------
// Preconditioners.
struct IluBlock {          // ILU(0) factors of one block-Jacobi block (matrix.f90:7821-8072)
  long r0, r1;             // 0-based local rows [r0, r1)
  std::vector<int> Lp, Lc; std::vector<double> Lv;   // L incl. unit diagonal stored last
  std::vector<int> Up, Uc; std::vector<double> Uv;   // U with diagonal stored first
};

struct DiluBlock {         // D-ILU ranges of one block (matrix.f90:5165-5412)
  long r0, r1;
  std::vector<long> Ls, Le, Us, Ue;  // 0-based nnz ranges, U scanned from Us down to Ue
};

struct Precon {
  int kind = ORC_PRECON_NONE;
  int ilu_method = ORC_ILU0;
  std::vector<double> Dinv;          // point Jacobi or D-ILU inverse diagonal
  std::vector<IluBlock> ilu;
  std::vector<DiluBlock> dilu;
  const OrcMat* A = nullptr;
};

// Explicit block boundaries (0-based row starts followed by n), set by orc_set_blocks for
// the stencil-format (DDM) solves, whose blocks are the boxes of a geometric split laid out
// one after another; empty: divide_region's equal split.
std::vector<long> g_blk;

int nblocks_for(const OrcMat& A, int thblock) {
  if (!g_blk.empty()) return (int)g_blk.size() - 1;
  // The reference uses one block per OpenMP thread, capped by precon_thblock
  // (common.f90:89-123).  The oracle takes the block count explicitly; <= 0 means one
  // block, which is what the reference GPU build computes per process (cusparse.cu:17-197).
  int nb = thblock > 0 ? thblock : 1;
  if (nb > A.n) nb = A.n;
  return nb;
}

// Rows of block b, 1-based inclusive like divide_region.
void block_rows(int b, int nb, long n, long* lo, long* hi) {
  if (!g_blk.empty()) { *lo = g_blk[b] + 1; *hi = g_blk[b + 1]; return; }
  divide_region(b, nb, 1, n, lo, hi);
}

// get_DInv_crs (matrix.f90:3104-3144): 1/a_ii, a zero pivot replaced by 1e-300.
void setup_pj(const OrcMat& A, Precon& P) {
  P.Dinv.assign(A.n, 0.0);
  for (long i = 0; i < A.n; ++i) {
    double d = 0.0;
    for (long j = A.rowptr[i] - 1; j < A.rowptr[i + 1] - 1; ++j)
      if (A.col[j] - A.istart == i) d = A.val[j];
    if (d == 0.0) d = 1.0e-300;
    P.Dinv[i] = 1.0 / d;
  }
}

// get_ILU_LU_crs + ILU_LU_crs + divide_ILU_crs (matrix.f90:8249-8392, 7970-8072, 7821-7897)
// with independ_nvec = 1: the block's rows restricted to in-block columns, IKJ ILU(0).
int setup_ilu0(const OrcMat& A, int nb, Precon& P) {
  P.ilu.resize(nb);
  int err = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(min : err)
  for (int b = 0; b < nb; ++b) {
    long lo, hi;
    block_rows(b, nb, A.n, &lo, &hi);
    IluBlock& B = P.ilu[b];
    B.r0 = lo - 1; B.r1 = hi;
    long m = B.r1 - B.r0;
    // block-local copy (local column = global - istart - r0)
    std::vector<int> p(m + 1), c; std::vector<double> v;
    p[0] = 0;
    for (long i = 0; i < m; ++i) {
      long gi = B.r0 + i;
      for (long j = A.rowptr[gi] - 1; j < A.rowptr[gi + 1] - 1; ++j) {
        long lc = (long)A.col[j] - A.istart - B.r0;
        if (lc >= 0 && lc < m) { c.push_back((int)lc); v.push_back(A.val[j]); }
      }
      p[i + 1] = (int)c.size();
    }
    // diagonal must exist (matrix.f90:8004-8021)
    std::vector<int> dptr(m, -1);
    for (long i = 0; i < m; ++i)
      for (int k = p[i]; k < p[i + 1]; ++k) if (c[k] == i) { dptr[i] = k; break; }
    bool ok = true;
    for (long i = 0; i < m; ++i) if (dptr[i] < 0) ok = false;
    if (!ok) { err = ORC_E_ZERO_PIVOT; continue; }
    // IKJ: for each row i, for each k < i in row i: a_ik /= a_kk; a_ij -= a_ik*a_kj (j > k)
    for (long i = 1; i < m; ++i) {
      for (int kc = p[i]; kc < p[i + 1]; ++kc) {
        int k = c[kc];
        if (k > i - 1) break;
        int kk = dptr[k];
        v[kc] = v[kc] / v[kk];
        for (int jc = p[i]; jc < p[i + 1]; ++jc) {
          int j = c[jc];
          if (j < k + 1) continue;
          for (int kj = kk; kj < p[k + 1]; ++kj)
            if (c[kj] == j) { v[jc] = v[jc] - v[kc] * v[kj]; break; }
        }
      }
    }
    // split (divide_ILU_crs): L = strictly lower + unit diagonal last, U = diagonal first
    B.Lp.assign(m + 1, 0); B.Up.assign(m + 1, 0);
    for (long i = 0; i < m; ++i) {
      for (int k = p[i]; k < p[i + 1]; ++k) {
        if (c[k] < i) { B.Lc.push_back(c[k]); B.Lv.push_back(v[k]); }
        if (c[k] > i) { B.Uc.push_back(c[k]); B.Uv.push_back(v[k]); }
        if (c[k] == i) {
          B.Lc.push_back(c[k]); B.Lv.push_back(1.0);
          B.Uc.push_back(c[k]); B.Uv.push_back(v[k]);
        }
      }
      B.Lp[i + 1] = (int)B.Lc.size();
      B.Up[i + 1] = (int)B.Uc.size();
    }
  }
  return err;
}

// solve_LU_crs (matrix.f90:8548-8747), independ_nvec = 1.
void solve_ilu0_block(const IluBlock& B, const double* r, double* s) {
  long m = B.r1 - B.r0;
  for (long i = 0; i < m; ++i) {
    double z = r[i];
    for (int j = B.Lp[i]; j < B.Lp[i + 1] - 1; ++j) z = z - s[B.Lc[j]] * B.Lv[j];
    s[i] = z / B.Lv[B.Lp[i + 1] - 1];
  }
  for (long i = m - 1; i >= 0; --i) {
    double z = s[i];
    for (int j = B.Up[i] + 1; j < B.Up[i + 1]; ++j) z = z - s[B.Uc[j]] * B.Uv[j];
    s[i] = z / B.Uv[B.Up[i]];
  }
}

// DILU_DInv_crs (matrix.f90:3482-3648) with independ_nvec = 1 and
// init_solve_ILU_crs (matrix.f90:5165-5412).
int setup_dilu(const OrcMat& A, int nb, int method, Precon& P) {
  P.Dinv.assign(A.n, 0.0);
  P.dilu.resize(nb);
  int err = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(min : err)
  for (int b = 0; b < nb; ++b) {
    long lo, hi;
    block_rows(b, nb, A.n, &lo, &hi);
    DiluBlock& B = P.dilu[b];
    B.r0 = lo - 1; B.r1 = hi;
    long gs = A.istart + B.r0, ge = A.istart + B.r1 - 1;   // global in-block column range
    long m = B.r1 - B.r0;
    std::vector<double> D(m, 0.0);
    // every row needs an in-block diagonal (matrix.f90:3519-3543)
    bool all_found = true;
    for (long k = 0; k < m; ++k) {
      long gk = B.r0 + k; bool found = false;
      for (long j = A.rowptr[gk] - 1; j < A.rowptr[gk + 1] - 1; ++j) {
        if (A.col[j] < gs || A.col[j] > ge) continue;
        if (A.col[j] - A.istart == gk) { found = true; break; }
      }
      if (!found) { all_found = false; break; }
    }
    if (!all_found) { err = ORC_E_ZERO_PIVOT; continue; }
    for (long k = 0; k < m; ++k) {
      long gk = B.r0 + k;
      long jstart = -1;
      for (long j = A.rowptr[gk] - 1; j < A.rowptr[gk + 1] - 1; ++j) {
        if (A.col[j] < gs || A.col[j] > ge) continue;
        if (jstart == -1) jstart = j;
        long colk = A.col[j] - A.istart;
        if (colk != gk) continue;
        D[k] = A.val[j];
        for (long jr = jstart; jr < j; ++jr) {
          long kr = A.col[jr] - A.istart;              // local row of the L entry
          for (long i = A.rowptr[kr] - 1; i < A.rowptr[kr + 1] - 1; ++i) {
            if (A.col[i] < gs || A.col[i] > ge) continue;
            long rc = A.col[i] - A.istart;
            if (method == ORC_ILUD) {
              if (rc == gk) { D[k] = D[k] - A.val[jr] * A.val[i] / D[kr - B.r0]; break; }
            } else {
              if (kr < rc) D[k] = D[k] - A.val[jr] * A.val[i] / D[kr - B.r0];
            }
          }
        }
        break;
      }
    }
    for (long k = 0; k < m; ++k) P.Dinv[B.r0 + k] = 1.0 / D[k];
    // L range: in-block entries with column < k; U range: in-block entries with column > k
    B.Ls.assign(m, 0); B.Le.assign(m, -1); B.Us.assign(m, 0); B.Ue.assign(m, 1);
    for (long k = 0; k < m; ++k) {
      long gk = B.r0 + k;
      long a = A.rowptr[gk] - 1, z = A.rowptr[gk + 1] - 1;
      B.Ls[k] = z - 1; B.Le[k] = a;                    // empty unless set below
      for (long j = a; j < z; ++j) { if (A.col[j] < gs) continue; B.Ls[k] = j; break; }
      for (long j = a; j < z; ++j) {
        if (A.col[j] < gs) continue;
        if (A.col[j] - A.istart >= gk) { B.Le[k] = j - 1; break; }
      }
      B.Us[k] = a; B.Ue[k] = z - 1;
      for (long j = z - 1; j >= a; --j) { if (A.col[j] > ge) continue; B.Us[k] = j; break; }
      for (long j = z - 1; j >= a; --j) {
        if (A.col[j] - A.istart > gk) continue;
        B.Ue[k] = j + 1; break;
      }
    }
  }
  return err;
}

// solve_ILU_crs (matrix.f90:4987-5163), independ_nvec = 1: (D+L) D^-1 (D+U) s = r.
void solve_dilu_block(const OrcMat& A, const DiluBlock& B, const double* Dinv,
                      const double* r, double* s) {
  long m = B.r1 - B.r0;
  long off = A.istart + B.r0;                          // global id of local row 0
  for (long k = 0; k < m; ++k) {
    double zz = r[k];
    for (long j = B.Ls[k]; j <= B.Le[k]; ++j) zz = zz - s[A.col[j] - off] * A.val[j];
    s[k] = Dinv[k] * zz;
  }
  for (long k = m - 1; k >= 0; --k) {
    double zz = 0.0;
    for (long j = B.Us[k]; j >= B.Ue[k]; --j) zz = zz + s[A.col[j] - off] * A.val[j];
    s[k] = s[k] - Dinv[k] * zz;
  }
}

int setup_precon(const OrcMat& A, const OrcParams& prm, Precon& P) {
  P.A = &A;
  int kind = prm.ipreflag;
  if (kind == ORC_PRECON_AS) kind = ORC_PRECON_BJ;     // one process: AS reduces to BJ
  P.kind = kind;
  P.ilu_method = prm.ILU_method < 0 ? ORC_ILUD : prm.ILU_method;  // default ILUD (type.f90:1042)
  if (!g_blk.empty() && g_blk.back() != A.n) return ORC_E_ARG;
  int nb = nblocks_for(A, prm.precon_thblock);
  switch (kind) {
    case ORC_PRECON_NONE: return 0;
    case ORC_PRECON_PJ: setup_pj(A, P); return 0;
    case ORC_PRECON_BJ:
      if (P.ilu_method == ORC_ILU0) return setup_ilu0(A, nb, P);
      return setup_dilu(A, nb, P.ilu_method, P);
    default: return ORC_E_UNSUPPORTED;
  }
}

// calc_precon (krylov_h.f90:2035-2058): s = M^-1 r.  With no preconditioner s = r.
void apply_precon(const Precon& P, const double* r, double* s) {
  const OrcMat& A = *P.A;
  switch (P.kind) {
    case ORC_PRECON_NONE:
#pragma omp parallel for schedule(static)
      for (long i = 0; i < A.n; ++i) s[i] = r[i];
      break;
    case ORC_PRECON_PJ:
#pragma omp parallel for schedule(static)
      for (long i = 0; i < A.n; ++i) s[i] = r[i] * P.Dinv[i];
      break;
    case ORC_PRECON_BJ:
      if (P.ilu_method == ORC_ILU0) {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t b = 0; b < P.ilu.size(); ++b)
          solve_ilu0_block(P.ilu[b], r + P.ilu[b].r0, s + P.ilu[b].r0);
      } else {
#pragma omp parallel for schedule(dynamic, 1)
        for (size_t b = 0; b < P.dilu.size(); ++b)
          solve_dilu_block(A, P.dilu[b], P.Dinv.data() + P.dilu[b].r0,
                           r + P.dilu[b].r0, s + P.dilu[b].r0);
      }
      break;
  }
}

// ---------------------------------------------------------------------------------
// Solvers.  Each returns niter/iret the way the reference does.

// KSP_pCG (pcg.f90:224-892), lagged x update.
void pcg(const OrcMat& A, const Precon& P, const OrcParams& prm, const double* b,
         double* x, double* hist, int* niter, int* iret) {
  long n = A.n;
  std::vector<double> r(n), p(n, 0.0), q(n), s(n);
  residual(A, x, b, r.data());
  double bnorm = std::sqrt(dot(n, b, b));
  double rnorm = std::sqrt(dot(n, r.data(), r.data()));
  double alpha = 0.0, beta = 0.0;
  apply_precon(P, r.data(), s.data());
  double rho0 = dot(n, s.data(), r.data());
  int itr;
  for (itr = 1; itr <= prm.itrmax; ++itr) {
    hist[itr - 1] = rnorm / bnorm;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {                 // CG_axpy2 (pcg.f90:4-20)
      x[i] = x[i] + alpha * p[i];
      p[i] = s[i] + beta * p[i];
    }
    spmv(A, p.data(), q.data());
    double gamma = dot(n, p.data(), q.data());
    alpha = rho0 / gamma;
    double ma = -alpha;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) r[i] = ma * q[i] + 1.0 * r[i];
    apply_precon(P, r.data(), s.data());
    double rho1 = dot(n, s.data(), r.data());      // CG_calc_dot2 (pcg.f90:22-53)
    rnorm = std::sqrt(dot(n, r.data(), r.data()));
    if (rnorm / bnorm < prm.rtolmax) break;
    if (rnorm / bnorm > 1.0e8) break;
    beta = rho1 / rho0;
    rho0 = rho1;
  }
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) x[i] = alpha * p[i] + 1.0 * x[i];
  *niter = std::min(prm.itrmax, itr);
  *iret = (prm.itrmax <= itr) ? 1 : 0;
}

// KSP_pBiCG (pbicg.f90:280-698): right-preconditioned BiCGStab.
void pbicg(const OrcMat& A, const Precon& P, const OrcParams& prm, const double* b,
           double* x, double* hist, int* niter, int* iret) {
  long n = A.n;
  std::vector<double> r(n), r0(n), p(n), q(n, 0.0), pp(n, 0.0), e(n, 0.0), pe(n, 0.0), v(n, 0.0);
  residual(A, x, b, r.data());
  double bnorm = std::sqrt(dot(n, b, b));
  double rnorm = std::sqrt(dot(n, r.data(), r.data()));
  r0 = r; p = r;
  double c1 = dot(n, r0.data(), r0.data()), c2 = 0.0, c3 = 0.0;
  int itr;
  for (itr = 1; itr <= prm.itrmax; ++itr) {
    hist[itr - 1] = rnorm / bnorm;
    apply_precon(P, p.data(), pp.data());
    spmv(A, pp.data(), q.data());
    c2 = dot(n, r0.data(), q.data());
    double alpha = c1 / c2;
    double ma = -alpha;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) e[i] = 1.0 * r[i] + ma * q[i] + 0.0 * e[i];   // axpy_vec3
    apply_precon(P, e.data(), pe.data());
    spmv(A, pe.data(), v.data());
    double ev = dot(n, e.data(), v.data());
    double vv = dot(n, v.data(), v.data());
    c3 = ev / vv;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) x[i] = alpha * pp[i] + c3 * pe[i] + 1.0 * x[i];
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) r[i] = e[i] - c3 * v[i];                      // BiCG_axpy3_dot
    c1 = dot(n, r.data(), r0.data());
    rnorm = std::sqrt(dot(n, r.data(), r.data()));
    if (rnorm / bnorm < prm.rtolmax) break;
    double beta = c1 / (c3 * c2);
    double t2 = -beta * c3;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) p[i] = 1.0 * r[i] + t2 * q[i] + beta * p[i];
  }
  *niter = std::min(prm.itrmax, itr);
  *iret = (prm.itrmax <= itr) ? 1 : 0;
}

// GivensRotations (pcagmres.f90:190-242), including its zero-diagonal guard
// `h/1.0d0-300`, which Fortran evaluates as (h/1) - 300.
void givens(int m, double* h, int i, double* c, double* s, double* e) {
  // h is (m+1) x m column-major, 1-based column i
  double* col = h + (long)(i - 1) * (m + 1);
  for (int k = 1; k <= i - 1; ++k) {
    double t1 = col[k - 1] * c[k - 1] - col[k] * s[k - 1];
    double t2 = col[k - 1] * s[k - 1] + col[k] * c[k - 1];
    col[k - 1] = t1; col[k] = t2;
  }
  double t;
  if (col[i - 1] == 0.0) t = col[i] / 1.0 - 300.0;
  else t = col[i] / col[i - 1];
  c[i - 1] = 1.0 / std::sqrt(1.0 + t * t);
  s[i - 1] = -c[i - 1] * t;
  double t1 = c[i - 1] * e[i - 1] - s[i - 1] * e[i];
  double t2 = s[i - 1] * e[i - 1] + c[i - 1] * e[i];
  e[i - 1] = t1; e[i] = t2;
  col[i - 1] = c[i - 1] * col[i - 1] - s[i - 1] * col[i];
  col[i] = 0.0;
}

// update_xVec (pcagmres.f90:1136-1236): y = H^-1 e, v0 = V y, x += M^-1 v0.
void update_x(const OrcMat& A, const Precon& P, int m0, int mm, const double* h,
              const double* e, const std::vector<double>& V, double* x) {
  long n = A.n;
  std::vector<double> y(m0 + 1, 0.0), v0(n), x0(n);
  for (int i = mm; i >= 1; --i) {
    y[i - 1] = e[i - 1];
    for (int j = mm; j >= i + 1; --j) y[i - 1] = y[i - 1] - h[(i - 1) + (long)(j - 1) * (m0 + 1)] * y[j - 1];
    double d = h[(i - 1) + (long)(i - 1) * (m0 + 1)];
    if (d == 0.0) y[i - 1] = y[i - 1] / 1.0e-300;
    else y[i - 1] = y[i - 1] / d;
  }
#pragma omp parallel for schedule(static)
  for (long j = 0; j < n; ++j) {                  // sum_vec_FP64_CPU (pcagmres.f90:54-90)
    double t = 0.0;
    for (int i = 0; i < mm; ++i) t = t + y[i] * V[(long)i * n + j];
    v0[j] = t;
  }
  apply_precon(P, v0.data(), x0.data());
#pragma omp parallel for schedule(static)
  for (long j = 0; j < n; ++j) x[j] = 1.0 * x0[j] + 1.0 * x[j];
}

// KSP_pGMRES (pgmres.f90:62-525): right-preconditioned GMRES(m), MGS or CGS.
void pgmres(const OrcMat& A, const Precon& P, const OrcParams& prm, const double* b,
            double* x, double* hist, int* niter, int* iret) {
  long n = A.n;
  int m = prm.GMRES_m > 0 ? prm.GMRES_m : 4;
  int gs = prm.GMRES_GSflag > 0 ? prm.GMRES_GSflag : ORC_GS_MGS;
  std::vector<double> r(n), V((long)(m + 1) * n, 0.0), pv(n), w(n);
  std::vector<double> h((long)(m + 1) * m), c(m + 1), s(m + 1), e(m + 1), hk(m + 1);
  double bnorm = std::sqrt(dot(n, b, b));
  double rnorm = 0.0;
  int itr = 1, inner = 1, mm = 0;
  bool done = false;
  for (itr = 1; itr <= prm.itrmax; itr += m) {
    std::fill(e.begin(), e.end(), 0.0); std::fill(c.begin(), c.end(), 0.0);
    std::fill(s.begin(), s.end(), 0.0); std::fill(h.begin(), h.end(), 0.0);
    residual(A, x, b, r.data());
    rnorm = std::sqrt(dot(n, r.data(), r.data()));
    double t1 = -1.0 / rnorm;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) V[i] = t1 * r[i] + 0.0 * V[i];
    e[0] = -rnorm;
    if (rnorm / bnorm < prm.rtolmax) break;
    if (itr == 1) hist[itr - 1] = rnorm / bnorm;
    bool exit_inner = false;
    for (inner = 1; inner <= m; ++inner) {
      apply_precon(P, V.data() + (long)(inner - 1) * n, pv.data());
      spmv(A, pv.data(), w.data());
      double* hcol = h.data() + (long)(inner - 1) * (m + 1);
      if (gs == ORC_GS_MGS) {
        for (int k = 1; k <= inner; ++k) {
          const double* vk = V.data() + (long)(k - 1) * n;
          double hkv = dot(n, w.data(), vk);
          hcol[k - 1] = hkv;
          double mh = -hkv;
#pragma omp parallel for schedule(static)
          for (long i = 0; i < n; ++i) w[i] = mh * vk[i] + 1.0 * w[i];
        }
      } else {
        // CGS_Orth (pgmres.f90:11-58): h = V^T w, then w -= V h
        for (int k = 1; k <= inner; ++k) hk[k - 1] = dot(n, w.data(), V.data() + (long)(k - 1) * n);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
          double t = w[i];
          for (int k = 1; k <= inner; ++k) t = t - hk[k - 1] * V[(long)(k - 1) * n + i];
          w[i] = t;
        }
        for (int k = 1; k <= inner; ++k) hcol[k - 1] = hk[k - 1];
      }
      double wn = std::sqrt(dot(n, w.data(), w.data()));
      hcol[inner] = wn;
      double inv = 1.0 / wn;
      double* vn = V.data() + (long)inner * n;
#pragma omp parallel for schedule(static)
      for (long i = 0; i < n; ++i) vn[i] = inv * w[i] + 0.0 * vn[i];
      givens(m, h.data(), inner, c.data(), s.data(), e.data());
      rnorm = std::fabs(e[inner]);
      mm = inner;
      if (itr + inner <= prm.itrmax) hist[itr + inner - 1] = rnorm / bnorm;
      if (rnorm / bnorm < prm.rtolmax) { exit_inner = true; break; }
      if (itr + inner == prm.itrmax) { exit_inner = true; break; }
    }
    if (!exit_inner) inner = m + 1;             // Fortran DO variable after completion
    if (m < mm) mm = m;
    update_x(A, P, m, mm, h.data(), e.data(), V, x);
    if (rnorm / bnorm < prm.rtolmax) { done = true; break; }
    if (itr + inner == prm.itrmax) { done = true; break; }
  }
  (void)done;
  *niter = std::min(prm.itrmax, itr + inner);
  *iret = (prm.itrmax <= itr) ? 1 : 0;
}

}  // namespace

// ---------------------------------------------------------------------------------
// Double-double CG (ddKSP_pCG, ddpcg.f90:247-563) and its building blocks.
//
// dd arithmetic (dd_func.f90:5-239): "sloppy" add/sub (two-sum of the high parts, low
// parts added, renormalised), Dekker product with the split constant 134217729 = 2^27+1,
// division by one Newton correction, square root from 1/sqrt(hi).  Built with
// -ffp-contract=off, so every operation rounds once, as the reference's Fortran does.
struct DD { double hi, lo; };

DD dd_add(DD a, DD b) {
  double p1 = a.hi + b.hi;
  double p2 = p1 - a.hi;
  double t1l = (a.hi - (p1 - p2)) + (b.hi - p2);
  double t1h = p1;
  t1l = t1l + a.lo + b.lo;
  double s1 = t1h + t1l;
  t1l = t1l - (s1 - t1h);
  return DD{s1, t1l};
}
DD dd_sub(DD a, DD b) {
  double p1 = a.hi - b.hi;
  double p2 = p1 - a.hi;
  double t1l = (a.hi - (p1 - p2)) - (b.hi + p2);
  double t1h = p1;
  t1l = t1l + a.lo - b.lo;
  double s1 = t1h + t1l;
  t1l = t1l - (s1 - t1h);
  return DD{s1, t1l};
}
DD dd_mul(DD a, DD b) {
  double t1h = a.hi * b.hi;
  double u1 = 134217729.0 * a.hi;
  double p1 = u1 - (u1 - a.hi);
  double p2 = a.hi - p1;
  u1 = 134217729.0 * b.hi;
  double r1 = u1 - (u1 - b.hi);
  double r2 = b.hi - r1;
  double t1l = ((p1 * r1 - t1h) + p1 * r2 + p2 * r1) + p2 * r2;
  t1l = t1l + (a.hi * b.lo + a.lo * b.hi);
  double s1 = t1h + t1l;
  t1l = t1l - (s1 - t1h);
  return DD{s1, t1l};
}
DD dd_div(DD a, DD b) {
  double q1 = a.hi / b.hi;
  double t1h = b.hi * q1;
  double u1 = 134217729.0 * b.hi;
  double p1 = u1 - (u1 - b.hi);
  double p2 = b.hi - p1;
  u1 = 134217729.0 * q1;
  double r1 = u1 - (u1 - q1);
  double r2 = q1 - r1;
  double t1l = ((p1 * r1 - t1h) + p1 * r2 + p2 * r1) + p2 * r2;
  t1l = t1l + (b.lo * q1);
  double s1 = t1h + t1l;
  t1l = t1l - (s1 - t1h);
  t1h = s1;
  s1 = a.hi - t1h;
  r1 = s1 - a.hi;
  double s2 = (a.hi - (s1 - r1)) - (t1h + r1);
  s2 = s2 - t1l;
  s2 = s2 + a.lo;
  double q2 = (s1 + s2) / b.hi;
  double h = q1 + q2;
  return DD{h, q2 - (h - q1)};
}
// A zero argument falls through to the general formula (the reference sets 0 and then
// overwrites it); a negative one gives 0.
DD dd_sqrt(DD a) {
  if (a.hi < 0.0 || (a.hi == 0.0 && a.lo < 0.0)) return DD{0.0, 0.0};
  double x = 1.0 / std::sqrt(a.hi);
  double ax = a.hi * x;
  DD y = dd_mul(DD{x, 0.0}, DD{0.5, 0.0});
  DD z = dd_mul(DD{ax, 0.0}, DD{ax, 0.0});
  DD t2 = dd_sub(a, z);
  DD t1 = dd_mul(t2, y);
  return dd_add(t1, DD{ax, 0.0});
}

// dd dot in a fixed order, independent of the thread count (the reference's blocked
// accumulators, ddvec.f90:111-240, follow its OpenMP split instead): stream t (0 <= t <
// 2^17) sums the products of the elements i = t, t + 2^17, ... in increasing i, starting
// from 0 and adding with dd_add(sum, term); the 2^17 stream sums are combined by a complete
// binary tree, level by level, neighbours in pairs (s'[k] = dd_add(s[2k], s[2k+1])).
constexpr long DD_NSTREAM = 1L << 17;
DD dd_dot(long n, const double* xh, const double* xl, const double* yh, const double* yl) {
  std::vector<DD> s(DD_NSTREAM);
#pragma omp parallel for schedule(static)
  for (long t = 0; t < DD_NSTREAM; ++t) {
    DD a{0.0, 0.0};
    for (long i = t; i < n; i += DD_NSTREAM) a = dd_add(a, dd_mul(DD{xh[i], xl[i]}, DD{yh[i], yl[i]}));
    s[t] = a;
  }
  std::vector<DD> u(DD_NSTREAM / 2);
  for (long h = DD_NSTREAM / 2; h > 0; h /= 2) {
#pragma omp parallel for schedule(static) if (h >= 4096)
    for (long k = 0; k < h; ++k) u[k] = dd_add(s[2 * k], s[2 * k + 1]);
    std::copy(u.begin(), u.begin() + h, s.begin());
  }
  return s[0];
}

// ddMatVec_crs (ddmatrix.f90:1785-2355), single process: per row, c = a_ij x_j and
// t = c + t over the row in CRS order.  A's low parts are used when alo is given.
void dd_spmv(const OrcMat& A, const double* alo, const double* xh, const double* xl, double* yh, double* yl) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < A.n; ++i) {
    DD t{0.0, 0.0};
    for (long j = A.rowptr[i] - 1; j < A.rowptr[i + 1] - 1; ++j) {
      const long c = A.col[j] - A.istart;
      t = dd_add(dd_mul(DD{A.val[j], alo ? alo[j] : 0.0}, DD{xh[c], xl[c]}), t);
    }
    yh[i] = t.hi;
    yl[i] = t.lo;
  }
}

// ddaxpy (ddvec.f90:14-54): y = alpha x + beta y
void dd_axpy(long n, DD alpha, DD beta, const double* xh, const double* xl, double* yh, double* yl) {
#pragma omp parallel for schedule(static)
  for (long i = 0; i < n; ++i) {
    DD c = dd_mul(beta, DD{yh[i], yl[i]});
    DD b = dd_mul(alpha, DD{xh[i], xl[i]});
    DD y = dd_add(b, c);
    yh[i] = y.hi;
    yl[i] = y.lo;
  }
}

struct DdPrecon {
  int kind = ORC_PRECON_NONE;
  int method = ORC_ILUD;
  int prec = 2;                          // PRECISION_PRECONDITION
  std::vector<double> dh, dl;            // D^-1 (point Jacobi or D-ILU), double-double
  std::vector<DiluBlock> blocks;         // D-ILU L / U ranges
};

// ddget_DInv_crs (ddmatrix.f90:283-349): D^-1 = 1 / a_ii, a zero pivot replaced by 1e-100.
void dd_setup_pj(const OrcMat& A, const double* alo, DdPrecon& P) {
  P.dh.assign(A.n, 0.0);
  P.dl.assign(A.n, 0.0);
  for (long k = 0; k < A.n; ++k)
    for (long j = A.rowptr[k] - 1; j < A.rowptr[k + 1] - 1; ++j)
      if (A.col[j] - A.istart == k) {
        DD a{A.val[j], alo ? alo[j] : 0.0};
        DD d = (a.hi == 0.0 && a.lo == 0.0) ? dd_div(DD{1.0, 0.0}, DD{1.0e-100, 0.0})
                                            : dd_div(DD{1.0, 0.0}, a);
        P.dh[k] = d.hi;
        P.dl[k] = d.lo;
      }
}

// ddDILU_DInv_crs (ddmatrix.f90:1451-1640) with independ_nvec = 1: the D-ILU diagonal in
// dd arithmetic, then D^-1 = 1 / D (a zero D replaced by 1e-100).  The L / U ranges of the
// sweeps are the double setup's.
int dd_setup_dilu(const OrcMat& A, const double* alo, int nb, int method, DdPrecon& P) {
  Precon tmp;
  int err = setup_dilu(A, nb, method, tmp);
  if (err) return err;
  P.blocks = tmp.dilu;
  P.dh.assign(A.n, 0.0);
  P.dl.assign(A.n, 0.0);
  auto av = [&](long j) { return DD{A.val[j], alo ? alo[j] : 0.0}; };
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < nb; ++b) {
    const DiluBlock& B = P.blocks[b];
    long gs = A.istart + B.r0, ge = A.istart + B.r1 - 1;
    long m = B.r1 - B.r0;
    std::vector<DD> D(m, DD{0.0, 0.0});
    for (long k = 0; k < m; ++k) {
      long gk = B.r0 + k;
      long jstart = -1;
      for (long j = A.rowptr[gk] - 1; j < A.rowptr[gk + 1] - 1; ++j) {
        if (A.col[j] < gs || A.col[j] > ge) continue;
        if (jstart == -1) jstart = j;
        long colk = A.col[j] - A.istart;
        if (colk < gk) continue;
        D[k] = colk == gk ? av(j) : DD{0.0, 0.0};
        for (long jr = jstart; jr < j; ++jr) {
          long kr = A.col[jr] - A.istart;              // local row of the L entry
          for (long i = A.rowptr[kr] - 1; i < A.rowptr[kr + 1] - 1; ++i) {
            if (A.col[i] < gs) continue;
            if (A.col[i] > ge) break;
            long rc = A.col[i] - A.istart;
            bool take = method == ORC_ILUD ? rc == gk : kr < rc;
            if (!take) continue;
            DD c = dd_mul(av(jr), av(i));
            DD dk = D[kr - B.r0];
            c = (dk.hi == 0.0 && dk.lo == 0.0) ? dd_div(c, DD{1.0e-100, 0.0}) : dd_div(c, dk);
            D[k] = dd_sub(D[k], c);
            if (method == ORC_ILUD) break;
          }
        }
        break;
      }
    }
    for (long k = 0; k < m; ++k) {
      DD d = (D[k].hi == 0.0 && D[k].lo == 0.0) ? dd_div(DD{1.0, 0.0}, DD{1.0e-100, 0.0})
                                                : dd_div(DD{1.0, 0.0}, D[k]);
      P.dh[B.r0 + k] = d.hi;
      P.dl[B.r0 + k] = d.lo;
    }
  }
  return 0;
}

// ddsolve_ILU_crs (ddmatrix.f90:4310-4680), independ_nvec = 1: forward
// z = r - sum L s, s = z D^-1; backward z = sum U s (Ustart down to Uend), s = s - D^-1 z.
// PRECISION_PRECONDITION 1 drops the low parts of A and of D^-1.
void dd_solve_dilu_block(const OrcMat& A, const double* alo, const DiluBlock& B, const double* dh,
                         const double* dl, int prec, const double* rh, const double* rl, double* sh,
                         double* sl) {
  long m = B.r1 - B.r0;
  long off = A.istart + B.r0;
  auto av = [&](long j) { return DD{A.val[j], (prec == 2 && alo) ? alo[j] : 0.0}; };
  for (long k = 0; k < m; ++k) {
    DD zz{rh[k], rl[k]};
    for (long j = B.Ls[k]; j <= B.Le[k]; ++j) {
      long c = A.col[j] - off;
      zz = dd_sub(zz, dd_mul(DD{sh[c], sl[c]}, av(j)));
    }
    DD s = dd_mul(zz, DD{dh[k], prec == 2 ? dl[k] : 0.0});
    sh[k] = s.hi;
    sl[k] = s.lo;
  }
  for (long k = m - 1; k >= 0; --k) {
    DD zz{0.0, 0.0};
    for (long j = B.Us[k]; j >= B.Ue[k]; --j) {
      long c = A.col[j] - off;
      zz = dd_add(zz, dd_mul(DD{sh[c], sl[c]}, av(j)));
    }
    DD c = dd_mul(DD{dh[k], prec == 2 ? dl[k] : 0.0}, zz);
    DD s = dd_sub(DD{sh[k], sl[k]}, c);
    sh[k] = s.hi;
    sl[k] = s.lo;
  }
}

void dd_apply_precon(const OrcMat& A, const double* alo, const DdPrecon& P, const double* rh,
                     const double* rl, double* sh, double* sl) {
  switch (P.kind) {
    case ORC_PRECON_NONE:
#pragma omp parallel for schedule(static)
      for (long i = 0; i < A.n; ++i) { sh[i] = rh[i]; sl[i] = rl[i]; }
      break;
    case ORC_PRECON_PJ:
#pragma omp parallel for schedule(static)
      for (long i = 0; i < A.n; ++i) {   // ddpointJacobi (ddmatrix.f90:3523-3567): z = D^-1 r
        DD z = dd_mul(DD{P.dh[i], P.prec == 2 ? P.dl[i] : 0.0}, DD{rh[i], rl[i]});
        sh[i] = z.hi;
        sl[i] = z.lo;
      }
      break;
    default:
#pragma omp parallel for schedule(dynamic, 1)
      for (size_t b = 0; b < P.blocks.size(); ++b) {
        const long r0 = P.blocks[b].r0;
        dd_solve_dilu_block(A, alo, P.blocks[b], P.dh.data() + r0, P.dl.data() + r0, P.prec, rh + r0,
                            rl + r0, sh + r0, sl + r0);
      }
      break;
  }
}

// ddKSP_pCG (ddpcg.f90:247-563): lagged x update, stop on the recursive residual.
void ddpcg(const OrcMat& A, const double* alo, const DdPrecon& P, const OrcParams& prm, const double* bh,
           const double* bl, double* xh, double* xl, double* hist, int* niter, int* iret) {
  long n = A.n;
  std::vector<double> rh(n), rl(n), ph(n, 0.0), pl(n, 0.0), qh(n), ql(n), sh(n), sl(n);
  dd_spmv(A, alo, xh, xl, rh.data(), rl.data());                 // ddcalc_res: r = A x,
  dd_axpy(n, DD{1.0, 0.0}, DD{-1.0, 0.0}, bh, bl, rh.data(), rl.data());   // r = 1 b - 1 r
  DD bnorm = dd_sqrt(dd_dot(n, bh, bl, bh, bl));
  DD rnorm = dd_sqrt(dd_dot(n, rh.data(), rl.data(), rh.data(), rl.data()));
  DD alpha{0.0, 0.0}, beta{0.0, 0.0};
  dd_apply_precon(A, alo, P, rh.data(), rl.data(), sh.data(), sl.data());
  DD rho0 = dd_dot(n, sh.data(), sl.data(), rh.data(), rl.data());
  int itr;
  for (itr = 1; itr <= prm.itrmax; ++itr) {
    hist[itr - 1] = rnorm.hi / bnorm.hi;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {                 // ddCG_axpy2 (ddpcg.f90:9-59)
      DD x = dd_add(DD{xh[i], xl[i]}, dd_mul(alpha, DD{ph[i], pl[i]}));
      DD p = dd_add(DD{sh[i], sl[i]}, dd_mul(beta, DD{ph[i], pl[i]}));
      xh[i] = x.hi; xl[i] = x.lo;
      ph[i] = p.hi; pl[i] = p.lo;
    }
    dd_spmv(A, alo, ph.data(), pl.data(), qh.data(), ql.data());
    DD gamma = dd_dot(n, ph.data(), pl.data(), qh.data(), ql.data());
    alpha = dd_div(rho0, gamma);
    DD t1 = dd_mul(DD{-1.0, 0.0}, alpha);
    dd_axpy(n, t1, DD{1.0, 0.0}, qh.data(), ql.data(), rh.data(), rl.data());
    dd_apply_precon(A, alo, P, rh.data(), rl.data(), sh.data(), sl.data());
    DD rho1 = dd_dot(n, sh.data(), sl.data(), rh.data(), rl.data());   // ddCG_calc_dot2
    rnorm = dd_sqrt(dd_dot(n, rh.data(), rl.data(), rh.data(), rl.data()));
    if (rnorm.hi / bnorm.hi < prm.rtolmax) break;
    beta = dd_div(rho1, rho0);
    rho0 = rho1;
  }
  dd_axpy(n, alpha, DD{1.0, 0.0}, ph.data(), pl.data(), xh, xl);
  *niter = std::min(prm.itrmax, itr);
  *iret = (prm.itrmax <= itr) ? 1 : 0;
}

// ddKSP_pBiCG (ddpbicg.f90:496-875): right-preconditioned BiCGStab in dd, with the vector
// updates of ddBiCG_axpy3 / axpy4 / axpy3_dot / axpy4_ (ddpbicg.f90:8-326).  The history
// entry is the high part of dd_div(rnorm, bnorm).
void ddbicg(const OrcMat& A, const double* alo, const DdPrecon& P, const OrcParams& prm, const double* bh,
            const double* bl, double* xh, double* xl, double* hist, int* niter, int* iret) {
  const long n = A.n;
  std::vector<double> rh(n), rl(n), r0h(n), r0l(n), ph(n), pl(n), pph(n), ppl(n), qh(n), ql(n), eh(n), el(n),
      peh(n), pel(n), vh(n), vl(n);
  dd_spmv(A, alo, xh, xl, rh.data(), rl.data());
  dd_axpy(n, DD{1.0, 0.0}, DD{-1.0, 0.0}, bh, bl, rh.data(), rl.data());
  r0h = rh; r0l = rl; ph = rh; pl = rl;
  DD bnorm = dd_dot(n, bh, bl, bh, bl);
  DD c1 = dd_dot(n, r0h.data(), r0l.data(), r0h.data(), r0l.data());
  DD rnorm = c1;
  bnorm = dd_sqrt(bnorm);
  rnorm = dd_sqrt(rnorm);
  DD c2{0.0, 0.0}, c3{0.0, 0.0};
  int itr;
  for (itr = 1; itr <= prm.itrmax; ++itr) {
    hist[itr - 1] = dd_div(rnorm, bnorm).hi;
    dd_apply_precon(A, alo, P, ph.data(), pl.data(), pph.data(), ppl.data());
    dd_spmv(A, alo, pph.data(), ppl.data(), qh.data(), ql.data());
    c2 = dd_dot(n, r0h.data(), r0l.data(), qh.data(), ql.data());
    const DD alpha = dd_div(c1, c2);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {   // ddBiCG_axpy3: e = r - alpha q
      DD e = dd_sub(DD{rh[i], rl[i]}, dd_mul(alpha, DD{qh[i], ql[i]}));
      eh[i] = e.hi; el[i] = e.lo;
    }
    dd_apply_precon(A, alo, P, eh.data(), el.data(), peh.data(), pel.data());
    dd_spmv(A, alo, peh.data(), pel.data(), vh.data(), vl.data());
    const DD t1 = dd_dot(n, eh.data(), el.data(), vh.data(), vl.data());   // ddBiCG_calc_dot2
    const DD t2 = dd_dot(n, vh.data(), vl.data(), vh.data(), vl.data());
    c3 = dd_div(t1, t2);
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {   // ddBiCG_axpy4: x = x + (alpha pp + c3 pe)
      DD c = dd_mul(c3, DD{peh[i], pel[i]});
      DD b = dd_mul(alpha, DD{pph[i], ppl[i]});
      c = dd_add(b, c);
      DD x = dd_add(DD{xh[i], xl[i]}, c);
      xh[i] = x.hi; xl[i] = x.lo;
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {   // ddBiCG_axpy3_dot: r = e - c3 v
      DD r = dd_sub(DD{eh[i], el[i]}, dd_mul(c3, DD{vh[i], vl[i]}));
      rh[i] = r.hi; rl[i] = r.lo;
    }
    c1 = dd_dot(n, rh.data(), rl.data(), r0h.data(), r0l.data());
    rnorm = dd_sqrt(dd_dot(n, rh.data(), rl.data(), rh.data(), rl.data()));
    if (rnorm.hi / bnorm.hi < prm.rtolmax) break;
    const DD beta = dd_div(c1, dd_mul(c3, c2));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) {   // ddBiCG_axpy4_: p = r + beta (p - c3 q)
      DD c = dd_mul(c3, DD{qh[i], ql[i]});
      c = dd_sub(DD{ph[i], pl[i]}, c);
      c = dd_mul(beta, c);
      DD pn = dd_add(DD{rh[i], rl[i]}, c);
      ph[i] = pn.hi; pl[i] = pn.lo;
    }
  }
  *niter = std::min(prm.itrmax, itr);
  *iret = (prm.itrmax <= itr) ? 1 : 0;
}

// ddGivensRotations (ddpgmres.f90:147-250) on column i (1-based) of the (m+1) x m
// Hessenberg matrix h, with the reference's operand orders and its zero-diagonal guard
// (divide by 1e-100).
void dd_givens(int m, DD* h, int i, DD* c, DD* s, DD* e) {
  DD* col = h + (long)(i - 1) * (m + 1);
  for (int k = 1; k <= i - 1; ++k) {
    const DD t1 = dd_sub(dd_mul(col[k - 1], c[k - 1]), dd_mul(col[k], s[k - 1]));
    const DD t2 = dd_add(dd_mul(col[k - 1], s[k - 1]), dd_mul(col[k], c[k - 1]));
    col[k - 1] = t1;
    col[k] = t2;
  }
  const DD d = col[i - 1];
  const DD t = (d.hi == 0.0 && d.lo == 0.0) ? dd_div(col[i], DD{1.0e-100, 0.0}) : dd_div(col[i], d);
  const DD q = dd_sqrt(dd_add(DD{1.0, 0.0}, dd_mul(t, t)));
  c[i - 1] = dd_div(DD{1.0, 0.0}, q);
  s[i - 1] = dd_mul(DD{-1.0, 0.0}, dd_mul(c[i - 1], t));
  const DD e1 = dd_sub(dd_mul(c[i - 1], e[i - 1]), dd_mul(s[i - 1], e[i]));
  const DD e2 = dd_add(dd_mul(s[i - 1], e[i - 1]), dd_mul(c[i - 1], e[i]));
  e[i - 1] = e1;
  e[i] = e2;
  col[i - 1] = dd_sub(dd_mul(c[i - 1], col[i - 1]), dd_mul(s[i - 1], col[i]));
  col[i] = DD{0.0, 0.0};
}

// ddKSP_pGMRES (ddpgmres.f90:254-713): right-preconditioned GMRES(m) in dd.  MGS
// (ddMGS_Orthonormalization, ddQRDecomposition.f90:4-47) projects w on v_1..v_{i-1} one
// at a time with <w, v_k>; CGS (ddCGS_Orthonormalization, :49-121) takes <v_k, w> for all
// k < i from the same w and then subtracts.  Both finish with <w, v_i>, w -= h_ii v_i and
// h_{i+1,i} = sqrt(<w, w>).  The restart residual is tested only against abstolmax, which
// parcel_ddgmres fixes at 0 (ddwrapper.f90:438), so that test never fires.  History
// entries are rnorm.hi / bnorm.hi; the first cycle also stores its starting residual.
// With itrmax = 1 the first cycle runs all m steps (the itr + inner == itrmax exit cannot
// fire) and the reference writes their history past entry itrmax; here those entries are
// dropped.  For itrmax > 1 an unconverged solve stops at itr + inner == itrmax with iret 0,
// as in the reference.
void ddgmres(const OrcMat& A, const double* alo, const DdPrecon& P, const OrcParams& prm, const double* bh,
             const double* bl, double* xh, double* xl, double* hist, int* niter, int* iret) {
  const long n = A.n;
  const int m = prm.GMRES_m > 0 ? prm.GMRES_m : 4;
  const int gs = prm.GMRES_GSflag > 0 ? prm.GMRES_GSflag : ORC_GS_MGS;
  std::vector<double> rh(n), rl(n), Vh((long)(m + 1) * n, 0.0), Vl((long)(m + 1) * n, 0.0), pvh(n), pvl(n),
      wh(n), wl(n), x0h(n), x0l(n), v0h(n), v0l(n);
  std::vector<DD> h((long)(m + 1) * m), c(m + 1), s(m + 1), e(m + 1), y(m + 1);
  const DD one{1.0, 0.0}, mone{-1.0, 0.0}, zero{0.0, 0.0};
  const DD bnorm = dd_sqrt(dd_dot(n, bh, bl, bh, bl));
  double rnorm = 0.0;
  int itr = 1, inner = 1, mm = 0;
  for (itr = 1; itr <= prm.itrmax; itr += m) {
    std::fill(e.begin(), e.end(), zero); std::fill(c.begin(), c.end(), zero);
    std::fill(s.begin(), s.end(), zero); std::fill(y.begin(), y.end(), zero);
    std::fill(h.begin(), h.end(), zero);
    dd_spmv(A, alo, xh, xl, rh.data(), rl.data());                        // ddcalc_res
    dd_axpy(n, one, mone, bh, bl, rh.data(), rl.data());
    const DD rn = dd_sqrt(dd_dot(n, rh.data(), rl.data(), rh.data(), rl.data()));
    dd_axpy(n, dd_div(mone, rn), zero, rh.data(), rl.data(), Vh.data(), Vl.data());   // v_1 = -r / |r|
    e[0] = dd_mul(mone, rn);
    rnorm = rn.hi;
    if (itr == 1) hist[itr - 1] = rnorm / bnorm.hi;
    bool exit_inner = false;
    for (inner = 1; inner <= m; ++inner) {
      const long off = (long)(inner - 1) * n;
      dd_apply_precon(A, alo, P, Vh.data() + off, Vl.data() + off, pvh.data(), pvl.data());
      dd_spmv(A, alo, pvh.data(), pvl.data(), wh.data(), wl.data());
      DD* col = h.data() + (long)(inner - 1) * (m + 1);
      if (gs == ORC_GS_MGS) {
        for (int k = 1; k < inner; ++k) {
          const long ok = (long)(k - 1) * n;
          col[k - 1] = dd_dot(n, wh.data(), wl.data(), Vh.data() + ok, Vl.data() + ok);
          dd_axpy(n, dd_mul(mone, col[k - 1]), one, Vh.data() + ok, Vl.data() + ok, wh.data(), wl.data());
        }
      } else {
        for (int k = 1; k < inner; ++k) {
          const long ok = (long)(k - 1) * n;
          col[k - 1] = dd_dot(n, Vh.data() + ok, Vl.data() + ok, wh.data(), wl.data());
        }
        for (int k = 1; k < inner; ++k) {
          const long ok = (long)(k - 1) * n;
          dd_axpy(n, dd_mul(mone, col[k - 1]), one, Vh.data() + ok, Vl.data() + ok, wh.data(), wl.data());
        }
      }
      col[inner - 1] = dd_dot(n, wh.data(), wl.data(), Vh.data() + off, Vl.data() + off);
      dd_axpy(n, dd_mul(mone, col[inner - 1]), one, Vh.data() + off, Vl.data() + off, wh.data(), wl.data());
      col[inner] = dd_sqrt(dd_dot(n, wh.data(), wl.data(), wh.data(), wl.data()));
      const long on = (long)inner * n;
      dd_axpy(n, dd_div(one, col[inner]), zero, wh.data(), wl.data(), Vh.data() + on, Vl.data() + on);
      dd_givens(m, h.data(), inner, c.data(), s.data(), e.data());
      rnorm = std::fabs(e[inner].hi);
      mm = inner;
      if (itr + inner <= prm.itrmax) hist[itr + inner - 1] = rnorm / bnorm.hi;
      if (rnorm / bnorm.hi < prm.rtolmax || itr + inner == prm.itrmax) { exit_inner = true; break; }
    }
    if (!exit_inner) inner = m + 1;             // Fortran DO variable after completion
    if (m < mm) mm = m;
    // ddupdate_xVec (ddpgmres.f90:52-145): y = H^-1 e, v0 = V y, x = M^-1 v0 + x
    for (int i = mm; i >= 1; --i) {
      y[i - 1] = e[i - 1];
      for (int j = mm; j >= i + 1; --j)
        y[i - 1] = dd_sub(y[i - 1], dd_mul(h[(i - 1) + (long)(j - 1) * (m + 1)], y[j - 1]));
      const DD d = h[(i - 1) + (long)(i - 1) * (m + 1)];
      y[i - 1] = (d.hi == 0.0 && d.lo == 0.0) ? dd_div(y[i - 1], DD{1.0e-100, 0.0}) : dd_div(y[i - 1], d);
    }
#pragma omp parallel for schedule(static)
    for (long j = 0; j < n; ++j) {               // ddsum_vec (ddpgmres.f90:7-50)
      DD t{0.0, 0.0};
      for (int i = 0; i < mm; ++i) t = dd_add(t, dd_mul(y[i], DD{Vh[(long)i * n + j], Vl[(long)i * n + j]}));
      v0h[j] = t.hi;
      v0l[j] = t.lo;
    }
    dd_apply_precon(A, alo, P, v0h.data(), v0l.data(), x0h.data(), x0l.data());
    dd_axpy(n, one, one, x0h.data(), x0l.data(), xh, xl);
    if (rnorm / bnorm.hi < prm.rtolmax) break;
    if (itr + inner == prm.itrmax) break;
  }
  *niter = std::min(prm.itrmax, itr + inner);
  *iret = (prm.itrmax <= itr) ? 1 : 0;
}

// ---------------------------------------------------------------------------------
// C entry points used by the tests and the CPU-baseline leg of bench.py.
extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int t) {
#ifdef _OPENMP
  if (t > 0) omp_set_num_threads(t);
#else
  (void)t;
#endif
}

// Explicit block-Jacobi blocks for the following calls: starts[0..nb] (0-based, starts[0]
// = 0, starts[nb] = n, increasing); nb = 0 returns to the equal split.
int orc_set_blocks(int nb, const long* starts) {
  g_blk.clear();
  if (nb <= 0) return 0;
  if (!starts || starts[0] != 0) return ORC_E_ARG;
  for (int b = 0; b < nb; ++b)
    if (starts[b + 1] <= starts[b]) return ORC_E_ARG;
  g_blk.assign(starts, starts + nb + 1);
  return 0;
}

void orc_spmv(const OrcMat* A, const double* x, double* y) { spmv(*A, x, y); }

double orc_dot(long n, const double* x, const double* y) { return dot(n, x, y); }

// Applies the preconditioner set up from prm to r (one call = setup + one application).
int orc_precon_apply(const OrcMat* A, const OrcParams* prm, const double* r, double* s) {
  Precon P;
  int err = setup_precon(*A, *prm, P);
  if (err) return err;
  apply_precon(P, r, s);
  return 0;
}

// Returns the inverse diagonal used by point Jacobi or D-ILU (n entries).
int orc_precon_dinv(const OrcMat* A, const OrcParams* prm, double* dinv) {
  Precon P;
  int err = setup_precon(*A, *prm, P);
  if (err) return err;
  if (P.Dinv.empty()) return ORC_E_ARG;
  std::memcpy(dinv, P.Dinv.data(), sizeof(double) * A->n);
  return 0;
}

// Full solve.  x holds x0 on entry and the solution on exit; hist has itrmax entries.
int orc_solve(const OrcMat* A, const OrcParams* prm, const double* b, double* x,
              double* hist, int* niter, int* iret) {
  if (!A || !prm || A->n <= 0) return ORC_E_ARG;
  Precon P;
  int err = setup_precon(*A, *prm, P);
  if (err) { *iret = err; *niter = 0; return err; }
  switch (prm->solver) {
    case ORC_SOLVER_CG: pcg(*A, P, *prm, b, x, hist, niter, iret); break;
    case ORC_SOLVER_BICG: pbicg(*A, P, *prm, b, x, hist, niter, iret); break;
    case ORC_SOLVER_GMRES: pgmres(*A, P, *prm, b, x, hist, niter, iret); break;
    default: return ORC_E_UNSUPPORTED;
  }
  return 0;
}

// True residual ||b - A x|| / ||b||.
double orc_true_relres(const OrcMat* A, const double* b, const double* x) {
  std::vector<double> r(A->n);
  residual(*A, x, b, r.data());
  return std::sqrt(dot(A->n, r.data(), r.data())) / std::sqrt(dot(A->n, b, b));
}

// Persistent preconditioner for the numpy CA-GMRES oracle (oracle/cagmres.py).
void* orc_precon_create(const OrcMat* A, const OrcParams* prm, int* err) {
  Precon* P = new Precon();
  int e = setup_precon(*A, *prm, *P);
  if (err) *err = e;
  if (e) { delete P; return nullptr; }
  return P;
}

void orc_precon_apply_h(void* h, const double* r, double* s) {
  apply_precon(*static_cast<Precon*>(h), r, s);
}

void orc_precon_destroy(void* h) { delete static_cast<Precon*>(h); }

// ddKSP_pCG (prm->solver 1) or ddKSP_pBiCG (2) through PARCEL_ddKSP_CRS's precision flags
// (ddwrapper.f90:184-280):
// prec_A/b/x/M = 1 (double) or 2 (double-double).  A low parts (alo), b low parts and the
// initial x low parts may be null.  ipreflag 0 / 1 / 2-3 (D-ILU, ILU_method 1 or 2).
int orc_ddcg(const OrcMat* A, const double* alo, const OrcParams* prm, int prec_A, int prec_b, int prec_x,
             int prec_M, const double* bh, const double* bl, double* xh, double* xl, double* hist, int* niter,
             int* iret) {
  const long n = A->n;
  std::vector<double> bl0(n, 0.0), xl0(n, 0.0);
  if (prec_b == 2 && bl) std::copy(bl, bl + n, bl0.begin());
  if (prec_x == 2 && xl) std::copy(xl, xl + n, xl0.begin());
  const double* a_lo = (prec_A == 2) ? alo : nullptr;
  DdPrecon P;
  P.prec = prec_M;
  int kind = prm->ipreflag == ORC_PRECON_AS ? ORC_PRECON_BJ : prm->ipreflag;
  P.kind = kind;
  P.method = prm->ILU_method < 0 ? ORC_ILUD : prm->ILU_method;
  if (kind == ORC_PRECON_PJ) {
    dd_setup_pj(*A, a_lo, P);
  } else if (kind == ORC_PRECON_BJ) {
    if (P.method == ORC_ILU0) return ORC_E_UNSUPPORTED;
    if (!g_blk.empty() && g_blk.back() != n) return ORC_E_ARG;
    int err = dd_setup_dilu(*A, a_lo, nblocks_for(*A, prm->precon_thblock), P.method, P);
    if (err) return err;
  } else if (kind != ORC_PRECON_NONE) {
    return ORC_E_UNSUPPORTED;
  }
  if (prm->solver == ORC_SOLVER_BICG)
    ddbicg(*A, a_lo, P, *prm, bh, bl0.data(), xh, xl0.data(), hist, niter, iret);
  else if (prm->solver == ORC_SOLVER_GMRES)
    ddgmres(*A, a_lo, P, *prm, bh, bl0.data(), xh, xl0.data(), hist, niter, iret);
  else
    ddpcg(*A, a_lo, P, *prm, bh, bl0.data(), xh, xl0.data(), hist, niter, iret);
  if (prec_x == 2 && xl) std::copy(xl0.begin(), xl0.end(), xl);
  return 0;
}

}  // extern "C"
