// pb_solvers.cuh -- solver drivers (pb_solvers.cu).
#pragma once

#include <chrono>
#include <functional>
#include <memory>

#include "pb_blas.cuh"
#include "pb_ilu.cuh"
#include "pb_spmv.cuh"

namespace pb {

// Resolved options (KSP_INPUT_PARAM after PARCEL_KSP_Default_Setting, type.f90:949-1132).
struct Options {
  int solver = PARCEL_B_SOLVER_GMRES;
  int precon = PARCEL_B_PRECON_NONE;
  int ilu_method = PARCEL_B_ILUD;
  int nblocks = 1;
  int m = 4;
  int gs = PARCEL_B_GS_MGS;
  int itrmax = 100;
  double rtol = 1e-8;
  double abstol = 0.0;
  int sstep = 4, tstep = 1, basis = PARCEL_B_BASIS_MONOMIAL, qrflag = PARCEL_B_QR_CHOLQR;
  int inner = PARCEL_B_INNER_FP64;
  int residual_dd = 0;
  double inner_rtol = 1e-4;
  int max_refine = 50;
  int independ_nvec = 1;
  std::vector<int> block_starts;                       // explicit block-Jacobi blocks (BlockSplit)
  bool use_graphs = true;
  bool fused_mgs = true;
  bool flexible = false;                               // GMRES: flexible variant (keeps M^-1 v_j)
  const std::function<void(int)>* on_cycle = nullptr;  // GMRES: called after each restart cycle
};

Options resolve_options(const parcel_b_input* p);

// The block-Jacobi blocks of an n-row solve: o.block_starts when given (checked: rising
// from 0 to n), else divide_region's split into min(o.nblocks, n) blocks.
BlockSplit block_split(const Options& o, int n);

// Explicit block starts for every resolve_options on this thread while the guard lives
// (a stencil-format solve hands its boxes to the CRS solvers this way).
struct ScopedBlockStarts {
  explicit ScopedBlockStarts(const std::vector<int>* starts);
  ~ScopedBlockStarts();
  ScopedBlockStarts(const ScopedBlockStarts&) = delete;
  ScopedBlockStarts& operator=(const ScopedBlockStarts&) = delete;
};

// Preconditioner on iteration-layout vectors.
template <class T>
struct Precon {
  int kind = PARCEL_B_PRECON_NONE;
  DBuf dinv;
  IluDev<T> ilu;
  int launches_per_apply() const { return 1; }
  void apply(int64_t np, const T* r, T* s, const int* gate, cudaStream_t st) const;
};

template <class T>
struct System;

// An extra preconditioner stage around M (flexible GMRES only): begin(r) is called before
// z = M^-1 r is launched (work that does not need z may start on a side stream there),
// apply(r, z) after it: z <- z + stage(r, z).  If az is not null and provides_az() is
// true, the stage also writes A z there (when it can do so without an SpMV of its own),
// and the caller skips its SpMV of z.
template <class T>
struct ExtraStage {
  virtual ~ExtraStage() = default;
  virtual void begin(const System<T>&, const T*, const int*, cudaStream_t) {}
  virtual void apply(const System<T>& S, const T* r, T* z, T* az, const int* gate, cudaStream_t st) = 0;
  virtual bool provides_az() const { return true; }
  virtual int launches() const = 0;
};

// Everything a solve needs on the device, in the iteration layout.
template <class T>
struct System {
  int n = 0;            // natural rows
  int np = 0;           // iteration-layout length
  int64_t nnz = 0;
  bool permuted = false;
  DevMat<double> Anat;  // natural matrix (reference layout)
  DBuf up_rowptr, up_col, up_val;   // uploaded copies of host inputs
  SellBuf<T> Asell;     // sliced-ELLPACK copy used by the SpMV
  DevMat<T> A;          // matrix of the iteration
  DBuf Aval_T;          // natural values cast to T (FP32 path, no permutation)
  DBuf pos, rowAt, lev; // layout maps (block Jacobi)
  Precon<T> M;
  ExtraStage<T>* extra = nullptr;   // not owned
  int ilu_levels_max = 0;
  int ilu_nblocks = 0;
  int spmv_diagonals = 0;           // > 0: the SpMV runs on a diagonal copy (natural layout)
};

template <class T>
void build_system(const Options& o, const parcel_b_crs& A, bool dev, System<T>& S);

struct SolveOut {
  int niter = 0;
  int iret = 0;
  int launches = 0;
  int breakdown = 0;
};

// Runs the Krylov iteration on iteration-layout vectors x (in/out) and b.  hist_dev has
// itrmax+1 entries on the device.
template <class T>
SolveOut run_krylov(const Options& o, const System<T>& S, const T* b, T* x, double* hist_dev);

// Workspace shared by the drivers.
struct Workspace {
  DBuf part, ticket, state;
  Red red(int epi) const;
  KState* st() const { return dp<KState>(state); }
  void init();
};

double now_s();

}  // namespace pb
