// pb_mixed.cuh -- mixed-precision refinement, double-double residual and CA-GMRES.
#pragma once

#include "pb_solvers.cuh"

namespace pb {

// r = b - A x in double-double (ddcalc_res_CRS, src/ddkrylov.f90:1281-1310: ddMatVec_crs
// then ddaxpy with alpha = 1, beta = -1).  val_lo / x_lo / b_lo may be null (zero).
void residual_dd(const DevMat<double>& A, const double* val_lo, const double* x_hi,
                 const double* x_lo, const double* b_hi, const double* b_lo, double* r_hi,
                 double* r_lo, cudaStream_t st);

struct MixedResult {
  int niter = 0;
  int iret = 0;
  int launches = 0;
  int refine_steps = 0;
  double true_relres = 0.0;
  double true_relres_dd = 0.0;
  int ilu_levels_max = 0;
  int ilu_nblocks = 0;
};

// FP32 Krylov solves (PCG / BiCGStab / GMRES with an FP32 block-Jacobi ILU or Jacobi
// preconditioner) inside an FP64 iterative-refinement loop whose residual is computed in
// FP64 or double-double.  b, x: natural-layout device arrays; x in/out.
// `attach`, if given, is called once on the FP32 system after it is built (it may set
// S.extra, which turns the inner GMRES into flexible GMRES).
MixedResult solve_mixed(const Options& o, const parcel_b_crs& A, bool dev, const double* b,
                        double* x, std::vector<double>& hist, double* setup_t,
                        const std::function<void(System<float>&)>* attach = nullptr);

// The same refinement loop on an FP32 system that is already built (several right-hand
// sides share one set-up).
MixedResult solve_mixed_on(const Options& o, System<float>& S, const double* b, double* x,
                           std::vector<double>& hist, double* setup_t);

// CA-GMRES(s, t) (KSP_pCAGMRES, src/pcagmres.f90:1557-2518) in FP64.
SolveOut solve_cagmres(const Options& o, System<double>& S, const double* b, double* x,
                       std::vector<double>& hist, double* setup_t);

template <class T>
double dev_dot(int64_t n, const T* x, const T* y);

}  // namespace pb
