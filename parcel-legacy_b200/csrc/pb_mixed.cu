// pb_mixed.cu -- mixed-precision iterative refinement and the double-double residual.
//
// The reference offers FP64 Krylov solvers and CPU-only double-double ones
// (ddKSP_CRS forces the CPU, src/ddkrylov.f90:81,207).  This file adds the B200 path:
// the Krylov iteration and the block-Jacobi ILU run in FP32 (half the bytes of the
// HBM-bound kernels) on correction equations A d = r, and an outer loop keeps x in FP64
// and recomputes r = b - A x in FP64 or in double-double with the reference's dd
// operation order, until the FP64 true relative residual meets rtolmax.
#include <cmath>

#include "pb_device.cuh"
#include "pb_mixed.cuh"

namespace pb {

__global__ void k_residual_dd(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                              const double* __restrict__ va, const double* __restrict__ va_lo,
                              int rbase, int cbase, const double* __restrict__ xh,
                              const double* __restrict__ xl, const double* __restrict__ bh,
                              const double* __restrict__ bl, double* __restrict__ rh,
                              double* __restrict__ rl) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    dd t{0.0, 0.0};
    for (int j = rp[i] - rbase; j < rp[i + 1] - rbase; ++j) {
      int c = ci[j] - cbase;
      dd a{va[j], va_lo ? va_lo[j] : 0.0};
      dd xv{xh[c], xl ? xl[c] : 0.0};
      t = dd_add(dd_mul(a, xv), t);           // ddMatVec_crs: ddadd(c, tmp, tmp)
    }
    dd bb = dd_mul(dd{1.0, 0.0}, dd{bh[i], bl ? bl[i] : 0.0});   // ddaxpy, vec.f90 ddvec:14-54
    dd cc = dd_mul(dd{-1.0, 0.0}, t);
    dd r = dd_add(bb, cc);
    rh[i] = r.hi;
    rl[i] = r.lo;
  }
}

void residual_dd(const DevMat<double>& A, const double* val_lo, const double* x_hi,
                 const double* x_lo, const double* b_hi, const double* b_lo, double* r_hi,
                 double* r_lo, cudaStream_t st) {
  int grid = std::max(1, std::min((A.n + 255) / 256, 8 * num_sms()));
  k_residual_dd<<<grid, 256, 0, st>>>(A.n, A.rowptr, A.col, A.val, val_lo, A.rbase, A.cbase, x_hi,
                                      x_lo, b_hi, b_lo, r_hi, r_lo);
  PB_CUDA(cudaGetLastError());
}

MixedResult solve_mixed(const Options& o, const parcel_b_crs& A, bool dev, const double* b,
                        double* x, std::vector<double>& hist, double* setup_t,
                        const std::function<void(System<float>&)>* attach) {
  System<float> S;
  build_system<float>(o, A, dev, S);
  if (attach) (*attach)(S);
  return solve_mixed_on(o, S, b, x, hist, setup_t);
}

MixedResult solve_mixed_on(const Options& o, System<float>& S, const double* b, double* x,
                           std::vector<double>& hist, double* setup_t) {
  cudaStream_t st = stream();
  MixedResult res;
  res.ilu_levels_max = S.ilu_levels_max;
  res.ilu_nblocks = S.ilu_nblocks;
  const int n = S.n, np = S.np;
  DBuf r(sizeof(double) * n), rlo(sizeof(double) * n), d64(sizeof(double) * n);
  DBuf r32(sizeof(float) * np), d32(sizeof(float) * np);
  DBuf hist_dev(sizeof(double) * (o.itrmax + 2));
  PB_CUDA(cudaMemsetAsync(r32.p, 0, sizeof(float) * np, st));
  const double bnorm = std::sqrt(dev_dot<double>(n, b, b));
  sync();
  if (setup_t) *setup_t = now_s();
  Options oi = o;
  oi.rtol = o.inner_rtol;
  int total = 0;
  hist.clear();
  double rel = 1.0;
  bool converged = false;
  for (int k = 0; k < o.max_refine; ++k) {
    if (o.residual_dd) {
      residual_dd(S.Anat, nullptr, x, nullptr, b, nullptr, dp<double>(r), dp<double>(rlo), st);
    } else {
      spmv<double, double>(S.Anat, x, dp<double>(r), SPMV_RES, b, nullptr, st);
    }
    res.launches += 1;
    const double rn = std::sqrt(dev_dot<double>(n, dp<double>(r), dp<double>(r)));
    rel = rn / bnorm;
    res.refine_steps = k;
    if (!(rel == rel)) { res.iret = PARCEL_B_E_BREAKDOWN; break; }
    if (rel < o.rtol) { converged = true; break; }
    if (total >= o.itrmax) break;
    // inner correction solve A d = r in FP32, x0 = 0
    if (S.permuted) scatter_perm<float>(n, dp<float>(r32), dp<double>(r), dp<int>(S.pos), st);
    else convert<float, double>(n, dp<float>(r32), dp<double>(r), st);
    PB_CUDA(cudaMemsetAsync(d32.p, 0, sizeof(float) * np, st));
    oi.itrmax = o.itrmax - total;
    trace_mark("refine: outer residual");
    SolveOut so = run_krylov<float>(oi, S, dp<float>(r32), dp<float>(d32), dp<double>(hist_dev));
    trace_mark("refine: inner solve");
    res.launches += so.launches + 2;
    if (so.niter > 0) {
      std::vector<double> h(so.niter);
      d2h(h.data(), hist_dev.p, sizeof(double) * so.niter);
      for (double v : h) hist.push_back(rel * v);
    }
    total += so.niter;
    if (S.permuted) gather_perm<float>(n, dp<double>(d64), dp<float>(d32), dp<int>(S.pos), st);
    else convert<double, float>(n, dp<double>(d64), dp<float>(d32), st);
    lincomb<double>(n, x, dp<double>(d64), cimm(1.0), x, cimm(1.0), nullptr, cimm(0.0), nullptr, st);
    res.launches += 2;
    if (so.iret < 0) { res.iret = so.iret; break; }
  }
  res.niter = total;
  if (res.iret == 0) res.iret = converged ? 0 : 1;
  // final true residuals in FP64 and double-double
  spmv<double, double>(S.Anat, x, dp<double>(r), SPMV_RES, b, nullptr, st);
  res.true_relres = std::sqrt(dev_dot<double>(n, dp<double>(r), dp<double>(r))) / bnorm;
  residual_dd(S.Anat, nullptr, x, nullptr, b, nullptr, dp<double>(r), dp<double>(rlo), st);
  res.true_relres_dd = std::sqrt(dev_dot<double>(n, dp<double>(r), dp<double>(r))) / bnorm;
  return res;
}

}  // namespace pb
