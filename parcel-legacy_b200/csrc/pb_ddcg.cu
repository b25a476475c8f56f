// pb_ddcg.cu -- double-double preconditioned CG, BiCGStab and GMRES(m) on the GPU
// (PARCEL_ddKSP_CRS, solvers 1, 2 and 3).
//
// Reference: ddKSP_pCG (src/ddpcg.f90:247-563), ddKSP_pBiCG (src/ddpbicg.f90:496-875) and
// ddKSP_pGMRES (src/ddpgmres.f90:254-713) with the precision flags of
// PARCEL_ddKSP_CRS (src/ddwrapper.f90:184-280): A, b, x and the preconditioner each in
// double (1) or double-double (2).  The reference runs its dd solvers on the CPU only
// (src/ddkrylov.f90:81,207); this is a GPU implementation of the same arithmetic.
//
// Every dd operation is the reference's sequence of explicitly rounded double operations
// (pb_device.cuh), every per-row loop runs in the reference's order (the CRS order for the
// SpMV, L start..end and U start down to end for the D-ILU sweeps, the D-ILU diagonal
// recurrence of ddDILU_DInv_crs), and the dot products sum in a fixed order (32,768
// contiguous chunks in index order, their sums in 256 groups, the group sums in order), so
// the solve is bit-for-bit reproducible and identical to the CPU oracle's restatement.
// The D-ILU rows run level by level on the wavefront plan of the FP64 block-Jacobi path;
// the level order changes no row's arithmetic.
#include <cstring>
#include <vector>

#include "pb_api.cuh"
#include "pb_device.cuh"
#include "pb_ilu.cuh"

namespace pb {

namespace {

constexpr int kDdStreams = 1 << 17;                 // dot-product streams (the oracle uses the same order)
constexpr int kDdDotThreads = 256;
constexpr int kDdDotCtas = kDdStreams / kDdDotThreads;   // 512
constexpr int kDdThreads = 256;

#define GRID_LOOP(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

inline int grid_for(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kDdThreads - 1) / kDdThreads, 8LL * num_sms()));
}

// Scalars of the iteration, on the device.
struct DdScal {
  dd bnorm, rnorm, rho0, rho1, gamma, alpha, beta, t1;
};

// ------------------------------------------------------------------ vector kernels
// y = A x: per row, c = a_ij x_j and t = c + t in CRS order (ddMatVec_crs, single process).
__global__ void k_dd_spmv(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ ah, const double* __restrict__ al, int cbase,
                          const double* __restrict__ xh, const double* __restrict__ xl, double* __restrict__ yh,
                          double* __restrict__ yl) {
  GRID_LOOP(i, n) {
    dd t{0.0, 0.0};
    for (int j = rp[i] - 1; j < rp[i + 1] - 1; ++j) {
      const int c = ci[j] - cbase;
      t = dd_add(dd_mul(dd{ah[j], al ? al[j] : 0.0}, dd{xh[c], xl[c]}), t);
    }
    yh[i] = t.hi;
    yl[i] = t.lo;
  }
}

// ddaxpy (ddvec.f90:14-54): y = alpha x + beta y, the scalars read from the device.
__global__ void k_dd_axpy(int n, const dd* alpha, const dd* beta, const double* __restrict__ xh,
                          const double* __restrict__ xl, double* __restrict__ yh, double* __restrict__ yl) {
  const dd a = *alpha, b = *beta;
  GRID_LOOP(i, n) {
    const dd c = dd_mul(b, dd{yh[i], yl[i]});
    const dd t = dd_mul(a, dd{xh[i], xl[i]});
    const dd y = dd_add(t, c);
    yh[i] = y.hi;
    yl[i] = y.lo;
  }
}

// ddCG_axpy2 (ddpcg.f90:9-59): x = x + alpha p, p = s + beta p.
__global__ void k_dd_cg_axpy2(int n, const DdScal* sc, double* __restrict__ xh, double* __restrict__ xl,
                              double* __restrict__ ph, double* __restrict__ pl, const double* __restrict__ sh,
                              const double* __restrict__ sl) {
  const dd a = sc->alpha, b = sc->beta;
  GRID_LOOP(i, n) {
    const dd p = dd{ph[i], pl[i]};
    const dd x = dd_add(dd{xh[i], xl[i]}, dd_mul(a, p));
    const dd q = dd_add(dd{sh[i], sl[i]}, dd_mul(b, p));
    xh[i] = x.hi;
    xl[i] = x.lo;
    ph[i] = q.hi;
    pl[i] = q.lo;
  }
}

// Dot product in a fixed order: stream t (0 <= t < 2^17) sums the products of the elements
// i = t, t + 2^17, ... in increasing i, from zero; the 2^17 stream sums are combined by a
// complete binary tree (level by level, neighbours in pairs: s'[k] = s[2k] + s[2k+1]).
// One launch: thread t of the grid owns stream t, so every load is coalesced; each CTA
// folds its 256 streams (an aligned subtree) in shared memory and stores its sum; the last
// CTA to finish (an atomic ticket, no waiting) folds the 512 CTA sums and stores the result.
// The ticket counter is reset by that CTA for the next dot on the stream.
__device__ __forceinline__ void dd_tree(dd* v, int count) {
  // v[0..count) -> v[0], count a power of two, all threads of the CTA taking part
  for (int h = count >> 1; h > 0; h >>= 1) {
    dd r{0.0, 0.0};
    for (int k = threadIdx.x; k < h; k += blockDim.x) r = dd_add(v[2 * k], v[2 * k + 1]);
    __syncthreads();
    for (int k = threadIdx.x; k < h; k += blockDim.x) v[k] = r;   // h <= blockDim.x after the first level
    __syncthreads();
  }
}

__global__ void __launch_bounds__(kDdDotThreads) k_dd_dot(int64_t n, const double* __restrict__ xh,
                                                        const double* __restrict__ xl, const double* __restrict__ yh,
                                                        const double* __restrict__ yl, dd* part, unsigned* ticket,
                                                        dd* out) {
  __shared__ dd tr[2 * kDdDotThreads];
  __shared__ bool last;
  const int64_t t = (int64_t)blockIdx.x * kDdDotThreads + threadIdx.x;
  dd s{0.0, 0.0};
  int64_t i = t;
  for (; i + 3 * (int64_t)kDdStreams < n; i += 4 * (int64_t)kDdStreams) {
    double ah[4], al[4], bh[4], bl[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int64_t q = i + u * (int64_t)kDdStreams;
      ah[u] = xh[q]; al[u] = xl[q]; bh[u] = yh[q]; bl[u] = yl[q];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) s = dd_add(s, dd_mul(dd{ah[u], al[u]}, dd{bh[u], bl[u]}));
  }
  for (; i < n; i += kDdStreams) s = dd_add(s, dd_mul(dd{xh[i], xl[i]}, dd{yh[i], yl[i]}));
  tr[threadIdx.x] = s;
  __syncthreads();
  dd_tree(tr, kDdDotThreads);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = tr[0];
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int k = threadIdx.x; k < kDdDotCtas; k += kDdDotThreads) {
    const double2 v = __ldcg(reinterpret_cast<const double2*>(part + k));
    tr[k] = dd{v.x, v.y};
  }
  __syncthreads();
  dd_tree(tr, kDdDotCtas);
  if (threadIdx.x == 0) {
    *out = tr[0];
    *ticket = 0u;
  }
}

enum DdStep { DD_INIT_NORMS = 0, DD_INIT_RHO, DD_ALPHA, DD_RNORM, DD_BETA };

// Scalar updates of ddKSP_pCG, one thread.
__global__ void k_dd_scal(DdScal* sc, int step, const dd* bdot, const dd* rdot) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  switch (step) {
    case DD_INIT_NORMS:
      sc->bnorm = dd_sqrt(*bdot);
      sc->rnorm = dd_sqrt(*rdot);
      sc->alpha = dd{0.0, 0.0};
      sc->beta = dd{0.0, 0.0};
      break;
    case DD_INIT_RHO:
      sc->rho0 = *bdot;
      break;
    case DD_ALPHA:
      sc->gamma = *bdot;
      sc->alpha = dd_div(sc->rho0, sc->gamma);
      sc->t1 = dd_mul(dd{-1.0, 0.0}, sc->alpha);
      break;
    case DD_RNORM:
      sc->rho1 = *bdot;
      sc->rnorm = dd_sqrt(*rdot);
      break;
    case DD_BETA:
      sc->beta = dd_div(sc->rho1, sc->rho0);
      sc->rho0 = sc->rho1;
      break;
  }
}

// ------------------------------------------------------------------ BiCGStab (ddKSP_pBiCG)
// Scalars of ddKSP_pBiCG (ddpbicg.f90:496-875); hist = high part of dd_div(rnorm, bnorm).
struct DdScalB {
  dd bnorm, rnorm, c1, c2, c3, alpha, beta;
  double hist;
};

enum DdStepB { DDB_INIT = 0, DDB_ALPHA, DDB_C3, DDB_RNORM, DDB_BETA };

__global__ void k_dd_scal_b(DdScalB* sc, int step, const dd* d1, const dd* d2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  switch (step) {
    case DDB_INIT:   // d1 = <b, b>, d2 = <r0, r0>
      sc->bnorm = dd_sqrt(*d1);
      sc->c1 = *d2;
      sc->rnorm = dd_sqrt(sc->c1);
      sc->hist = dd_div(sc->rnorm, sc->bnorm).hi;
      sc->c2 = dd{0.0, 0.0};
      sc->c3 = dd{0.0, 0.0};
      break;
    case DDB_ALPHA:   // d1 = <r0, q>
      sc->c2 = *d1;
      sc->alpha = dd_div(sc->c1, sc->c2);
      break;
    case DDB_C3:   // d1 = <e, v>, d2 = <v, v>
      sc->c3 = dd_div(*d1, *d2);
      break;
    case DDB_RNORM:   // d1 = <r, r0>, d2 = <r, r>
      sc->c1 = *d1;
      sc->rnorm = dd_sqrt(*d2);
      sc->hist = dd_div(sc->rnorm, sc->bnorm).hi;
      break;
    case DDB_BETA:
      sc->beta = dd_div(sc->c1, dd_mul(sc->c3, sc->c2));
      break;
  }
}

// ddBiCG_axpy3 (ddpbicg.f90:8-43): e = r - alpha q
__global__ void k_dd_bicg_axpy3(int n, const DdScalB* sc, const double* __restrict__ rh, const double* __restrict__ rl,
                                const double* __restrict__ qh, const double* __restrict__ ql, double* __restrict__ eh,
                                double* __restrict__ el) {
  const dd a = sc->alpha;
  GRID_LOOP(i, n) {
    const dd e = dd_sub(dd{rh[i], rl[i]}, dd_mul(a, dd{qh[i], ql[i]}));
    eh[i] = e.hi;
    el[i] = e.lo;
  }
}

// ddBiCG_axpy4 (ddpbicg.f90:282-326): x = x + (alpha pp + c3 pe)
__global__ void k_dd_bicg_axpy4(int n, const DdScalB* sc, double* __restrict__ xh, double* __restrict__ xl,
                                const double* __restrict__ pph, const double* __restrict__ ppl,
                                const double* __restrict__ peh, const double* __restrict__ pel) {
  const dd a = sc->alpha, c3 = sc->c3;
  GRID_LOOP(i, n) {
    dd c = dd_mul(c3, dd{peh[i], pel[i]});
    const dd b = dd_mul(a, dd{pph[i], ppl[i]});
    c = dd_add(b, c);
    const dd x = dd_add(dd{xh[i], xl[i]}, c);
    xh[i] = x.hi;
    xl[i] = x.lo;
  }
}

// ddBiCG_axpy3_dot's update (ddpbicg.f90:95-279): r = e - c3 v (its two dot products
// follow as separate fixed-order dots)
__global__ void k_dd_bicg_axpy3r(int n, const DdScalB* sc, const double* __restrict__ eh, const double* __restrict__ el,
                                 const double* __restrict__ vh, const double* __restrict__ vl, double* __restrict__ rh,
                                 double* __restrict__ rl) {
  const dd c3 = sc->c3;
  GRID_LOOP(i, n) {
    const dd r = dd_sub(dd{eh[i], el[i]}, dd_mul(c3, dd{vh[i], vl[i]}));
    rh[i] = r.hi;
    rl[i] = r.lo;
  }
}

// ddBiCG_axpy4_ (ddpbicg.f90:46-90): p = r + beta (p - c3 q)
__global__ void k_dd_bicg_axpy4p(int n, const DdScalB* sc, double* __restrict__ ph, double* __restrict__ pl,
                                 const double* __restrict__ rh, const double* __restrict__ rl,
                                 const double* __restrict__ qh, const double* __restrict__ ql) {
  const dd c3 = sc->c3, beta = sc->beta;
  GRID_LOOP(i, n) {
    dd c = dd_mul(c3, dd{qh[i], ql[i]});
    c = dd_sub(dd{ph[i], pl[i]}, c);
    c = dd_mul(beta, c);
    const dd p = dd_add(dd{rh[i], rl[i]}, c);
    ph[i] = p.hi;
    pl[i] = p.lo;
  }
}

// ------------------------------------------------------------------ GMRES (ddKSP_pGMRES)
// Small state of ddKSP_pGMRES (ddpgmres.f90:254-713), on the device: the (m+1) x m
// Hessenberg matrix (column-major), the rotations c and s, the rotated right-hand side e
// and the update coefficients y.
struct DdGm {
  int m = 0;
  dd* h = nullptr;
  dd* c = nullptr;
  dd* s = nullptr;
  dd* e = nullptr;
  dd* y = nullptr;
  dd* bnorm = nullptr;
  dd* t1 = nullptr;       // the scale of the next basis vector
  double* rn = nullptr;   // the residual norm's high part, read by the host
};

enum DdStepG { DDG_BNORM = 0, DDG_START, DDG_NORM, DDG_SOLVE };

// ddGivensRotations (ddpgmres.f90:147-250) on column i (1-based).
__device__ void dd_givens(const DdGm& g, int i) {
  dd* col = g.h + (int64_t)(i - 1) * (g.m + 1);
  dd* c = g.c;
  dd* s = g.s;
  dd* e = g.e;
  for (int k = 1; k <= i - 1; ++k) {
    const dd t1 = dd_sub(dd_mul(col[k - 1], c[k - 1]), dd_mul(col[k], s[k - 1]));
    const dd t2 = dd_add(dd_mul(col[k - 1], s[k - 1]), dd_mul(col[k], c[k - 1]));
    col[k - 1] = t1;
    col[k] = t2;
  }
  const dd d = col[i - 1];
  const dd t = (d.hi == 0.0 && d.lo == 0.0) ? dd_div(col[i], dd{1.0e-100, 0.0}) : dd_div(col[i], d);
  const dd q = dd_sqrt(dd_add(dd{1.0, 0.0}, dd_mul(t, t)));
  c[i - 1] = dd_div(dd{1.0, 0.0}, q);
  s[i - 1] = dd_mul(dd{-1.0, 0.0}, dd_mul(c[i - 1], t));
  const dd e1 = dd_sub(dd_mul(c[i - 1], e[i - 1]), dd_mul(s[i - 1], e[i]));
  const dd e2 = dd_add(dd_mul(s[i - 1], e[i - 1]), dd_mul(c[i - 1], e[i]));
  e[i - 1] = e1;
  e[i] = e2;
  col[i - 1] = dd_sub(dd_mul(c[i - 1], col[i - 1]), dd_mul(s[i - 1], col[i]));
  col[i] = dd{0.0, 0.0};
}

// Scalar steps of ddKSP_pGMRES, one thread.  DDG_START: d = <r, r> of the restart
// residual; DDG_NORM: d = <w, w> for column i, then the rotation of that column;
// DDG_SOLVE: y = H^-1 e over the first i columns (ddupdate_xVec, ddpgmres.f90:98-118).
__global__ void k_dd_gm_scal(DdGm g, int step, int i, const dd* d) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int ld = g.m + 1;
  switch (step) {
    case DDG_BNORM:
      *g.bnorm = dd_sqrt(*d);
      break;
    case DDG_START: {
      for (int k = 0; k < ld * g.m; ++k) g.h[k] = dd{0.0, 0.0};
      for (int k = 0; k < ld; ++k) g.c[k] = g.s[k] = g.e[k] = g.y[k] = dd{0.0, 0.0};
      const dd rn = dd_sqrt(*d);
      *g.t1 = dd_div(dd{-1.0, 0.0}, rn);
      g.e[0] = dd_mul(dd{-1.0, 0.0}, rn);
      *g.rn = rn.hi;
      break;
    }
    case DDG_NORM: {
      dd* col = g.h + (int64_t)(i - 1) * ld;
      col[i] = dd_sqrt(*d);
      *g.t1 = dd_div(dd{1.0, 0.0}, col[i]);
      dd_givens(g, i);
      *g.rn = fabs(g.e[i].hi);
      break;
    }
    case DDG_SOLVE:
      for (int r = i; r >= 1; --r) {
        dd y = g.e[r - 1];
        for (int j = i; j >= r + 1; --j) y = dd_sub(y, dd_mul(g.h[(r - 1) + (int64_t)(j - 1) * ld], g.y[j - 1]));
        const dd dg = g.h[(r - 1) + (int64_t)(r - 1) * ld];
        g.y[r - 1] = (dg.hi == 0.0 && dg.lo == 0.0) ? dd_div(y, dd{1.0e-100, 0.0}) : dd_div(y, dg);
      }
      break;
  }
}

// w = (-h) v + 1 w with h read from the device (the projection step of
// ddMGS_Orthonormalization, ddQRDecomposition.f90:27-44).
__global__ void k_dd_axpy_nh(int n, const dd* hk, const double* __restrict__ vh, const double* __restrict__ vl,
                             double* __restrict__ wh, double* __restrict__ wl) {
  const dd a = dd_mul(dd{-1.0, 0.0}, *hk), b = dd{1.0, 0.0};
  GRID_LOOP(i, n) {
    const dd c = dd_mul(b, dd{wh[i], wl[i]});
    const dd t = dd_mul(a, dd{vh[i], vl[i]});
    const dd w = dd_add(t, c);
    wh[i] = w.hi;
    wl[i] = w.lo;
  }
}

// The subtractions of ddCGS_Orthonormalization (ddQRDecomposition.f90:73-86),
// w = (-h_k) v_k + 1 w for k = 1..cnt in that order, in one pass over w and the basis.
__global__ void k_dd_cgs_sub(int n, int cnt, const dd* hcol, const double* __restrict__ Vh,
                             const double* __restrict__ Vl, int64_t ldv, double* __restrict__ wh,
                             double* __restrict__ wl) {
  const dd b = dd{1.0, 0.0};
  GRID_LOOP(i, n) {
    dd w = dd{wh[i], wl[i]};
    for (int k = 0; k < cnt; ++k) {
      const dd a = dd_mul(dd{-1.0, 0.0}, hcol[k]);
      const dd c = dd_mul(b, w);
      const dd t = dd_mul(a, dd{Vh[k * ldv + i], Vl[k * ldv + i]});
      w = dd_add(t, c);
    }
    wh[i] = w.hi;
    wl[i] = w.lo;
  }
}

// ddsum_vec (ddpgmres.f90:7-50): v0 = sum_k y_k v_k, k in order, from 0.
__global__ void k_dd_sum_vec(int n, int mm, const dd* y, const double* __restrict__ Vh,
                             const double* __restrict__ Vl, int64_t ldv, double* __restrict__ v0h,
                             double* __restrict__ v0l) {
  GRID_LOOP(i, n) {
    dd t{0.0, 0.0};
    for (int k = 0; k < mm; ++k) t = dd_add(t, dd_mul(y[k], dd{Vh[k * ldv + i], Vl[k * ldv + i]}));
    v0h[i] = t.hi;
    v0l[i] = t.lo;
  }
}

// ------------------------------------------------------------------ preconditioners
// ddget_DInv_crs (ddmatrix.f90:283-349): 1 / a_ii, a zero pivot replaced by 1e-100.
__global__ void k_dd_pj_dinv(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                             const double* __restrict__ ah, const double* __restrict__ al, int cbase,
                             double* __restrict__ dh, double* __restrict__ dl) {
  GRID_LOOP(k, n) {
    for (int j = rp[k] - 1; j < rp[k + 1] - 1; ++j)
      if (ci[j] - cbase == k) {
        const dd a{ah[j], al ? al[j] : 0.0};
        const dd d = (a.hi == 0.0 && a.lo == 0.0) ? dd_div(dd{1.0, 0.0}, dd{1.0e-100, 0.0})
                                                  : dd_div(dd{1.0, 0.0}, a);
        dh[k] = d.hi;
        dl[k] = d.lo;
      }
  }
}

// ddpointJacobi (ddmatrix.f90:3523-3567): s = D^-1 r; precision 1 drops D^-1's low part.
__global__ void k_dd_pj_apply(int n, const double* __restrict__ dh, const double* __restrict__ dl, int prec,
                              const double* __restrict__ rh, const double* __restrict__ rl, double* __restrict__ sh,
                              double* __restrict__ sl) {
  GRID_LOOP(i, n) {
    const dd z = dd_mul(dd{dh[i], prec == 2 ? dl[i] : 0.0}, dd{rh[i], rl[i]});
    sh[i] = z.hi;
    sl[i] = z.lo;
  }
}

__global__ void k_dd_copy(int n, const double* __restrict__ rh, const double* __restrict__ rl,
                          double* __restrict__ sh, double* __restrict__ sl) {
  GRID_LOOP(i, n) {
    sh[i] = rh[i];
    sl[i] = rl[i];
  }
}

// In-block L / U ranges of every row (the sweeps of ddsolve_ILU_crs): forward j = Ls..Le,
// backward j = Us down to Ue (0-based positions).
__global__ void k_dd_ranges(int n, int nb, const int* __restrict__ blk_lo, const int* __restrict__ blk_hi,
                            const int* __restrict__ blk_of, const int* __restrict__ rp, const int* __restrict__ ci,
                            int cbase, int4* __restrict__ rng) {
  GRID_LOOP(k, n) {
    const int b = blk_of[k];
    const int lo = blk_lo[b], hi = blk_hi[b];
    const int a = rp[k] - 1, z = rp[k + 1] - 1;
    int Ls = z - 1, Le = a, Us = a, Ue = z - 1;
    for (int j = a; j < z; ++j)
      if (ci[j] - cbase >= lo) { Ls = j; break; }
    for (int j = a; j < z; ++j) {
      const int c = ci[j] - cbase;
      if (c < lo) continue;
      if (c >= k) { Le = j - 1; break; }
    }
    for (int j = z - 1; j >= a; --j)
      if (ci[j] - cbase <= hi - 1) { Us = j; break; }
    for (int j = z - 1; j >= a; --j)
      if (ci[j] - cbase <= k) { Ue = j + 1; break; }
    rng[k] = make_int4(Ls, Le, Us, Ue);
  }
}

// ddDILU_DInv_crs (ddmatrix.f90:1451-1640), independ_nvec = 1, one CTA per block, level by
// level: D_k = a_kk - sum over the lower in-block entries a_kr (kr < k) of a_kr a_rk / D_r
// (ILUD: the entry of row r in column k only; MLUD: every entry of row r right of r), then
// D^-1 = 1 / D (a zero D replaced by 1e-100).
__global__ void k_dd_dilu_diag(const IluChunk* __restrict__ ch, const int* __restrict__ blk_chunk,
                               const int* __restrict__ blk_lo, const int* __restrict__ blk_hi,
                               const int* __restrict__ rowAt, const int* __restrict__ rp,
                               const int* __restrict__ ci, const double* __restrict__ ah,
                               const double* __restrict__ al, int cbase, int mlud, double* Dh, double* Dl,
                               double* __restrict__ dih, double* __restrict__ dil) {
  const int b = blockIdx.x;
  const int lo = blk_lo[b], hi = blk_hi[b];
  auto av = [&](int j) { return dd{ah[j], al ? al[j] : 0.0}; };
  for (int c = blk_chunk[b]; c < blk_chunk[b + 1]; ++c) {
    const IluChunk C = ch[c];
    for (int p = threadIdx.x; p < C.w; p += blockDim.x) {
      const int k = rowAt[C.start + p];
      dd D{0.0, 0.0};
      int jstart = -1;
      for (int j = rp[k] - 1; j < rp[k + 1] - 1; ++j) {
        const int col = ci[j] - cbase;
        if (col < lo || col >= hi) continue;
        if (jstart == -1) jstart = j;
        if (col < k) continue;
        D = col == k ? av(j) : dd{0.0, 0.0};
        for (int jr = jstart; jr < j; ++jr) {
          const int kr = ci[jr] - cbase;
          const dd Dr{Dh[kr], Dl[kr]};
          for (int i = rp[kr] - 1; i < rp[kr + 1] - 1; ++i) {
            const int rc = ci[i] - cbase;
            if (rc < lo) continue;
            if (rc >= hi) break;
            const bool take = mlud ? kr < rc : rc == k;
            if (!take) continue;
            dd t = dd_mul(av(jr), av(i));
            t = (Dr.hi == 0.0 && Dr.lo == 0.0) ? dd_div(t, dd{1.0e-100, 0.0}) : dd_div(t, Dr);
            D = dd_sub(D, t);
            if (!mlud) break;
          }
        }
        break;
      }
      Dh[k] = D.hi;
      Dl[k] = D.lo;
      const dd di = (D.hi == 0.0 && D.lo == 0.0) ? dd_div(dd{1.0, 0.0}, dd{1.0e-100, 0.0})
                                                 : dd_div(dd{1.0, 0.0}, D);
      dih[k] = di.hi;
      dil[k] = di.lo;
    }
    __syncthreads();
  }
}

// ddsolve_ILU_crs (ddmatrix.f90:4310-4680), independ_nvec = 1, one CTA per block, the
// forward levels in order then the backward levels in reverse:
//   forward  z = r_k - sum_{j=Ls..Le} s_c a_j,  s_k = z D^-1
//   backward z = sum_{j=Us..Ue, descending} s_c a_j,  s_k = s_k - D^-1 z
// Precision 1 drops the low parts of A and of D^-1 (baked into the row records).
//
// Each row's data sits in level order (position q of the wavefront layout): its natural
// index, its first kPre couplings (column and value) in the loop order above, its
// coupling count and first position (for couplings past kPre, read from the CRS), its
// D^-1, and its input (r for the forward sweep; the forward result, written in level order
// as well, for the backward sweep).  So everything a level needs except the values s_c of
// the rows it depends on is read by position, independent of earlier levels, and the next
// level's part is loaded before the current level's barrier: after the barrier only the
// gathers of s_c, the dd chain and the stores remain.
constexpr int kPre = 3;       // couplings per row held in the records
constexpr int kRowsPer = 2;   // rows per thread staged ahead (levels of up to 512 rows)
constexpr int kDdRingBytes = 160 * 1024;   // largest shared-memory ring of the sweep

struct DdRecords {
  int np = 0;
  const int* k;             // natural row at position q, -1 = padding
  const int* rs;            // ring slot of the row at position q (ring mode)
  const int2* nj[2];        // [fwd, bwd]: (coupling count, first position)
  const int* col[2];        // [dir][t * np + q]: natural column, or its ring slot (ring mode)
  const double* ah[2];
  const double* al[2];
  const double* dh;         // D^-1 at q (low part 0 under precision 1)
  const double* dl;
};

__global__ void k_dd_records(int np, const int* __restrict__ rowAt, const int4* __restrict__ rng,
                             const int* __restrict__ ci, const double* __restrict__ ah, const double* __restrict__ al,
                             int cbase, const double* __restrict__ dih, const double* __restrict__ dil, int prec,
                             const int* __restrict__ rslot, int* rk, int* rs, int2* nj0, int2* nj1, int* c0, int* c1,
                             double* a0h, double* a0l, double* a1h, double* a1l, double* rdh, double* rdl) {
  GRID_LOOP(q, np) {
    const int k = rowAt[q];
    rk[q] = k;
    rs[q] = (rslot && k >= 0) ? rslot[k] : 0;
    if (k < 0) {
      nj0[q] = make_int2(0, 0);
      nj1[q] = make_int2(0, 0);
      rdh[q] = 0.0;
      rdl[q] = 0.0;
      continue;
    }
    const int4 r = rng[k];
    const int nf = max(0, r.y - r.x + 1), nb = max(0, r.z - r.w + 1);
    nj0[q] = make_int2(nf, r.x);
    nj1[q] = make_int2(nb, r.z);
    for (int t = 0; t < kPre; ++t) {
      const int64_t o = (int64_t)t * np + q;
      if (t < nf) {
        const int j = r.x + t;
        c0[o] = rslot ? rslot[ci[j] - cbase] : ci[j] - cbase;
        a0h[o] = ah[j];
        a0l[o] = (prec == 2 && al) ? al[j] : 0.0;
      }
      if (t < nb) {
        const int j = r.z - t;
        c1[o] = rslot ? rslot[ci[j] - cbase] : ci[j] - cbase;
        a1h[o] = ah[j];
        a1l[o] = (prec == 2 && al) ? al[j] : 0.0;
      }
    }
    rdh[q] = dih[k];
    rdl[q] = prec == 2 ? dil[k] : 0.0;
  }
}

// r in level order (padding positions 0).
__global__ void k_dd_gather(int np, const int* __restrict__ rk, const double* __restrict__ xh,
                            const double* __restrict__ xl, double* __restrict__ qh, double* __restrict__ ql) {
  GRID_LOOP(q, np) {
    const int k = rk[q];
    qh[q] = k >= 0 ? xh[k] : 0.0;
    ql[q] = k >= 0 ? xl[k] : 0.0;
  }
}

struct DdStage {
  int k[kRowsPer], n[kRowsPer], j0[kRowsPer], q[kRowsPer], rs[kRowsPer];
  int col[kRowsPer][kPre];
  dd a[kRowsPer][kPre];
  dd x[kRowsPer], di[kRowsPer];
};

template <int DIR>
__device__ __forceinline__ void dd_stage(DdStage& S, const IluChunk& C, const DdRecords& R, const double* xh,
                                         const double* xl) {
#pragma unroll
  for (int u = 0; u < kRowsPer; ++u) {
    const int p = threadIdx.x + u * blockDim.x;
    S.k[u] = -1;
    if (p < C.w) {
      const int q = C.start + p;
      S.q[u] = q;
      S.k[u] = R.k[q];
      S.rs[u] = R.rs[q];
      const int2 nj = R.nj[DIR][q];
      S.n[u] = nj.x;
      S.j0[u] = nj.y;
#pragma unroll
      for (int t = 0; t < kPre; ++t)
        if (t < nj.x) {
          const int64_t o = (int64_t)t * R.np + q;
          S.col[u][t] = R.col[DIR][o];
          S.a[u][t] = dd{R.ah[DIR][o], R.al[DIR][o]};
        }
      S.x[u] = dd{xh[q], xl[q]};
      S.di[u] = dd{R.dh[q], R.dl[q]};
    }
  }
}

// ringh / ringl: the shared-memory ring of the last W levels' results (RING), indexed by the
// records' slots; otherwise the staged couplings read the natural-order output sh / sl.
template <int DIR, bool RING>
__device__ __forceinline__ dd dd_row(int k, int n, int j0, const int* col, const dd* a, dd x, dd di,
                                     const int* __restrict__ ci, const double* __restrict__ ah,
                                     const double* __restrict__ al, int cbase, int prec, const double* sh,
                                     const double* sl, const double* ringh, const double* ringl) {
  dd z = DIR == 0 ? x : dd{0.0, 0.0};
#pragma unroll
  for (int t = 0; t < kPre; ++t)
    if (t < n) {
      const dd v = RING ? dd_mul(dd{ringh[col[t]], ringl[col[t]]}, a[t]) : dd_mul(dd{sh[col[t]], sl[col[t]]}, a[t]);
      z = DIR == 0 ? dd_sub(z, v) : dd_add(z, v);
    }
  for (int t = kPre; t < n; ++t) {   // couplings past the records, straight from the CRS
    const int j = DIR == 0 ? j0 + t : j0 - t;
    const int c = ci[j] - cbase;
    const dd v = dd_mul(dd{sh[c], sl[c]}, dd{ah[j], (prec == 2 && al) ? al[j] : 0.0});
    z = DIR == 0 ? dd_sub(z, v) : dd_add(z, v);
  }
  (void)k;
  return DIR == 0 ? dd_mul(z, di) : dd_sub(x, dd_mul(di, z));
}

// The rows of one level: the staged ones, then any past kRowsPer per thread.
template <int DIR, bool RING>
__device__ __forceinline__ void dd_level(const DdStage& S, const IluChunk& C, const DdRecords& R, const double* xh,
                                         const double* xl, const int* __restrict__ ci, const double* __restrict__ ah,
                                         const double* __restrict__ al, int cbase, int prec, double* sh, double* sl,
                                         double* fqh, double* fql, double* ringh, double* ringl) {
#pragma unroll
  for (int u = 0; u < kRowsPer; ++u) {
    const int k = S.k[u];
    if (k < 0) continue;
    const dd s = dd_row<DIR, RING>(k, S.n[u], S.j0[u], S.col[u], S.a[u], S.x[u], S.di[u], ci, ah, al, cbase, prec, sh,
                                   sl, ringh, ringl);
    if (RING) {
      ringh[S.rs[u]] = s.hi;
      ringl[S.rs[u]] = s.lo;
    }
    sh[k] = s.hi;
    sl[k] = s.lo;
    if (DIR == 0) {
      fqh[S.q[u]] = s.hi;
      fql[S.q[u]] = s.lo;
    }
  }
  for (int p = threadIdx.x + kRowsPer * blockDim.x; p < C.w; p += blockDim.x) {
    const int q = C.start + p;
    const int k = R.k[q];
    const int2 nj = R.nj[DIR][q];
    int col[kPre];
    dd a[kPre];
#pragma unroll
    for (int t = 0; t < kPre; ++t)
      if (t < nj.x) {
        const int64_t o = (int64_t)t * R.np + q;
        col[t] = R.col[DIR][o];
        a[t] = dd{R.ah[DIR][o], R.al[DIR][o]};
      }
    const dd s = dd_row<DIR, RING>(k, nj.x, nj.y, col, a, dd{xh[q], xl[q]}, dd{R.dh[q], R.dl[q]}, ci, ah, al, cbase,
                                   prec, sh, sl, ringh, ringl);
    if (RING) {
      ringh[R.rs[q]] = s.hi;
      ringl[R.rs[q]] = s.lo;
    }
    sh[k] = s.hi;
    sl[k] = s.lo;
    if (DIR == 0) {
      fqh[q] = s.hi;
      fql[q] = s.lo;
    }
  }
}

// RING: the results of the last W levels also go to a shared-memory ring (ring_rows slots),
// from which the staged couplings are read: a level's dependency gathers are then
// shared-memory loads instead of L2 round trips.
template <bool RING>
__global__ void __launch_bounds__(256, 1)
    k_dd_dilu_sweep(const IluChunk* __restrict__ ch, const int* __restrict__ blk_chunk, DdRecords R,
                    const int* __restrict__ ci, const double* __restrict__ ah, const double* __restrict__ al, int cbase,
                    int prec, const double* __restrict__ rqh, const double* __restrict__ rql, double* fqh, double* fql,
                    double* sh, double* sl, int ring_rows) {
  extern __shared__ double ringbuf[];
  double* ringh = ringbuf;
  double* ringl = ringbuf + ring_rows;
  const int b = blockIdx.x;
  const int c0 = blk_chunk[b], c1 = blk_chunk[b + 1];
  if (c1 <= c0) return;
  DdStage A, B;
  // forward: input r in level order; the results also go to level order for the backward
  dd_stage<0>(A, ch[c0], R, rqh, rql);
  for (int c = c0; c < c1; ++c) {
    const IluChunk C = ch[c];
    if (c + 1 < c1) dd_stage<0>(B, ch[c + 1], R, rqh, rql);
    dd_level<0, RING>(A, C, R, rqh, rql, ci, ah, al, cbase, prec, sh, sl, fqh, fql, ringh, ringl);
    __syncthreads();
    A = B;
  }
  // backward: input the forward result (complete after the barrier above)
  dd_stage<1>(A, ch[c1 - 1], R, fqh, fql);
  for (int c = c1 - 1; c >= c0; --c) {
    const IluChunk C = ch[c];
    if (c - 1 >= c0) dd_stage<1>(B, ch[c - 1], R, fqh, fql);
    dd_level<1, RING>(A, C, R, fqh, fql, ci, ah, al, cbase, prec, sh, sl, nullptr, nullptr, ringh, ringl);
    __syncthreads();
    A = B;
  }
}

__global__ void k_block_of(int nb, const int* __restrict__ blk_lo, const int* __restrict__ blk_hi, int* blk_of) {
  const int b = blockIdx.x;
  if (b >= nb) return;
  for (int k = blk_lo[b] + threadIdx.x; k < blk_hi[b]; k += blockDim.x) blk_of[k] = b;
}

// ------------------------------------------------------------------ host side
struct DdVec {
  DBuf h, l;
  explicit DdVec(int n) : h(sizeof(double) * std::max(n, 1)), l(sizeof(double) * std::max(n, 1)) {}
  double* hi() const { return dp<double>(h); }
  double* lo() const { return dp<double>(l); }
};

struct DdPrecon {
  int kind = PARCEL_B_PRECON_NONE;
  int prec = 2;
  DBuf dih, dil;                        // D^-1 (point Jacobi, D-ILU)
  DBuf chunks, blk_chunk, rowAt, rng;   // D-ILU level plan and row ranges
  int nb = 0, np = 0;
  DBuf rk, rs, nj0, nj1, c0, c1, a0h, a0l, a1h, a1l, rdh, rdl;   // level-ordered row records
  int ring_rows = 0;                                               // > 0: the sweep's shared-memory ring
  DBuf rqh, rql, fqh, fql;                                     // r and the forward result in level order
  DdRecords rec() const {
    DdRecords R;
    R.np = np;
    R.k = dp<int>(rk);
    R.rs = dp<int>(rs);
    R.nj[0] = dp<int2>(nj0);
    R.nj[1] = dp<int2>(nj1);
    R.col[0] = dp<int>(c0);
    R.col[1] = dp<int>(c1);
    R.ah[0] = dp<double>(a0h);
    R.al[0] = dp<double>(a0l);
    R.ah[1] = dp<double>(a1h);
    R.al[1] = dp<double>(a1l);
    R.dh = dp<double>(rdh);
    R.dl = dp<double>(rdl);
    return R;
  }
};

// Device copy of a natural-layout array given by host or device pointer (null stays null).
struct Arr {
  DBuf own;
  const void* p = nullptr;
  Arr(const void* src, size_t bytes) {
    if (!src) return;
    if (is_device_ptr(src)) { p = src; return; }
    own.alloc(bytes);
    h2d(own.p, src, bytes);
    p = own.p;
  }
};

struct DdSystem {
  int n = 0, cbase = 1;
  const int* rp = nullptr;
  const int* ci = nullptr;
  const double* ah = nullptr;
  const double* al = nullptr;   // null: A's low parts are zero
};

// part: kDdDotCtas CTA sums followed by the ticket counter (zero between dots).
void dd_dot(const DdSystem& S, const double* xh, const double* xl, const double* yh, const double* yl, dd* part,
            dd* out, cudaStream_t st) {
  k_dd_dot<<<kDdDotCtas, kDdDotThreads, 0, st>>>(S.n, xh, xl, yh, yl, part,
                                                reinterpret_cast<unsigned*>(part + kDdDotCtas), out);
}

void dd_setup_precon(const Options& o, const parcel_b_crs& A, const DdSystem& S, int prec_M, DdPrecon& P) {
  cudaStream_t st = stream();
  P.kind = o.precon == PARCEL_B_PRECON_ADDITIVESCHWARZ ? PARCEL_B_PRECON_BLOCKJACOBI : o.precon;
  P.prec = prec_M;
  if (P.kind == PARCEL_B_PRECON_NONE) return;
  P.dih.alloc(sizeof(double) * S.n);
  P.dil.alloc(sizeof(double) * S.n);
  if (P.kind == PARCEL_B_PRECON_POINTJACOBI) {
    k_dd_pj_dinv<<<grid_for(S.n), kDdThreads, 0, st>>>(S.n, S.rp, S.ci, S.ah, S.al, S.cbase, dp<double>(P.dih),
                                                        dp<double>(P.dil));
    PB_CUDA(cudaGetLastError());
    return;
  }
  PB_CHECK(P.kind == PARCEL_B_PRECON_BLOCKJACOBI, PARCEL_B_E_UNSUPPORTED,
           "ipreflag=%d: the dd CG provides none, point Jacobi and block Jacobi", o.precon);
  PB_CHECK(o.ilu_method == 1 || o.ilu_method == 2, PARCEL_B_E_UNSUPPORTED,
           "ILU_method=%d: the dd CG's block-Jacobi preconditioner is D-ILU (1 or 2)", o.ilu_method);
  // wavefront plan on the host (the structure comes back from the device if it lives there)
  std::vector<int> hrp, hci;
  const int* hrpp = A.rowptr;
  const int* hcip = A.col;
  if (is_device_ptr(A.rowptr)) {
    hrp.resize((size_t)A.n + 1);
    hci.resize((size_t)A.nnz);
    d2h(hrp.data(), A.rowptr, sizeof(int) * hrp.size());
    d2h(hci.data(), A.col, sizeof(int) * hci.size());
    hrpp = hrp.data();
    hcip = hci.data();
  }
  HostCSR H;
  H.n = A.n; H.nnz = A.nnz; H.istart = A.istart; H.rowptr = hrpp; H.col = hcip;
  std::vector<int> pos(A.n), lev(A.n);
  IluPlan plan;
  ilu_build_plan(H, block_split(o, A.n), plan, pos.data(), lev.data());
  P.nb = plan.nb;
  P.chunks.alloc(sizeof(IluChunk) * std::max<size_t>(plan.chunks.size(), 1));
  h2d(P.chunks.p, plan.chunks.data(), sizeof(IluChunk) * plan.chunks.size());
  P.blk_chunk.alloc(sizeof(int) * (plan.nb + 1));
  h2d(P.blk_chunk.p, plan.blk_chunk.data(), sizeof(int) * (plan.nb + 1));
  DBuf dpos(sizeof(int) * A.n), blo(sizeof(int) * plan.nb), bhi(sizeof(int) * plan.nb), bof(sizeof(int) * A.n);
  h2d(dpos.p, pos.data(), sizeof(int) * A.n);
  h2d(blo.p, plan.blk_lo.data(), sizeof(int) * plan.nb);
  h2d(bhi.p, plan.blk_hi.data(), sizeof(int) * plan.nb);
  P.rowAt.alloc(sizeof(int) * plan.np);
  PB_CUDA(cudaMemsetAsync(P.rowAt.p, 0xFF, sizeof(int) * plan.np, st));
  scatter_positions(A.n, dp<int>(dpos), dp<int>(P.rowAt), st);
  k_block_of<<<plan.nb, 256, 0, st>>>(plan.nb, dp<int>(blo), dp<int>(bhi), dp<int>(bof));
  P.rng.alloc(sizeof(int4) * A.n);
  k_dd_ranges<<<grid_for(A.n), kDdThreads, 0, st>>>(A.n, plan.nb, dp<int>(blo), dp<int>(bhi), dp<int>(bof), S.rp,
                                                     S.ci, S.cbase, dp<int4>(P.rng));
  DBuf Dh(sizeof(double) * A.n), Dl(sizeof(double) * A.n);
  k_dd_dilu_diag<<<plan.nb, ilu_factor_threads(plan.maxWp), 0, st>>>(dp<IluChunk>(P.chunks), dp<int>(P.blk_chunk), dp<int>(blo),
                                                 dp<int>(bhi), dp<int>(P.rowAt), S.rp, S.ci, S.ah, S.al, S.cbase,
                                                 o.ilu_method == 2 ? 1 : 0, dp<double>(Dh), dp<double>(Dl),
                                                 dp<double>(P.dih), dp<double>(P.dil));
  PB_CUDA(cudaGetLastError());
  const int np = plan.np;
  P.np = np;
  // ring: slot of natural row c = (level % W) * LW + (position - the level's first position),
  // LW the widest level; used when its hi and lo parts fit kDdRingBytes of shared memory
  const int LW = plan.maxWp;   // the widest level (rows, rounded up to 4)
  const int64_t ring_rows = (int64_t)plan.W * LW;
  DBuf drs;
  if (ring_rows > 0 && 2 * ring_rows * (int64_t)sizeof(double) <= kDdRingBytes) {
    std::vector<int> rslot(A.n);
    for (int b = 0; b < plan.nb; ++b)
      for (int c = plan.blk_lo[b]; c < plan.blk_hi[b]; ++c) {
        const int l = lev[c];
        rslot[c] = (l % plan.W) * LW + (pos[c] - plan.lvl_start[plan.blk_lvl[b] + l]);
      }
    drs.alloc(sizeof(int) * A.n);
    h2d(drs.p, rslot.data(), sizeof(int) * A.n);
    P.ring_rows = (int)ring_rows;
  }
  const size_t nq = (size_t)np, nt = (size_t)kPre * np;
  P.rk.alloc(sizeof(int) * nq);
  P.rs.alloc(sizeof(int) * nq);
  P.nj0.alloc(sizeof(int2) * nq);
  P.nj1.alloc(sizeof(int2) * nq);
  P.c0.alloc(sizeof(int) * nt);
  P.c1.alloc(sizeof(int) * nt);
  for (DBuf* d : {&P.a0h, &P.a0l, &P.a1h, &P.a1l}) d->alloc(sizeof(double) * nt);
  for (DBuf* d : {&P.rdh, &P.rdl, &P.rqh, &P.rql, &P.fqh, &P.fql}) d->alloc(sizeof(double) * nq);
  k_dd_records<<<grid_for(np), kDdThreads, 0, st>>>(np, dp<int>(P.rowAt), dp<int4>(P.rng), S.ci, S.ah, S.al, S.cbase,
                                                     dp<double>(P.dih), dp<double>(P.dil), prec_M,
                                                     P.ring_rows ? dp<int>(drs) : nullptr, dp<int>(P.rk),
                                                     dp<int>(P.rs), dp<int2>(P.nj0), dp<int2>(P.nj1), dp<int>(P.c0), dp<int>(P.c1),
                                                     dp<double>(P.a0h), dp<double>(P.a0l), dp<double>(P.a1h),
                                                     dp<double>(P.a1l), dp<double>(P.rdh), dp<double>(P.rdl));
  PB_CUDA(cudaGetLastError());
  sync();   // the temporaries above are released on return
}

void dd_apply_precon(const DdSystem& S, const DdPrecon& P, const double* rh, const double* rl, double* sh,
                     double* sl, cudaStream_t st) {
  switch (P.kind) {
    case PARCEL_B_PRECON_NONE:
      k_dd_copy<<<grid_for(S.n), kDdThreads, 0, st>>>(S.n, rh, rl, sh, sl);
      break;
    case PARCEL_B_PRECON_POINTJACOBI:
      k_dd_pj_apply<<<grid_for(S.n), kDdThreads, 0, st>>>(S.n, dp<double>(P.dih), dp<double>(P.dil), P.prec, rh,
                                                          rl, sh, sl);
      break;
    default:
      k_dd_gather<<<grid_for(P.np), kDdThreads, 0, st>>>(P.np, dp<int>(P.rk), rh, rl, dp<double>(P.rqh),
                                                          dp<double>(P.rql));
      if (P.ring_rows) {
        static bool attr = false;
        if (!attr) {
          PB_CUDA(cudaFuncSetAttribute(k_dd_dilu_sweep<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       kDdRingBytes));
          attr = true;
        }
        k_dd_dilu_sweep<true><<<P.nb, kDdThreads, 2 * sizeof(double) * P.ring_rows, st>>>(
            dp<IluChunk>(P.chunks), dp<int>(P.blk_chunk), P.rec(), S.ci, S.ah, S.al, S.cbase, P.prec,
            dp<double>(P.rqh), dp<double>(P.rql), dp<double>(P.fqh), dp<double>(P.fql), sh, sl, P.ring_rows);
      } else {
        k_dd_dilu_sweep<false><<<P.nb, kDdThreads, 0, st>>>(dp<IluChunk>(P.chunks), dp<int>(P.blk_chunk), P.rec(),
                                                            S.ci, S.ah, S.al, S.cbase, P.prec, dp<double>(P.rqh),
                                                            dp<double>(P.rql), dp<double>(P.fqh), dp<double>(P.fql),
                                                            sh, sl, 0);
      }
      break;
  }
}

}  // namespace

}  // namespace pb

using namespace pb;

namespace {

// What the dd solver loops share: the system, the preconditioner, the stream, the dot
// scratch and the constants 1, -1 and 0 on the device.
struct DdRun {
  const DdSystem& S;
  const DdPrecon& P;
  cudaStream_t st;
  int n, g;
  dd* part;
  dd* one;
  dd* mone;
  dd* zero;
  void spmv(const double* xh, const double* xl, double* yh, double* yl) const {
    k_dd_spmv<<<g, kDdThreads, 0, st>>>(n, S.rp, S.ci, S.ah, S.al, S.cbase, xh, xl, yh, yl);
  }
  void spmv(const DdVec& x, DdVec& y) const { spmv(x.hi(), x.lo(), y.hi(), y.lo()); }
  void dot(const double* xh, const double* xl, const double* yh, const double* yl, dd* out) const {
    dd_dot(S, xh, xl, yh, yl, part, out, st);
  }
  void dot(const DdVec& u, const DdVec& v, DBuf& out) const { dot(u.hi(), u.lo(), v.hi(), v.lo(), dp<dd>(out)); }
  // y = alpha x + beta y (ddaxpy)
  void axpy(const dd* alpha, const dd* beta, const double* xh, const double* xl, double* yh, double* yl) const {
    k_dd_axpy<<<g, kDdThreads, 0, st>>>(n, alpha, beta, xh, xl, yh, yl);
  }
  void precon(const double* rh, const double* rl, double* sh, double* sl) const {
    dd_apply_precon(S, P, rh, rl, sh, sl, st);
  }
  // r = b - A x (ddcalc_res: r = A x, then r = 1 b + (-1) r)
  void residual(const DdVec& x, const DdVec& b, DdVec& r) const {
    spmv(x, r);
    axpy(one, mone, b.hi(), b.lo(), r.hi(), r.lo());
  }
};

struct DdLoop {
  int used = 0, iret = 0;
  double setup_end = 0.0;
};

double read_double(const double* dev, cudaStream_t st) {
  double v;
  PB_CUDA(cudaMemcpyAsync(&v, dev, sizeof(double), cudaMemcpyDeviceToHost, st));
  PB_CUDA(cudaStreamSynchronize(st));
  return v;
}

// ddKSP_pCG (ddpcg.f90:247-563).
DdLoop dd_cg_loop(const DdRun& R, const Options& o, DdVec& x, const DdVec& b, double* reshistory) {
  const int n = R.n, g = R.g;
  cudaStream_t st = R.st;
  DdLoop L;
  DdVec r(n), p(n), q(n), s(n);
  DBuf scal(sizeof(DdScal)), d1(sizeof(dd)), d2(sizeof(dd));
  DdScal* sc = dp<DdScal>(scal);
  R.residual(x, b, r);
  R.dot(b, b, d1);
  R.dot(r, r, d2);
  k_dd_scal<<<1, 32, 0, st>>>(sc, DD_INIT_NORMS, dp<dd>(d1), dp<dd>(d2));
  R.precon(r.hi(), r.lo(), s.hi(), s.lo());
  R.dot(s, r, d1);
  k_dd_scal<<<1, 32, 0, st>>>(sc, DD_INIT_RHO, dp<dd>(d1), nullptr);
  PB_CUDA(cudaGetLastError());
  L.setup_end = now_s();
  DdScal h;
  PB_CUDA(cudaMemcpyAsync(&h, sc, sizeof(DdScal), cudaMemcpyDeviceToHost, st));
  sync();
  const double bnorm = h.bnorm.hi;
  double rnorm = h.rnorm.hi;
  int itr;
  for (itr = 1; itr <= o.itrmax; ++itr) {
    if (reshistory) reshistory[itr - 1] = rnorm / bnorm;
    k_dd_cg_axpy2<<<g, kDdThreads, 0, st>>>(n, sc, x.hi(), x.lo(), p.hi(), p.lo(), s.hi(), s.lo());
    R.spmv(p, q);
    R.dot(p, q, d1);
    k_dd_scal<<<1, 32, 0, st>>>(sc, DD_ALPHA, dp<dd>(d1), nullptr);
    R.axpy(&sc->t1, R.one, q.hi(), q.lo(), r.hi(), r.lo());
    R.precon(r.hi(), r.lo(), s.hi(), s.lo());
    R.dot(s, r, d1);
    R.dot(r, r, d2);
    k_dd_scal<<<1, 32, 0, st>>>(sc, DD_RNORM, dp<dd>(d1), dp<dd>(d2));
    PB_CUDA(cudaGetLastError());
    rnorm = read_double(&sc->rnorm.hi, st);
    if (rnorm / bnorm < o.rtol) break;
    k_dd_scal<<<1, 32, 0, st>>>(sc, DD_BETA, nullptr, nullptr);
  }
  // x = alpha p + 1 x
  R.axpy(&sc->alpha, R.one, p.hi(), p.lo(), x.hi(), x.lo());
  PB_CUDA(cudaGetLastError());
  L.used = std::min(o.itrmax, itr);
  L.iret = (o.itrmax <= itr) ? 1 : 0;
  return L;
}

// ddKSP_pBiCG (ddpbicg.f90:496-875): r0 = p = r, c1 = <r0, r0>.
DdLoop dd_bicg_loop(const DdRun& R, const Options& o, DdVec& x, const DdVec& b, double* reshistory) {
  const int n = R.n, g = R.g;
  cudaStream_t st = R.st;
  DdLoop L;
  DdVec r(n), p(n), q(n), r0(n), pp(n), e(n), pe(n), v(n);
  DBuf scb(sizeof(DdScalB)), d1(sizeof(dd)), d2(sizeof(dd));
  DdScalB* sb = dp<DdScalB>(scb);
  R.residual(x, b, r);
  k_dd_copy<<<g, kDdThreads, 0, st>>>(n, r.hi(), r.lo(), r0.hi(), r0.lo());
  k_dd_copy<<<g, kDdThreads, 0, st>>>(n, r.hi(), r.lo(), p.hi(), p.lo());
  R.dot(b, b, d1);
  R.dot(r0, r0, d2);
  k_dd_scal_b<<<1, 32, 0, st>>>(sb, DDB_INIT, dp<dd>(d1), dp<dd>(d2));
  PB_CUDA(cudaGetLastError());
  L.setup_end = now_s();
  DdScalB h;
  PB_CUDA(cudaMemcpyAsync(&h, sb, sizeof(DdScalB), cudaMemcpyDeviceToHost, st));
  sync();
  const double bnorm = h.bnorm.hi;
  double hist = h.hist;
  int itr;
  for (itr = 1; itr <= o.itrmax; ++itr) {
    if (reshistory) reshistory[itr - 1] = hist;
    R.precon(p.hi(), p.lo(), pp.hi(), pp.lo());
    R.spmv(pp, q);
    R.dot(r0, q, d1);
    k_dd_scal_b<<<1, 32, 0, st>>>(sb, DDB_ALPHA, dp<dd>(d1), nullptr);
    k_dd_bicg_axpy3<<<g, kDdThreads, 0, st>>>(n, sb, r.hi(), r.lo(), q.hi(), q.lo(), e.hi(), e.lo());
    R.precon(e.hi(), e.lo(), pe.hi(), pe.lo());
    R.spmv(pe, v);
    R.dot(e, v, d1);
    R.dot(v, v, d2);
    k_dd_scal_b<<<1, 32, 0, st>>>(sb, DDB_C3, dp<dd>(d1), dp<dd>(d2));
    k_dd_bicg_axpy4<<<g, kDdThreads, 0, st>>>(n, sb, x.hi(), x.lo(), pp.hi(), pp.lo(), pe.hi(), pe.lo());
    k_dd_bicg_axpy3r<<<g, kDdThreads, 0, st>>>(n, sb, e.hi(), e.lo(), v.hi(), v.lo(), r.hi(), r.lo());
    R.dot(r, r0, d1);
    R.dot(r, r, d2);
    k_dd_scal_b<<<1, 32, 0, st>>>(sb, DDB_RNORM, dp<dd>(d1), dp<dd>(d2));
    PB_CUDA(cudaGetLastError());
    double rn[2];
    PB_CUDA(cudaMemcpyAsync(&rn[0], &sb->rnorm.hi, sizeof(double), cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaMemcpyAsync(&rn[1], &sb->hist, sizeof(double), cudaMemcpyDeviceToHost, st));
    sync();
    hist = rn[1];
    if (rn[0] / bnorm < o.rtol) break;
    k_dd_scal_b<<<1, 32, 0, st>>>(sb, DDB_BETA, nullptr, nullptr);
    k_dd_bicg_axpy4p<<<g, kDdThreads, 0, st>>>(n, sb, p.hi(), p.lo(), r.hi(), r.lo(), q.hi(), q.lo());
  }
  PB_CUDA(cudaGetLastError());
  L.used = std::min(o.itrmax, itr);
  L.iret = (o.itrmax <= itr) ? 1 : 0;
  return L;
}

// ddKSP_pGMRES (ddpgmres.f90:254-713): right-preconditioned GMRES(m), MGS or CGS.  The
// restart residual is tested only against abstolmax, which parcel_ddgmres fixes at 0
// (ddwrapper.f90:438), so that test is left out.  History entries are rnorm.hi / bnorm.hi;
// the first cycle also stores its starting residual.  Entries past itrmax (the reference
// writes m of them when itrmax is 1) are not stored.
DdLoop dd_gmres_loop(const DdRun& R, const Options& o, DdVec& x, const DdVec& b, double* reshistory) {
  const int n = R.n, g = R.g;
  cudaStream_t st = R.st;
  DdLoop L;
  const int m = std::max(1, o.m);
  const bool mgs = o.gs != PARCEL_B_GS_CGS;
  const int64_t ldv = n;
  DdVec r(n), pv(n), w(n), x0(n), v0(n);
  DBuf Vh(sizeof(double) * (size_t)(m + 1) * ldv), Vl(sizeof(double) * (size_t)(m + 1) * ldv);   // zero-filled
  auto vh = [&](int k) { return dp<double>(Vh) + (int64_t)k * ldv; };   // v_{k+1}
  auto vl = [&](int k) { return dp<double>(Vl) + (int64_t)k * ldv; };
  const int ld = m + 1;
  DBuf hbuf(sizeof(dd) * (size_t)ld * m), cbuf(sizeof(dd) * ld), sbuf(sizeof(dd) * ld), ebuf(sizeof(dd) * ld),
      ybuf(sizeof(dd) * ld), sc(sizeof(dd) * 2 + sizeof(double)), d1(sizeof(dd));
  DdGm G;
  G.m = m;
  G.h = dp<dd>(hbuf);
  G.c = dp<dd>(cbuf);
  G.s = dp<dd>(sbuf);
  G.e = dp<dd>(ebuf);
  G.y = dp<dd>(ybuf);
  G.bnorm = dp<dd>(sc);
  G.t1 = G.bnorm + 1;
  G.rn = reinterpret_cast<double*>(G.bnorm + 2);
  R.dot(b, b, d1);
  k_dd_gm_scal<<<1, 32, 0, st>>>(G, DDG_BNORM, 0, dp<dd>(d1));
  PB_CUDA(cudaGetLastError());
  dd bn;
  PB_CUDA(cudaMemcpyAsync(&bn, G.bnorm, sizeof(dd), cudaMemcpyDeviceToHost, st));
  sync();
  L.setup_end = now_s();
  const double bnorm = bn.hi;
  auto hist_at = [&](int k, double v) {   // 1-based entry k
    if (reshistory && k >= 1 && k <= o.itrmax) reshistory[k - 1] = v;
  };
  double rnorm = 0.0;
  int itr = 1, inner = 1, mm = 0;
  for (itr = 1; itr <= o.itrmax; itr += m) {
    R.residual(x, b, r);
    R.dot(r, r, d1);
    k_dd_gm_scal<<<1, 32, 0, st>>>(G, DDG_START, 0, dp<dd>(d1));
    R.axpy(G.t1, R.zero, r.hi(), r.lo(), vh(0), vl(0));   // v_1 = -r / |r|
    PB_CUDA(cudaGetLastError());
    rnorm = read_double(G.rn, st);
    if (itr == 1) hist_at(itr, rnorm / bnorm);
    bool exit_inner = false;
    for (inner = 1; inner <= m; ++inner) {
      R.precon(vh(inner - 1), vl(inner - 1), pv.hi(), pv.lo());
      R.spmv(pv, w);
      dd* col = G.h + (int64_t)(inner - 1) * ld;
      if (mgs) {
        for (int k = 1; k < inner; ++k) {
          R.dot(w.hi(), w.lo(), vh(k - 1), vl(k - 1), col + (k - 1));
          k_dd_axpy_nh<<<g, kDdThreads, 0, st>>>(n, col + (k - 1), vh(k - 1), vl(k - 1), w.hi(), w.lo());
        }
      } else if (inner > 1) {
        for (int k = 1; k < inner; ++k) R.dot(vh(k - 1), vl(k - 1), w.hi(), w.lo(), col + (k - 1));
        k_dd_cgs_sub<<<g, kDdThreads, 0, st>>>(n, inner - 1, col, dp<double>(Vh), dp<double>(Vl), ldv, w.hi(),
                                               w.lo());
      }
      R.dot(w.hi(), w.lo(), vh(inner - 1), vl(inner - 1), col + (inner - 1));
      k_dd_axpy_nh<<<g, kDdThreads, 0, st>>>(n, col + (inner - 1), vh(inner - 1), vl(inner - 1), w.hi(), w.lo());
      R.dot(w, w, d1);
      k_dd_gm_scal<<<1, 32, 0, st>>>(G, DDG_NORM, inner, dp<dd>(d1));
      R.axpy(G.t1, R.zero, w.hi(), w.lo(), vh(inner), vl(inner));   // v_{i+1} = w / |w|
      PB_CUDA(cudaGetLastError());
      rnorm = read_double(G.rn, st);
      mm = inner;
      hist_at(itr + inner, rnorm / bnorm);
      if (rnorm / bnorm < o.rtol || itr + inner == o.itrmax) { exit_inner = true; break; }
    }
    if (!exit_inner) inner = m + 1;   // the Fortran DO variable after a completed loop
    if (m < mm) mm = m;
    // ddupdate_xVec (ddpgmres.f90:52-145): y = H^-1 e, v0 = V y, x = M^-1 v0 + x
    k_dd_gm_scal<<<1, 32, 0, st>>>(G, DDG_SOLVE, mm, nullptr);
    k_dd_sum_vec<<<g, kDdThreads, 0, st>>>(n, mm, G.y, dp<double>(Vh), dp<double>(Vl), ldv, v0.hi(), v0.lo());
    R.precon(v0.hi(), v0.lo(), x0.hi(), x0.lo());
    R.axpy(R.one, R.one, x0.hi(), x0.lo(), x.hi(), x.lo());
    PB_CUDA(cudaGetLastError());
    if (rnorm / bnorm < o.rtol) break;
    if (itr + inner == o.itrmax) break;
  }
  sync();
  L.used = std::min(o.itrmax, itr + inner);
  L.iret = (o.itrmax <= itr) ? 1 : 0;
  return L;
}

// The dd Krylov solves of PARCEL_ddKSP_CRS: CG (ddKSP_pCG), BiCGStab (ddKSP_pBiCG) or
// GMRES(m) (ddKSP_pGMRES).
int dd_krylov(int solver, const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo, int precision_A,
              int precision_b, int precision_x, int precision_precondition, const double* b_hi, const double* b_lo,
              double* x_hi, double* x_lo, double* reshistory, int* niter, int* iret) {
  int used = 0, ir = 0;
  const int rc = guarded([&]() -> int {
    ensure_init();
    validate(A);
    PB_CHECK(b_hi && x_hi, PARCEL_B_E_ARG, "b_hi and x_hi must not be NULL");
    for (int f : {precision_A, precision_b, precision_x, precision_precondition})
      PB_CHECK(f == 1 || f == 2, PARCEL_B_E_ARG, "precision flags are 1 (double) or 2 (double-double)");
    Options o = resolve_options(prm);
    PB_CHECK(o.independ_nvec == 1, PARCEL_B_E_UNSUPPORTED,
             "independ_nvec=%d: only 1 (the reference default) is provided", o.independ_nvec);
    cudaStream_t st = stream();
    const int n = A->n;
    const double t0 = now_s();
    DdSystem S;
    S.n = n;
    S.cbase = A->istart;
    Arr arp(A->rowptr, sizeof(int) * ((size_t)n + 1)), aci(A->col, sizeof(int) * (size_t)A->nnz),
        aah(A->val, sizeof(double) * (size_t)A->nnz),
        aal(precision_A == 2 ? val_lo : nullptr, sizeof(double) * (size_t)A->nnz);
    S.rp = static_cast<const int*>(arp.p);
    S.ci = static_cast<const int*>(aci.p);
    S.ah = static_cast<const double*>(aah.p);
    S.al = static_cast<const double*>(aal.p);
    DdPrecon P;
    dd_setup_precon(o, *A, S, precision_precondition, P);
    // x and b in dd, the low parts zero unless their precision is 2
    DdVec x(n), b(n);
    auto load = [&](DdVec& v, const double* hi, const double* lo, bool use_lo) {
      if (is_device_ptr(hi)) PB_CUDA(cudaMemcpyAsync(v.hi(), hi, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      else h2d(v.hi(), hi, sizeof(double) * n);
      if (use_lo && lo) {
        if (is_device_ptr(lo)) PB_CUDA(cudaMemcpyAsync(v.lo(), lo, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        else h2d(v.lo(), lo, sizeof(double) * n);
      }
    };
    load(x, x_hi, x_lo, precision_x == 2);
    load(b, b_hi, b_lo, precision_b == 2);
    DBuf part(sizeof(dd) * (kDdDotCtas + 1)), cst(sizeof(dd) * 3);
    dd* dcst = dp<dd>(cst);
    {
      const dd h[3] = {dd{1.0, 0.0}, dd{-1.0, 0.0}, dd{0.0, 0.0}};
      h2d(dcst, h, sizeof(h));
    }
    const DdRun R{S, P, st, n, grid_for(n), dp<dd>(part), dcst, dcst + 1, dcst + 2};
    DdLoop L;
    if (solver == PARCEL_B_SOLVER_BICG) L = dd_bicg_loop(R, o, x, b, reshistory);
    else if (solver == PARCEL_B_SOLVER_GMRES) L = dd_gmres_loop(R, o, x, b, reshistory);
    else L = dd_cg_loop(R, o, x, b, reshistory);
    used = L.used;
    ir = L.iret;
    auto store = [&](double* dst, const double* src) {
      if (is_device_ptr(dst)) PB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      else PB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    };
    store(x_hi, x.hi());
    if (precision_x == 2 && x_lo) store(x_lo, x.lo());
    sync();
    parcel_b_stats stt;
    memset(&stt, 0, sizeof(stt));
    stt.setup_s = L.setup_end - t0;
    stt.solve_s = now_s() - L.setup_end;
    stt.ilu_nblocks = P.nb;
    set_stats(stt);
    return 0;
  });
  if (niter) *niter = rc == 0 ? used : 0;
  if (iret) *iret = rc == 0 ? ir : rc;
  return rc;
}

}  // namespace

extern "C" int parcel_b_ddcg(const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo,
                             int precision_A, int precision_b, int precision_x, int precision_precondition,
                             const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                             double* reshistory, int* niter, int* iret) {
  return dd_krylov(PARCEL_B_SOLVER_CG, prm, A, val_lo, precision_A, precision_b, precision_x, precision_precondition,
                   b_hi, b_lo, x_hi, x_lo, reshistory, niter, iret);
}

extern "C" int parcel_b_ddbicgstab(const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo,
                                   int precision_A, int precision_b, int precision_x, int precision_precondition,
                                   const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                                   double* reshistory, int* niter, int* iret) {
  return dd_krylov(PARCEL_B_SOLVER_BICG, prm, A, val_lo, precision_A, precision_b, precision_x,
                   precision_precondition, b_hi, b_lo, x_hi, x_lo, reshistory, niter, iret);
}

extern "C" int parcel_b_ddgmres(const parcel_b_input* prm, const parcel_b_crs* A, const double* val_lo,
                                int precision_A, int precision_b, int precision_x, int precision_precondition,
                                const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                                double* reshistory, int* niter, int* iret) {
  return dd_krylov(PARCEL_B_SOLVER_GMRES, prm, A, val_lo, precision_A, precision_b, precision_x,
                   precision_precondition, b_hi, b_lo, x_hi, x_lo, reshistory, niter, iret);
}

namespace {

// parcel_dd*_c (src/example/c2fortran_kernel.f90:620-898): every argument by reference,
// host arrays, niter in = itrmax and out = iterations.
void dd_shim(int solver, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n, int32_t* gn,
             int32_t* nnz, int32_t* istart, double* crsa, double* crsa_lo, int32_t* crsrow_ptr, int32_t* crscol,
             int* ipreflag, int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
             double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
             int* nblock, int* precision_a, int* precision_b, int* precision_x, int* precision_precondition,
             int* iret, int* restart = nullptr, int* gmres_gsflag = nullptr) {
  parcel_b_input p;
  parcel_b_input_init(&p);
  p.solver = solver;
  if (restart) p.GMRES_m = *restart;
  if (gmres_gsflag) p.GMRES_GSflag = *gmres_gsflag;
  p.ipreflag = *ipreflag;
  p.ILU_method = *ilu_method;
  p.addL = *addl;
  p.iflagAS = *iflagas;
  p.itrmax = *niter;
  p.rtolmax = *rtolmax;
  p.abstolmax = 0.0;
  p.iovlflag = *iovlflag;
  p.precon_thblock = *precon_thblock;
  p.Neuman_itr = *neuman_itr;
  p.independ_nvec = *independ_nvec;
  p.nBlock = *nblock;
  parcel_b_crs A;
  A.n = *n; A.gn = *gn; A.nnz = *nnz; A.istart = *istart;
  A.rowptr = crsrow_ptr; A.col = crscol; A.val = crsa;
  int used = 0, ir = 0;
  dd_krylov(solver, &p, &A, crsa_lo, *precision_a, *precision_b, *precision_x, *precision_precondition, vecb,
            vecb_lo, vecx, vecx_lo, reshistory, &used, &ir);
  *niter = used;
  *iret = ir;
}

}  // namespace

extern "C" void parcel_ddcg_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                               int32_t* n, int32_t* gn, int32_t* nnz, int32_t* istart, double* crsa,
                               double* crsa_lo, int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag,
                               int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                               double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                               int* independ_nvec, int* nblock, int* precision_a, int* precision_b,
                               int* precision_x, int* precision_precondition, int* iret) {
  (void)icomm;
  dd_shim(PARCEL_B_SOLVER_CG, vecx, vecx_lo, vecb, vecb_lo, n, gn, nnz, istart, crsa, crsa_lo, crsrow_ptr, crscol,
          ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, precon_thblock, neuman_itr,
          independ_nvec, nblock, precision_a, precision_b, precision_x, precision_precondition, iret);
}

extern "C" void parcel_ddbicgstab_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                                     int32_t* n, int32_t* gn, int32_t* nnz, int32_t* istart, double* crsa,
                                     double* crsa_lo, int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag,
                                     int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                                     double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                                     int* independ_nvec, int* nblock, int* precision_a, int* precision_b,
                                     int* precision_x, int* precision_precondition, int* iret) {
  (void)icomm;
  dd_shim(PARCEL_B_SOLVER_BICG, vecx, vecx_lo, vecb, vecb_lo, n, gn, nnz, istart, crsa, crsa_lo, crsrow_ptr,
          crscol, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, precon_thblock,
          neuman_itr, independ_nvec, nblock, precision_a, precision_b, precision_x, precision_precondition, iret);
}

extern "C" void parcel_ddgmres_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                                  int32_t* n, int32_t* gn, int32_t* nnz, int32_t* istart, double* crsa,
                                  double* crsa_lo, int32_t* crsrow_ptr, int32_t* crscol, int* ipreflag,
                                  int* ilu_method, int* addl, int* iflagas, int* niter, double* rtolmax,
                                  double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                                  int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag,
                                  int* precision_a, int* precision_b, int* precision_x, int* precision_precondition,
                                  int* iret) {
  (void)icomm;
  dd_shim(PARCEL_B_SOLVER_GMRES, vecx, vecx_lo, vecb, vecb_lo, n, gn, nnz, istart, crsa, crsa_lo, crsrow_ptr,
          crscol, ipreflag, ilu_method, addl, iflagas, niter, rtolmax, reshistory, iovlflag, precon_thblock,
          neuman_itr, independ_nvec, nblock, precision_a, precision_b, precision_x, precision_precondition, iret,
          restart, gmres_gsflag);
}
