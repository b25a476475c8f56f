// pb_blas.cu -- vector kernels, deterministic reductions and the solver epilogues.
//
// Replaces the reference's vector layer (src/parcel_vec.f90:351-1178; GPU kernels in
// src/CUDA/src/cu_common.hpp:10-230, cu_pcg.hpp, cu_pbicg.cu, cu_qrdecomposition.cu,
// cu_pcagmres.cu).  The reference reduces every dot product into a device scalar, copies
// it to the host and runs MPI_Allreduce (cu_common.cu:412-446), and reads alpha / beta
// back before every axpy (parcel_vec.f90:466-470).  Here every scalar stays on the device:
// the last block of each reduction finishes the sum in a fixed order and runs the solver
// logic that the reference runs on the host (step lengths, Givens rotations, stop tests).
#include <cmath>

#include "pb_blas.cuh"
#include "pb_device.cuh"
#include "pb_epilogue.cuh"

namespace pb {

// ------------------------------------------------------------------ kernels
// Grid-stride helpers: the reduction kernels always run on the fixed grid red_blocks().
#define GRID_LOOP(i, n) \
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// Grid-stride loop over groups of kU elements per thread (i0 + u*stride, u < kU): the
// loads of a group are issued before any result is stored, which keeps kU independent
// loads per operand in flight for the HBM-bound vector kernels.
constexpr int kU = 4;
#define GRID_LOOP_U(i0, st, n)                                                            \
  for (int64_t st = (int64_t)gridDim.x * blockDim.x,                                       \
               i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;                       \
       i0 < (n); i0 += kU * st)

__device__ __forceinline__ double cval(const Coef& c) { return c.p ? (*c.p) * c.mul : c.v; }

// out = c0*x0 + c1*x1 (+ c2*x2), evaluated left to right as the reference's axpy
// (y = alpha*x + beta*y, vec.f90:952) and axpy_vec3 (vec.f90:975).
template <class T>
__global__ void k_lincomb(int64_t n, T* __restrict__ out, const T* __restrict__ x0,
                          const T* __restrict__ x1, const T* __restrict__ x2, Coef c0, Coef c1,
                          Coef c2, const int* gate) {
  if (gated(gate)) return;
  const T a0 = (T)cval(c0), a1 = (T)cval(c1), a2 = (T)cval(c2);
  GRID_LOOP_U(i0, st, n) {
    T v0[kU], v1[kU], v2[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int64_t i = i0 + u * st;
      const bool ok = i < n;
      v0[u] = ok ? x0[i] : T(0);
      v1[u] = (ok && x1) ? x1[i] : T(0);
      v2[u] = (ok && x2) ? x2[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int64_t i = i0 + u * st;
      if (i < n) {
        T v = a0 * v0[u];
        if (x1) v = v + a1 * v1[u];
        if (x2) v = v + a2 * v2[u];
        out[i] = v;
      }
    }
  }
}

// Same as k_lincomb, fused with up to three dot products of the result or inputs.
// dot pairs select from {0: out, 1: x0, 2: x1, 3: x2, 4: d0, 5: d1}.
template <class T, int ND>
__global__ void __launch_bounds__(kRedThreads, 4) k_lincomb_dot(int64_t n, T* __restrict__ out,
                                                             const T* __restrict__ x0,
                                                             const T* __restrict__ x1,
                                                             const T* __restrict__ x2, Coef c0,
                                                             Coef c1, Coef c2, const T* d0,
                                                             const T* d1, DotSel sel, Red red,
                                                             const int* gate) {
  if (gated(gate)) return;
  const T a0 = (T)cval(c0), a1 = (T)cval(c1), a2 = (T)cval(c2);
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int k = 0; k < ND; ++k) acc[k] = 0.0;
  // three elements per thread and step (a thread still visits its elements in increasing
  // order): four CTAs of 256 threads per SM then fit the registers without spilling
  constexpr int kUD = 3;
  const int64_t st = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += kUD * st) {
    T s0[kUD], s1[kUD], s2[kUD], s4[kUD], s5[kUD];
#pragma unroll
    for (int u = 0; u < kUD; ++u) {
      const int64_t i = i0 + u * st;
      const bool ok = i < n;
      s0[u] = (ok && x0) ? x0[i] : T(0);
      s1[u] = (ok && x1) ? x1[i] : T(0);
      s2[u] = (ok && x2) ? x2[i] : T(0);
      s4[u] = (ok && d0) ? d0[i] : T(0);
      s5[u] = (ok && d1) ? d1[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kUD; ++u) {
      const int64_t i = i0 + u * st;
      if (i >= n) continue;
      T v = T(0);
      if (out) {
        v = a0 * s0[u];
        if (x1) v = v + a1 * s1[u];
        if (x2) v = v + a2 * s2[u];
        out[i] = v;
      }
      // operand s of a dot: 0 the result, 1-3 the summands, 4-5 the extra vectors (a
      // select chain on the uniform selector keeps the operands in registers; an array
      // indexed by it would live in local memory)
      auto pick = [&](int sidx) -> T {
        return sidx == 0 ? v : sidx == 1 ? s0[u] : sidx == 2 ? s1[u] : sidx == 3 ? s2[u] : sidx == 4 ? s4[u] : s5[u];
      };
#pragma unroll
      for (int k = 0; k < ND; ++k) acc[k] += (double)(pick(sel.a[k]) * pick(sel.b[k]));
    }
  }
  reduce_and_finish<ND>(acc, red);
}

// CG_axpy2 (pcg.f90:4-20): x = x + alpha p; p = s + beta p.
template <class T>
__global__ void k_cg_axpy2(int64_t n, T* __restrict__ x, T* __restrict__ p, const T* __restrict__ s,
                           const KState* st, const int* gate) {
  if (gated(gate)) return;
  const T alpha = (T)st->alpha, beta = (T)st->beta;
  GRID_LOOP_U(i0, stp, n) {
    T pv[kU], xv[kU], sv[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int64_t i = i0 + u * stp;
      const bool ok = i < n;
      pv[u] = ok ? p[i] : T(0);
      xv[u] = ok ? x[i] : T(0);
      sv[u] = ok ? s[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int64_t i = i0 + u * stp;
      if (i < n) {
        x[i] = xv[u] + alpha * pv[u];
        p[i] = sv[u] + beta * pv[u];
      }
    }
  }
}

// s = D^-1 r (pointJacobi, matrix.f90:4452-4468)
template <class T>
__global__ void k_scale(int64_t n, T* __restrict__ s, const T* __restrict__ d, const T* __restrict__ r,
                        const int* gate) {
  if (gated(gate)) return;
  GRID_LOOP_U(i0, st, n) {
    T rv[kU], dv[kU];
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int64_t i = i0 + u * st;
      const bool ok = i < n;
      rv[u] = ok ? r[i] : T(0);
      dv[u] = ok ? d[i] : T(0);
    }
#pragma unroll
    for (int u = 0; u < kU; ++u) {
      const int64_t i = i0 + u * st;
      if (i < n) s[i] = rv[u] * dv[u];
    }
  }
}

// CGS multi-dot h(k) = <w, v_k>, k = 1..j (cuda_CGS_Orth dot phase, cu_qrdecomposition.cu:45)
template <class T>
__global__ void __launch_bounds__(kRedThreads) k_multidot(int64_t n, int j, const T* __restrict__ w,
                                                          const T* __restrict__ V, int64_t ldv,
                                                          Red red, const int* gate) {
  if (gated(gate)) return;
  __shared__ double wsum[kMaxRed * (kRedThreads / 32)];
  const int l = threadIdx.x & 31, wi = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k0 = 0; k0 < j; k0 += 8) {
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int kk = min(8, j - k0);
    GRID_LOOP(i, n) {
      double wi_ = (double)w[i];
#pragma unroll
      for (int k = 0; k < 8; ++k)
        if (k < kk) acc[k] += wi_ * (double)V[(size_t)(k0 + k) * ldv + i];
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      double x = acc[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
      if (l == 0 && k < kk) wsum[(k0 + k) * nw + wi] = x;
    }
  }
  reduce_and_finish_dyn(wsum, j, red);
}

// w = w - sum_k h(k,j) v_k (cuda_CGS_Orth axpy phase) fused with <w,w>.
template <class T>
__global__ void __launch_bounds__(kRedThreads) k_cgs_update(int64_t n, int j, T* __restrict__ w,
                                                            const T* __restrict__ V, int64_t ldv,
                                                            const double* __restrict__ hcol,
                                                            Red red, const int* gate) {
  if (gated(gate)) return;
  __shared__ double hs[kMaxRed];
  for (int k = threadIdx.x; k < j; k += blockDim.x) hs[k] = hcol[k];
  __syncthreads();
  double acc[1] = {0.0};
  GRID_LOOP(i, n) {
    T t = w[i];
    for (int k = 0; k < j; ++k) t = t - (T)hs[k] * V[(size_t)k * ldv + i];
    w[i] = t;
    acc[0] += (double)t * (double)t;
  }
  reduce_and_finish<1>(acc, red);
}

// v0 = sum_i y_i v_i (sum_vec_FP64_CPU, pcagmres.f90:54-90; cuda_sum_vec_, cu_pcagmres.cu:91)
template <class T>
__global__ void k_sum_vec(int64_t n, T* __restrict__ v0, const T* __restrict__ V, int64_t ldv,
                          const double* __restrict__ y, const KState* st, const int* gate) {
  if (gated(gate)) return;
  __shared__ double ys[kMaxRed];
  const int mm = st->mm;
  for (int k = threadIdx.x; k < mm; k += blockDim.x) ys[k] = y[k];
  __syncthreads();
  GRID_LOOP(i, n) {
    T t = T(0);
    for (int k = 0; k < mm; ++k) t = t + (T)ys[k] * V[(size_t)k * ldv + i];
    v0[i] = t;
  }
}

// y = H^-1 e by back substitution over the mm used columns (update_xVec,
// pcagmres.f90:1136-1236).  The warp stages the used part of H and e in shared memory
// (coalesced); one thread then substitutes in the reference's order.  Restarts up to
// kBackSmemM use the staged copy, longer ones read H from global memory.
constexpr int kBackSmemM = 64;
__global__ void k_gm_backsolve(const double* h, const double* e, double* y, int m0, KState* st,
                               const int* gate) {
  if (gated(gate)) return;
  __shared__ double sh[kBackSmemM * kBackSmemM], se[kBackSmemM], sy[kBackSmemM];
  const int m = st->mm;
  const bool staged = m <= kBackSmemM;
  if (staged) {
    for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
      const int r = t % m, c = t / m;   // H(r, c), column-major
      sh[r + c * kBackSmemM] = h[(size_t)r + (size_t)c * (m0 + 1)];
    }
    for (int t = threadIdx.x; t < m; t += blockDim.x) se[t] = e[t];
    __syncthreads();
  }
  if (threadIdx.x != 0) return;
  if (staged) {
    for (int i = m; i >= 1; --i) {
      double v = se[i - 1];
      for (int j = m; j >= i + 1; --j) v = v - sh[(i - 1) + (j - 1) * kBackSmemM] * sy[j - 1];
      const double d = sh[(i - 1) + (i - 1) * kBackSmemM];
      sy[i - 1] = (d == 0.0) ? v / 1.0e-300 : v / d;
    }
    for (int i = 0; i < m; ++i) y[i] = sy[i];
    return;
  }
  for (int i = m; i >= 1; --i) {
    double v = e[i - 1];
    for (int j = m; j >= i + 1; --j) v = v - h[(size_t)(i - 1) + (size_t)(j - 1) * (m0 + 1)] * y[j - 1];
    double d = h[(size_t)(i - 1) + (size_t)(i - 1) * (m0 + 1)];
    y[i - 1] = (d == 0.0) ? v / 1.0e-300 : v / d;
  }
}

// After the restart cycle's update: exit test of pgmres.f90 (after update_xVec) and the
// loop increment itr += m.
__global__ void k_gm_post(KState* st, int m, int itrmax) {
  if (st->done) return;
  const int itr = st->itr;
  const int inner_end = st->stop_after_update ? st->inner : m + 1;
  if (st->stop_after_update) {
    st->done = 1;
    st->niter = min(itrmax, itr + inner_end);
    st->iret = st->breakdown ? PARCEL_B_E_BREAKDOWN : ((itrmax <= itr) ? 1 : 0);
    return;
  }
  st->last_inner = inner_end;
  st->itr = itr + m;
  if (st->itr > itrmax) {
    st->done = 1;
    st->niter = min(itrmax, st->itr + inner_end);
    st->iret = 1;
  }
}

__global__ void k_fill(int64_t n, double* p, double v) { GRID_LOOP(i, n) p[i] = v; }
__global__ void k_fillf(int64_t n, float* p, float v) { GRID_LOOP(i, n) p[i] = v; }

template <class TO, class TI>
__global__ void k_convert(int64_t n, TO* __restrict__ o, const TI* __restrict__ in) {
  GRID_LOOP(i, n) o[i] = (TO)in[i];
}

// Natural <-> permuted layout.  perm[i] = permuted position of natural row i.
template <class T>
__global__ void k_scatter_perm(int n, T* __restrict__ outp, const double* __restrict__ in,
                               const int* __restrict__ perm) {
  GRID_LOOP(i, n) outp[perm[i]] = (T)in[i];
}
template <class T>
__global__ void k_gather_perm(int n, double* __restrict__ out, const T* __restrict__ inp,
                              const int* __restrict__ perm) {
  GRID_LOOP(i, n) out[i] = (double)inp[perm[i]];
}

// ------------------------------------------------------------------ host launchers
static inline int eb(int64_t n) {
  int64_t b = (n + 255) / 256;
  int64_t cap = 8LL * num_sms();
  return (int)std::max<int64_t>(1, std::min<int64_t>(b, cap));
}

template <class T>
void lincomb(int64_t n, T* out, const T* x0, Coef c0, const T* x1, Coef c1, const T* x2, Coef c2,
             const int* gate, cudaStream_t st) {
  k_lincomb<T><<<eb(n), 256, 0, st>>>(n, out, x0, x1, x2, c0, c1, c2, gate);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void lincomb_dot(int64_t n, T* out, const T* x0, Coef c0, const T* x1, Coef c1, const T* x2,
                 Coef c2, const T* d0, const T* d1, DotSel sel, int nd, const Red& red,
                 const int* gate, cudaStream_t st) {
  const int g = red_blocks();
  switch (nd) {
    case 1: k_lincomb_dot<T, 1><<<g, kRedThreads, 0, st>>>(n, out, x0, x1, x2, c0, c1, c2, d0, d1, sel, red, gate); break;
    case 2: k_lincomb_dot<T, 2><<<g, kRedThreads, 0, st>>>(n, out, x0, x1, x2, c0, c1, c2, d0, d1, sel, red, gate); break;
    case 3: k_lincomb_dot<T, 3><<<g, kRedThreads, 0, st>>>(n, out, x0, x1, x2, c0, c1, c2, d0, d1, sel, red, gate); break;
    default: PB_CHECK(false, PARCEL_B_E_ARG, "lincomb_dot: nd=%d", nd);
  }
  PB_CUDA(cudaGetLastError());
}

template <class T>
void cg_axpy2(int64_t n, T* x, T* p, const T* s, const KState* st, const int* gate, cudaStream_t s_) {
  k_cg_axpy2<T><<<eb(n), 256, 0, s_>>>(n, x, p, s, st, gate);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void scale(int64_t n, T* s, const T* d, const T* r, const int* gate, cudaStream_t st) {
  k_scale<T><<<eb(n), 256, 0, st>>>(n, s, d, r, gate);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void multidot(int64_t n, int j, const T* w, const T* V, int64_t ldv, const Red& red, const int* gate,
              cudaStream_t st) {
  k_multidot<T><<<red_blocks(), kRedThreads, 0, st>>>(n, j, w, V, ldv, red, gate);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void cgs_update(int64_t n, int j, T* w, const T* V, int64_t ldv, const double* hcol, const Red& red,
                const int* gate, cudaStream_t st) {
  k_cgs_update<T><<<red_blocks(), kRedThreads, 0, st>>>(n, j, w, V, ldv, hcol, red, gate);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void sum_vec(int64_t n, T* v0, const T* V, int64_t ldv, const double* y, const KState* st,
             const int* gate, cudaStream_t s_) {
  k_sum_vec<T><<<eb(n), 256, 0, s_>>>(n, v0, V, ldv, y, st, gate);
  PB_CUDA(cudaGetLastError());
}

void gm_backsolve(const double* h, const double* e, double* y, int m0, KState* st, const int* gate,
                  cudaStream_t s_) {
  k_gm_backsolve<<<1, 256, 0, s_>>>(h, e, y, m0, st, gate);
  PB_CUDA(cudaGetLastError());
}

void gm_post(KState* st, int m, int itrmax, cudaStream_t s_) {
  k_gm_post<<<1, 1, 0, s_>>>(st, m, itrmax);
  PB_CUDA(cudaGetLastError());
}

void fill(int64_t n, double* p, double v, cudaStream_t st) {
  k_fill<<<eb(n), 256, 0, st>>>(n, p, v);
  PB_CUDA(cudaGetLastError());
}

template <class TO, class TI>
void convert(int64_t n, TO* o, const TI* in, cudaStream_t st) {
  k_convert<TO, TI><<<eb(n), 256, 0, st>>>(n, o, in);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void scatter_perm(int n, T* outp, const double* in, const int* perm, cudaStream_t st) {
  k_scatter_perm<T><<<eb(n), 256, 0, st>>>(n, outp, in, perm);
  PB_CUDA(cudaGetLastError());
}
template <class T>
void gather_perm(int n, double* out, const T* inp, const int* perm, cudaStream_t st) {
  k_gather_perm<T><<<eb(n), 256, 0, st>>>(n, out, inp, perm);
  PB_CUDA(cudaGetLastError());
}

#define INST(T)                                                                                  \
  template void lincomb<T>(int64_t, T*, const T*, Coef, const T*, Coef, const T*, Coef,          \
                           const int*, cudaStream_t);                                            \
  template void lincomb_dot<T>(int64_t, T*, const T*, Coef, const T*, Coef, const T*, Coef,      \
                               const T*, const T*, DotSel, int, const Red&, const int*,          \
                               cudaStream_t);                                                    \
  template void cg_axpy2<T>(int64_t, T*, T*, const T*, const KState*, const int*, cudaStream_t); \
  template void scale<T>(int64_t, T*, const T*, const T*, const int*, cudaStream_t);             \
  template void multidot<T>(int64_t, int, const T*, const T*, int64_t, const Red&, const int*,   \
                            cudaStream_t);                                                       \
  template void cgs_update<T>(int64_t, int, T*, const T*, int64_t, const double*, const Red&,    \
                              const int*, cudaStream_t);                                         \
  template void sum_vec<T>(int64_t, T*, const T*, int64_t, const double*, const KState*,         \
                           const int*, cudaStream_t);                                            \
  template void scatter_perm<T>(int, T*, const double*, const int*, cudaStream_t);               \
  template void gather_perm<T>(int, double*, const T*, const int*, cudaStream_t);
INST(double)
INST(float)
template void convert<float, double>(int64_t, float*, const double*, cudaStream_t);
template void convert<double, float>(int64_t, double*, const float*, cudaStream_t);

}  // namespace pb
