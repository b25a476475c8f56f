// pb_epilogue.cuh -- solver epilogues run by the last block of a reduction, and the
// block reductions that call them.  Included by every file with reduction kernels so the
// epilogue inlines into each kernel.
#pragma once

#include <cmath>

#include "pb_device.cuh"

namespace pb {

// ------------------------------------------------------------------ epilogues
// GivensRotations (src/pcagmres.f90:190-242), column j (1-based), h (m+1) x m column
// major.  The reference's zero-diagonal guard `h/1.0d0-300` evaluates to h - 300; it is
// kept as written.
static __device__ void givens(int m, double* h, int j, double* c, double* s, double* e) {
  double* col = h + (size_t)(j - 1) * (m + 1);
  for (int k = 1; k <= j - 1; ++k) {
    double t1 = col[k - 1] * c[k - 1] - col[k] * s[k - 1];
    double t2 = col[k - 1] * s[k - 1] + col[k] * c[k - 1];
    col[k - 1] = t1;
    col[k] = t2;
  }
  double t = (col[j - 1] == 0.0) ? col[j] / 1.0 - 300.0 : col[j] / col[j - 1];
  c[j - 1] = 1.0 / sqrt(1.0 + t * t);
  s[j - 1] = -c[j - 1] * t;
  double t1 = c[j - 1] * e[j - 1] - s[j - 1] * e[j];
  double t2 = s[j - 1] * e[j - 1] + c[j - 1] * e[j];
  e[j - 1] = t1;
  e[j] = t2;
  col[j - 1] = c[j - 1] * col[j - 1] - s[j - 1] * col[j];
  col[j] = 0.0;
}

static __device__ __forceinline__ bool bad(double x) { return !isfinite(x); }

static __device__ void epilogue(const double* S, int K, const Red& r) {
  const EpiArgs& a = r.ea;
  KState* st = a.st;
  if (r.epi == EPI_STORE) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) a.out[k] = S[k];
    return;
  }
  if (r.epi == EPI_GM_HCGS) {
    for (int k = threadIdx.x; k < K; k += blockDim.x) a.h[(size_t)(a.j - 1) * (a.m + 1) + k] = S[k];
    return;
  }
  if (threadIdx.x != 0) return;
  switch (r.epi) {
    case EPI_NORM2:
      a.out[0] = sqrt(S[0]);
      break;
    // ---- PCG (pcg.f90:224-892)
    case EPI_CG_INIT: {
      st->bnorm = sqrt(S[0]);
      st->rnorm = sqrt(S[1]);
      st->rho0 = S[2];
      st->alpha = 0.0;
      st->beta = 0.0;
      st->itr = 1;
      st->done = 0;
      st->niter = 0;
      st->iret = 0;
      if (a.itrmax < 1) { st->done = 1; st->iret = 1; break; }
      a.hist[0] = st->rnorm / st->bnorm;
      if (bad(st->rho0) || bad(st->bnorm)) { st->done = 1; st->breakdown = 1; st->niter = 1; }
      break;
    }
    case EPI_CG_GAMMA:
      st->gamma = S[0];
      st->alpha = st->rho0 / st->gamma;
      st->tmp[0] = -st->alpha;
      break;
    case EPI_CG_DOT2: {
      st->rho1 = S[0];
      double rn = sqrt(S[1]);
      st->rnorm = rn;
      const int itr = st->itr;
      double rel = rn / st->bnorm;
      if (rel < a.rtol) {
        st->done = 1; st->niter = min(a.itrmax, itr); st->iret = (a.itrmax <= itr) ? 1 : 0;
      } else if (rel > 1.0e8) {
        st->done = 1; st->diverged = 1; st->niter = min(a.itrmax, itr);
        st->iret = (a.itrmax <= itr) ? 1 : 0;
      } else if (bad(rel) || bad(st->rho1)) {
        st->done = 1; st->breakdown = 1; st->niter = min(a.itrmax, itr);
        st->iret = PARCEL_B_E_BREAKDOWN;
      } else {
        st->beta = st->rho1 / st->rho0;
        st->rho0 = st->rho1;
        if (itr + 1 > a.itrmax) {
          st->done = 1; st->niter = a.itrmax; st->iret = 1;
        } else {
          st->itr = itr + 1;
          a.hist[itr] = rn / st->bnorm;
        }
      }
      break;
    }
    // ---- BiCGStab (pbicg.f90:280-698)
    case EPI_BICG_INIT:
      st->bnorm = sqrt(S[0]);
      st->rnorm = sqrt(S[1]);
      st->c1 = S[1];   // <r0, r0> with r0 = r
      st->c2 = 0.0; st->c3 = 0.0;
      st->itr = 1; st->done = 0; st->niter = 0; st->iret = 0;
      if (a.itrmax < 1) { st->done = 1; st->iret = 1; break; }
      a.hist[0] = st->rnorm / st->bnorm;
      break;
    case EPI_BICG_C2:
      st->c2 = S[0];
      st->alpha = st->c1 / st->c2;
      st->tmp[0] = -st->alpha;
      break;
    case EPI_BICG_C3:
      st->ev = S[0];
      st->vv = S[1];
      st->c3 = st->ev / st->vv;
      st->tmp[1] = -st->c3;
      break;
    case EPI_BICG_END: {
      st->c1 = S[0];
      double rn = sqrt(S[1]);
      st->rnorm = rn;
      const int itr = st->itr;
      double rel = rn / st->bnorm;
      if (rel < a.rtol) {
        st->done = 1; st->niter = min(a.itrmax, itr); st->iret = (a.itrmax <= itr) ? 1 : 0;
      } else if (bad(rel) || bad(st->c1)) {
        st->done = 1; st->breakdown = 1; st->niter = min(a.itrmax, itr);
        st->iret = PARCEL_B_E_BREAKDOWN;
      } else {
        st->beta = st->c1 / (st->c3 * st->c2);
        st->tmp[2] = -st->beta * st->c3;
        if (itr + 1 > a.itrmax) {
          st->done = 1; st->niter = a.itrmax; st->iret = 1;
        } else {
          st->itr = itr + 1;
          a.hist[itr] = rn / st->bnorm;
        }
      }
      break;
    }
    // ---- GMRES(m) (pgmres.f90:62-525)
    case EPI_GM_RESTART: {
      double rn = sqrt(S[0]);
      st->rnorm = rn;
      st->tmp[0] = -1.0 / rn;           // v1 = (-1/||r||) r
      for (int i = 0; i <= a.m; ++i) { a.e[i] = 0.0; a.cs[i] = 0.0; a.sn[i] = 0.0; }
      for (int i = 0; i < (a.m + 1) * a.m; ++i) a.h[i] = 0.0;
      a.e[0] = -rn;
      st->inner = 0;
      const int itr = st->itr;
      if (rn < a.abstol || rn / st->bnorm < a.rtol) {
        // exit at the top of the restart loop: niter = min(itrmax, itr + inner)
        st->done = 1;
        st->niter = min(a.itrmax, itr + st->last_inner);
        st->skip_inner = 1;
        st->iret = (a.itrmax <= itr) ? 1 : 0;
        break;
      }
      if (bad(rn)) { st->done = 1; st->skip_inner = 1; st->breakdown = 1; st->iret = PARCEL_B_E_BREAKDOWN; st->niter = itr; break; }
      if (itr == 1) a.hist[0] = rn / st->bnorm;
      st->skip_inner = 0;
      st->stop_after_update = 0;
      break;
    }
    case EPI_GM_H:
      a.h[(size_t)(a.j - 1) * (a.m + 1) + (a.k - 1)] = S[0];
      st->tmp[1] = -S[0];
      break;
    case EPI_GM_NORM: {
      const int j = a.j;
      double wn = sqrt(S[0]);
      a.h[(size_t)(j - 1) * (a.m + 1) + j] = wn;
      st->tmp[2] = 1.0 / wn;
      givens(a.m, a.h, j, a.cs, a.sn, a.e);
      double rn = fabs(a.e[j]);
      st->rnorm = rn;
      st->mm = j;
      st->inner = j;
      const int itr = st->itr;
      a.hist[itr + j - 1] = rn / st->bnorm;
      if (rn / st->bnorm < a.rtol) { st->skip_inner = 1; st->stop_after_update = 1; }
      else if (itr + j == a.itrmax) { st->skip_inner = 1; st->stop_after_update = 1; }
      else if (bad(rn)) { st->skip_inner = 1; st->stop_after_update = 1; st->breakdown = 1; }
      break;
    }
  }
}

// Runtime-K block reduction, values in shared memory vals[K][blockDim.x / 32] already
// reduced per warp by the caller.
static __device__ void reduce_and_finish_dyn(double* wsum, int K, const Red& r) {
  __shared__ unsigned am_last;
  __shared__ double S[kMaxRed];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  __syncthreads();
  for (int k = threadIdx.x; k < K; k += blockDim.x) {
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s += wsum[k * nw + i];
    r.part[(size_t)blockIdx.x * K + k] = s;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(r.ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  for (int k = w; k < K; k += nw) {
    double s = 0.0;
    for (int b = l; b < (int)gridDim.x; b += 32) s += __ldcg(r.part + (size_t)b * K + k);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (l == 0) S[k] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *r.ticket = 0u;
  epilogue(S, K, r);
}


// Block-reduces K per-thread values, writes this block's partials, and lets the last
// block (by ticket) sum all partials in block order and run the epilogue.  Every thread of
// the block must call it.  Deterministic for a fixed grid size.
template <int K>
__device__ __forceinline__ void reduce_and_finish(double (&v)[K], const Red& r) {
  __shared__ double sm[K][32];
  __shared__ double S[K > 0 ? K : 1];
  __shared__ unsigned am_last;
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    if (l == 0) sm[k][w] = x;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0.0;
    for (int i = 0; i < nw; ++i) s += sm[threadIdx.x][i];
    r.part[(size_t)blockIdx.x * K + threadIdx.x] = s;
    __threadfence();
  }
  __syncthreads();
  if (threadIdx.x == 0) am_last = (atomicAdd(r.ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  for (int k = w; k < K; k += nw) {
    double s = 0.0;
    for (int b = l; b < (int)gridDim.x; b += 32) s += __ldcg(r.part + (size_t)b * K + k);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (l == 0) S[k] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) *r.ticket = 0u;
  epilogue(S, K, r);
}

}  // namespace pb
