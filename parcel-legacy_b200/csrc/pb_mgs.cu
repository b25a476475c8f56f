// pb_mgs.cu -- GMRES modified Gram-Schmidt for one Arnoldi column in one launch.
//
// Reference: the MGS branch of KSP_pGMRES (src/pgmres.f90:333-351): for k = 1..j,
// h(k,j) = <w, v_k> then w = -h(k,j) v_k + w; then h(j+1,j) = ||w|| and
// v_{j+1} = (1/h(j+1,j)) w, followed by GivensRotations (src/pcagmres.f90:190-242).  The
// reference runs every dot product as a device reduction, a copy to the host and an
// MPI_Allreduce (src/CUDA/src/cu_common.cu:412-446).
//
// B200 design.  A cooperative (co-resident) grid keeps w in registers for the whole
// column: pass p reads v_{p-1} (an L2 hit: it was read by the previous pass) and v_p from
// HBM, applies w -= h(p-1) v_{p-1} and accumulates <w, v_p> (or <w, w> in the last pass)
// in the same sweep, so each HBM byte of the basis is read once per column.  Passes are
// separated by a grid barrier with a bounded wait; every CTA sums the per-CTA partials in
// the same fixed order, so all CTAs hold bit-identical coefficients and the result is
// deterministic.  CTA 0 runs the Givens / stop-test epilogue.
#include "pb_epilogue.cuh"
#include "pb_mgs.cuh"

namespace pb {

constexpr unsigned kBarrierLimit = 1u << 22;

// Bounded grid barrier on a counter that is zero before its first use.
__device__ __forceinline__ void grid_barrier(unsigned* ctr, unsigned G, int* err) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(ctr, 1u);
    unsigned it = 0;
    while (*(volatile unsigned*)ctr < G) {
      if (++it > kBarrierLimit) { atomicExch(err, 1); break; }
      __nanosleep(20);
    }
    __threadfence();
  }
  __syncthreads();
}

template <class T, int ELEMS>
__global__ void __launch_bounds__(kMgsThreads, 2) k_gm_mgs(MgsArgs<T> a) {
  if (gated(a.gate)) return;
  __shared__ double wsum[kMgsThreads / 32];
  __shared__ double total;
  const unsigned G = gridDim.x;
  const int64_t nthr = (int64_t)G * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = a.j;
  T w[ELEMS];
#pragma unroll
  for (int e = 0; e < ELEMS; ++e) {
    const int64_t i = tid + e * nthr;
    w[e] = i < a.np ? a.w[i] : T(0);
  }
  double hprev = 0.0;
  for (int p = 1; p <= j + 1; ++p) {
    const T* vprev = a.V + (size_t)(p - 2) * a.ldv;
    const T* vcur = a.V + (size_t)(p - 1) * a.ldv;
    const T mh = (T)(-hprev);
    double part = 0.0;
    // Batches of EB elements: all loads of a batch are issued before any is used, so
    // every thread keeps 2*EB loads in flight.
    constexpr int EB = ELEMS < 8 ? ELEMS : 8;
    const bool upd = p > 1, dotv = p <= j;
#pragma unroll
    for (int e0 = 0; e0 < ELEMS; e0 += EB) {
      T vp[EB], vc[EB];
#pragma unroll
      for (int u = 0; u < EB; ++u) {
        const int64_t i = tid + (e0 + u) * nthr;
        const bool ok = i < a.np;
        vp[u] = (upd && ok) ? __ldcg(vprev + i) : T(0);
        vc[u] = (dotv && ok) ? __ldcs(vcur + i) : T(0);
      }
#pragma unroll
      for (int u = 0; u < EB; ++u) {
        T& we = w[e0 + u];
        if (upd) we = mh * vp[u] + we;                          // w = -h v + 1*w
        part += dotv ? (double)(we * vc[u]) : (double)(we * we);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    if (lane == 0) wsum[warp] = part;
    __syncthreads();
    double* parts = a.parts + (size_t)(p & 1) * G;
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += wsum[i];
      parts[blockIdx.x] = s;
    }
    grid_barrier(a.ctr + (p - 1), G, a.err);
    if (warp == 0) {
      double s = 0.0;
      for (unsigned b = lane; b < G; b += 32) s += __ldcg(parts + b);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
      if (lane == 0) total = s;
    }
    __syncthreads();
    const double S = total;
    if (p <= j) {
      hprev = S;
      if (blockIdx.x == 0 && threadIdx.x == 0) a.red.ea.h[(size_t)(j - 1) * (a.red.ea.m + 1) + (p - 1)] = S;
    } else {
      // v_{j+1} = (1/||w||) w
      if (a.vnext) {
        const T inv = (T)(1.0 / sqrt(S));
#pragma unroll
        for (int e = 0; e < ELEMS; ++e) {
          const int64_t i = tid + e * nthr;
          if (i < a.np) a.vnext[i] = inv * w[e];
        }
      }
      if (blockIdx.x == 0) {
        __shared__ double Sv[1];
        if (threadIdx.x == 0) Sv[0] = S;
        __syncthreads();
        epilogue(Sv, 1, a.red);   // EPI_GM_NORM: h(j+1,j), Givens, history, stop test
      }
    }
    __syncthreads();
  }
}

// Streaming variant for vectors too long to stay in registers (more than 32 elements per
// thread of the co-resident grid, e.g. 256^3 unknowns): w lives in global memory and is
// updated in place, pass p reading w, v_{p-1} and v_p and writing w, with the same
// operations in the same order as the register version.  Successive passes walk the rows
// in opposite directions, so a pass starts on the rows the previous one touched last,
// which are still in L2.  A final pass writes v_{j+1} = w / ||w||.
template <class T>
__global__ void __launch_bounds__(kMgsThreads, 2) k_gm_mgs_stream(MgsArgs<T> a) {
  if (gated(a.gate)) return;
  __shared__ double wsum[kMgsThreads / 32];
  __shared__ double total;
  constexpr int EB = 8;
  const unsigned G = gridDim.x;
  const int64_t nthr = (int64_t)G * blockDim.x;
  const int64_t tid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nb = (a.np + nthr * EB - 1) / (nthr * EB);   // batches of EB elements per thread
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = a.j;
  T* __restrict__ w = a.w;
  double hprev = 0.0, S = 0.0;
  for (int p = 1; p <= j + 1; ++p) {
    const T* vprev = a.V + (size_t)(p - 2) * a.ldv;
    const T* vcur = a.V + (size_t)(p - 1) * a.ldv;
    const T mh = (T)(-hprev);
    const bool upd = p > 1, dotv = p <= j;
    double part = 0.0;
    for (int64_t bb = 0; bb < nb; ++bb) {
      const int64_t b = (p & 1) ? bb : nb - 1 - bb;
      T wv[EB], vp[EB], vc[EB];
#pragma unroll
      for (int u = 0; u < EB; ++u) {
        const int64_t i = (b * EB + u) * nthr + tid;
        const bool ok = i < a.np;
        wv[u] = ok ? w[i] : T(0);
        // basis vectors stream with evict-first loads, so w (read and written every pass)
        // stays in L2 whenever it fits (an FP32 vector of 16.8M rows is 67 MB)
        vp[u] = (upd && ok) ? __ldcs(vprev + i) : T(0);
        vc[u] = (dotv && ok) ? __ldcs(vcur + i) : T(0);
      }
#pragma unroll
      for (int u = 0; u < EB; ++u) {
        const int64_t i = (b * EB + u) * nthr + tid;
        T we = wv[u];
        if (upd) we = mh * vp[u] + we;                          // w = -h v + 1*w
        part += dotv ? (double)(we * vc[u]) : (double)(we * we);
        if (upd && i < a.np) w[i] = we;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    if (lane == 0) wsum[warp] = part;
    __syncthreads();
    double* parts = a.parts + (size_t)(p & 1) * G;
    if (threadIdx.x == 0) {
      double s = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += wsum[i];
      parts[blockIdx.x] = s;
    }
    grid_barrier(a.ctr + (p - 1), G, a.err);
    if (warp == 0) {
      double s = 0.0;
      for (unsigned b = lane; b < G; b += 32) s += __ldcg(parts + b);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
      if (lane == 0) total = s;
    }
    __syncthreads();
    S = total;
    if (p <= j) {
      hprev = S;
      if (blockIdx.x == 0 && threadIdx.x == 0) a.red.ea.h[(size_t)(j - 1) * (a.red.ea.m + 1) + (p - 1)] = S;
    } else if (blockIdx.x == 0) {
      __shared__ double Sv[1];
      if (threadIdx.x == 0) Sv[0] = S;
      __syncthreads();
      epilogue(Sv, 1, a.red);   // EPI_GM_NORM: h(j+1,j), Givens, history, stop test
    }
    __syncthreads();
  }
  if (a.vnext) {   // v_{j+1} = (1/||w||) w; each thread rereads only what it wrote itself
    const T inv = (T)(1.0 / sqrt(S));
    for (int64_t bb = 0; bb < nb; ++bb) {
      const int64_t b = ((j + 2) & 1) ? bb : nb - 1 - bb;
#pragma unroll
      for (int u = 0; u < EB; ++u) {
        const int64_t i = (b * EB + u) * nthr + tid;
        if (i < a.np) a.vnext[i] = inv * w[i];
      }
    }
  }
}

template <class T>
int mgs_elems_needed(int64_t np, int grid) {
  int64_t nthr = (int64_t)grid * kMgsThreads;
  int64_t e = (np + nthr - 1) / nthr;
  for (int c : {1, 2, 4, 8, 16, 32})
    if (e <= c) return c;
  return -1;
}

template <class T>
static void launch_stream(const MgsArgs<T>& a, int grid, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kMgsThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PB_CUDA(cudaLaunchKernelEx(&cfg, k_gm_mgs_stream<T>, a));
}

template <class T, int E>
static void launch_e(const MgsArgs<T>& a, int grid, cudaStream_t st) {
  // Co-resident launch (the passes are separated by grid barriers).
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kMgsThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PB_CUDA(cudaLaunchKernelEx(&cfg, k_gm_mgs<T, E>, a));
}

template <class T>
int mgs_grid() {
  static int g = 0;
  if (!g) {
    int per = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gm_mgs<T, 32>, kMgsThreads, 0));
    g = std::max(1, std::min(per, 2)) * num_sms();
  }
  return g;
}

template <class T>
bool mgs_supported(int64_t np) {
  return np > 0;   // register-resident up to 32 elements per thread, streaming beyond
}

template <class T>
void mgs_column(const MgsArgs<T>& a, cudaStream_t st) {
  const int grid = mgs_grid<T>();
  switch (mgs_elems_needed<T>(a.np, grid)) {
    case 1: launch_e<T, 1>(a, grid, st); break;
    case 2: launch_e<T, 2>(a, grid, st); break;
    case 4: launch_e<T, 4>(a, grid, st); break;
    case 8: launch_e<T, 8>(a, grid, st); break;
    case 16: launch_e<T, 16>(a, grid, st); break;
    case 32: launch_e<T, 32>(a, grid, st); break;
    default: launch_stream<T>(a, grid, st); break;
  }
}

template bool mgs_supported<double>(int64_t);
template bool mgs_supported<float>(int64_t);
template void mgs_column<double>(const MgsArgs<double>&, cudaStream_t);
template void mgs_column<float>(const MgsArgs<float>&, cudaStream_t);
template int mgs_grid<double>();
template int mgs_grid<float>();

}  // namespace pb
