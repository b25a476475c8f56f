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


// Shared-memory-staged variant, for vectors of which the grid's shared memory holds two
// copies (about 2.1M FP64 or 4.2M FP32 rows on 148 SMs).  One CTA per SM owns a contiguous
// range of R rows: w stays in the registers of 15 consumer warps, and the CTA's slices of
// two basis vectors sit in shared memory -- v_{p-1} (for the update) and v_p (for the dot
// product), v_k in buffer k & 1.  A producer warp moves the slices with bulk copies (TMA)
// in chunks of kMgsChunk elements per consumer thread; all chunks of one copy of a vector
// complete on full[q] (one wait per pass: the copy of v_p is issued a whole pass before it
// is needed, and 15 warps polling one mbarrier word per chunk cost more than the chunks'
// arrival times could save).  The consumers release chunk c of v_{p-1} on empty[q][c] as
// soon as pass p has read it, whereupon the producer refills it with v_{p+1}.  Copy issue
// blocks under memory back-pressure, so it lives in its own warp: the consumers' sweep
// never waits for an issue, and the copy queue stays full while the grid reduction runs.
// Every basis byte is read from HBM once per column.
//
// Grid reduction without a counter: CTA b stores its partial sum of pass p in slot
// (p, b); warp 0 of CTA 0 waits until the pass's G slots are all written, sums them in a
// fixed order and stores the total in total(p); every CTA waits for total(p).  All slots
// hold the all-ones bit pattern (a NaN no arithmetic produces) before the launch and are
// written once per launch; a partial or total that is itself a NaN is stored as the
// canonical quiet NaN, so that it cannot read as empty.  Two L2 round trips per pass;
// an all-to-all read of the slots costs more because 148 CTAs contend for the same lines.
// Waits are bounded: a wait that runs out sets *err, and the CTA stops waiting and
// issuing, then waits (bounded) for the copies it has in flight before it exits.
// 15 consumer warps and one producer warp: 4 warps per SM sub-partition, so that each
// thread can hold 128 registers (a 17th warp would cap them at 96)
constexpr int kMgsConsumers = 480;
constexpr int kMgsTmaThreads = kMgsConsumers + 32;
constexpr int kMgsChunk = 4;                          // elements per consumer per chunk
constexpr unsigned long long kMgsEmpty = ~0ull;       // empty slot
constexpr unsigned kSlotLimit = 1u << 21;
constexpr unsigned kCopyLimit = 1u << 20;
constexpr int kMgsSlotsPerLane = 8;                   // grids of up to 256 CTAs

__device__ __forceinline__ unsigned long long ld_slot(const double* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_slot(double* p, double v) {
  if (v != v) v = __longlong_as_double(0x7ff8000000000000ll);
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(__double_as_longlong(v)) : "memory");
}

template <class T, int ELEMS>
__global__ void __launch_bounds__(kMgsTmaThreads, 1) k_gm_mgs_tma(MgsArgs<T> a, int R) {
  if (gated(a.gate)) return;
  constexpr int NT = kMgsConsumers, CH = NT * kMgsChunk, NC = (ELEMS + kMgsChunk - 1) / kMgsChunk;
  extern __shared__ __align__(128) unsigned char mgs_smem[];
  __shared__ __align__(8) uint64_t full[2], empty[2][NC];
  __shared__ double wsum[NT / 32];
  __shared__ double total;
  __shared__ int sbad;
  T* const b0 = reinterpret_cast<T*>(mgs_smem);
  T* const b1 = b0 + R;
  const int G = gridDim.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int j = a.j;
  const int64_t row0 = (int64_t)blockIdx.x * R;
  const int rows = (int)max((int64_t)0, min((int64_t)R, a.np - row0));   // rows owned
  const int crows = (rows + 31) & ~31;   // rows copied (within ldv: ldv is a multiple of 32)
  const int nch = (crows + CH - 1) / CH;
  if (t == 0) {
    for (int q = 0; q < 2; ++q) {
      mbar_init(&full[q], 1);
      for (int c = 0; c < NC; ++c) mbar_init(&empty[q][c], NT / 32);
    }
    sbad = 0;
    mbar_fence_init();
  }
  __syncthreads();
  double S = 0.0;
  int last0 = 0, last1 = 0;   // (producer) last vector whose copy into buffer 0 / 1 is complete
  if (warp == NT / 32) {
    // ---------------------------------------------------------------- producer warp
    if (lane == 0 && nch > 0) {   // a CTA without rows copies and waits for nothing
      // chunk c of v_k into buffer k & 1; the arrival after the last chunk closes the copy
      auto issue = [&](int k, int c) {
        const int r0 = c * CH, nr = min(CH, crows - r0);
        const unsigned bytes = (unsigned)(nr * sizeof(T));
        mbar_expect_tx(&full[k & 1], bytes);
        bulk_g2s(((k & 1) ? b1 : b0) + r0, a.V + (size_t)(k - 1) * a.ldv + row0 + r0, bytes, &full[k & 1]);
      };
      auto close = [&](int k) {
        mbar_arrive(&full[k & 1]);
        if (k & 1) last1 = k; else last0 = k;
      };
      auto fail = [&] {
        sbad = 1;
        atomicExch(a.err, 1);
      };
      for (int c = 0; c < nch; ++c) issue(1, c);
      close(1);
      // v_2 streams while pass 1 runs: w and v_1 get the bandwidth first
      if (j >= 2) {
        if (mbar_wait(&full[1], 0, kCopyLimit)) {
          for (int c = 0; c < nch; ++c) issue(2, c);
          close(2);
        } else {
          fail();
        }
      }
      // v_k (k >= 3) replaces v_{k-2}, released in pass k-1: the ((k-3)/2)-th release.
      // A failed wait still closes the copy, so that its phase completes once the chunks
      // already issued have landed.
      for (int k = 3; k <= j && !sbad; ++k) {
        for (int c = 0; c < nch; ++c) {
          if (!mbar_wait(&empty[k & 1][c], ((k - 3) >> 1) & 1, kCopyLimit)) {
            fail();
            break;
          }
          issue(k, c);
        }
        close(k);
      }
    }
  } else {
    // ---------------------------------------------------------------- consumer warps
    T w[ELEMS];
#pragma unroll
    for (int e = 0; e < ELEMS; ++e) {
      const int lr = t + e * NT;
      w[e] = lr < rows ? a.w[row0 + lr] : T(0);
    }
    double hprev = 0.0;
    for (int p = 1; p <= j + 1; ++p) {
      const bool upd = p > 1, dotv = p <= j, release = upd && p + 1 <= j;
      const T mh = (T)(-hprev);
      const T* bu = (p & 1) ? b0 : b1;   // v_{p-1}
      const T* bd = (p & 1) ? b1 : b0;   // v_p
      const unsigned par = ((p - 1) >> 1) & 1;   // v_p is the ((p-1)/2)-th copy into its buffer
      double part = 0.0;
      if (dotv && nch > 0 && !sbad && !mbar_wait(&full[p & 1], par, kCopyLimit)) {
        sbad = 1;
        atomicExch(a.err, 1);
      }
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        if (c < nch) {
#pragma unroll
          for (int u = 0; u < kMgsChunk; ++u) {
            const int e = c * kMgsChunk + u, lr = t + e * NT;
            if (e < ELEMS && lr < rows) {
              T& we = w[e];
              if (upd) we = mh * bu[lr] + we;                          // w = -h v + 1*w
              part += dotv ? (double)(we * bd[lr]) : (double)(we * we);
            }
          }
          if (release) {   // this warp is done with chunk c of v_{p-1}
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[(p - 1) & 1][c]);
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
      if (lane == 0) wsum[warp] = part;
      named_bar_sync(1, NT);
      if (warp == 0) {
        double* sl = a.slots + (size_t)(p - 1) * G;
        if (lane == 0) {
          double s = 0.0;
          for (int i = 0; i < NT / 32; ++i) s += wsum[i];
          st_slot(sl + blockIdx.x, s);
        }
        bool bad = sbad != 0;
        if (blockIdx.x == 0) {   // aggregator: all partial loads in flight at once
          unsigned long long v[kMgsSlotsPerLane];
#pragma unroll
          for (int i = 0; i < kMgsSlotsPerLane; ++i)
            v[i] = lane + 32 * i < G ? ld_slot(sl + lane + 32 * i) : 0ull;
          for (unsigned it = 0;; ++it) {
            bool pending = false;
#pragma unroll
            for (int i = 0; i < kMgsSlotsPerLane; ++i) pending |= v[i] == kMgsEmpty;
            if (!pending || bad) break;
            if (it >= kSlotLimit) {
              bad = true;
              break;
            }
#pragma unroll
            for (int i = 0; i < kMgsSlotsPerLane; ++i)
              if (v[i] == kMgsEmpty) v[i] = ld_slot(sl + lane + 32 * i);
          }
          double s = 0.0;
#pragma unroll
          for (int i = 0; i < kMgsSlotsPerLane; ++i) s += __longlong_as_double(v[i]);
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
          if (lane == 0) st_slot(a.totals + (p - 1), s);
        }
        if (lane == 0) {
          unsigned long long v = ld_slot(a.totals + (p - 1));
          for (unsigned it = 0; v == kMgsEmpty && !bad; v = ld_slot(a.totals + (p - 1)))
            if (++it > kSlotLimit) bad = true;
          total = __longlong_as_double(v);
        }
        if (__any_sync(kFull, bad) && lane == 0) {
          sbad = 1;
          atomicExch(a.err, 1);
        }
      }
      named_bar_sync(1, NT);
      S = total;
      if (p <= j) {
        hprev = S;
        if (blockIdx.x == 0 && t == 0) a.red.ea.h[(size_t)(j - 1) * (a.red.ea.m + 1) + (p - 1)] = S;
      } else if (a.vnext) {   // v_{j+1} = (1/||w||) w
        const T inv = (T)(1.0 / sqrt(S));
#pragma unroll
        for (int e = 0; e < ELEMS; ++e) {
          const int lr = t + e * NT;
          if (lr < rows) a.vnext[row0 + lr] = inv * w[e];
        }
      }
    }
  }
  __syncthreads();   // producer and consumers
  if (blockIdx.x == 0 && t == 0) epilogue(&S, 1, a.red);   // EPI_GM_NORM: h(j+1,j), Givens, stop test
  if (sbad && t == NT) {
    // After a failed wait the consumers may not have waited for every copy: wait (bounded)
    // for the last copy into each buffer (every copy is closed, so its phase completes
    // once its bytes have landed; the copies before it into the same buffer had completed).
    for (int q = 0; q < 2; ++q) {
      const int k = q ? last1 : last0;
      if (k > 0) mbar_wait(&full[q], ((k - 1) >> 1) & 1, kCopyLimit);
    }
  }}

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

// Rows per CTA of the staged variant (a multiple of 32), or 0 when two slices of that
// length do not fit one CTA's shared memory or 35 elements per consumer thread.
template <class T>
static int mgs_tma_rows(int64_t np) {
  static int cap = -1;
  if (cap < 0) {
    int optin = 0, dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    PB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cudaFuncAttributes fa;
    PB_CUDA(cudaFuncGetAttributes(&fa, k_gm_mgs_tma<T, 35>));   // the most static shared memory
    cap = std::max(0, optin - (int)fa.sharedSizeBytes);
    for (auto f : {k_gm_mgs_tma<T, 4>, k_gm_mgs_tma<T, 8>, k_gm_mgs_tma<T, 16>, k_gm_mgs_tma<T, 24>,
                   k_gm_mgs_tma<T, 31>, k_gm_mgs_tma<T, 35>})
      PB_CUDA(cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, cap));
  }
  const int G = num_sms();
  if (np <= 0 || G <= 0 || G > 32 * kMgsSlotsPerLane) return 0;
  const int64_t R = (((np + G - 1) / G) + 31) & ~int64_t(31);
  if (R > 35 * kMgsConsumers || 2 * R * (int64_t)sizeof(T) > cap) return 0;
  return (int)R;
}

template <class T>
bool mgs_staged(int64_t np) {
  return mgs_tma_rows<T>(np) > 0;
}

template <class T, int E>
static void launch_tma(const MgsArgs<T>& a, int R, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(num_sms());
  cfg.blockDim = dim3(kMgsTmaThreads);
  cfg.dynamicSmemBytes = 2 * (size_t)R * sizeof(T);
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  PB_CUDA(cudaLaunchKernelEx(&cfg, k_gm_mgs_tma<T, E>, a, R));
}

template <class T>
bool mgs_supported(int64_t np) {
  return np > 0;   // register-resident up to 32 elements per thread, streaming beyond
}

template <class T>
void mgs_column(const MgsArgs<T>& a, cudaStream_t st) {
  if (const int R = mgs_tma_rows<T>(a.np)) {
    PB_CHECK(a.slots != nullptr && a.totals != nullptr, PARCEL_B_E_ARG, "staged MGS launched without slots");
    if (R <= 4 * kMgsConsumers) launch_tma<T, 4>(a, R, st);
    else if (R <= 8 * kMgsConsumers) launch_tma<T, 8>(a, R, st);
    else if (R <= 16 * kMgsConsumers) launch_tma<T, 16>(a, R, st);
    else if (R <= 24 * kMgsConsumers) launch_tma<T, 24>(a, R, st);
    else if (R <= 31 * kMgsConsumers) launch_tma<T, 31>(a, R, st);
    else launch_tma<T, 35>(a, R, st);
    return;
  }
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
template bool mgs_staged<double>(int64_t);
template bool mgs_staged<float>(int64_t);

}  // namespace pb
