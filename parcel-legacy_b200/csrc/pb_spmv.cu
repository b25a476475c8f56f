// pb_spmv.cu -- CRS sparse matrix-vector product for B200.
//
// Replaces MatVec_crs (src/matrix.f90:1348-1512) on the CPU and cusparse_SpMV
// (src/CUDA/src/cusparse.cu:632-672) on the GPU, which the reference calls with four
// device synchronisations and a DnVec descriptor re-creation per product
// (src/krylov_h.f90:11-78).
//
// Layout: LPR lanes of a warp share a row (LPR from the mean row length: 8 for the
// 7-point stencils), so a warp covers 32/LPR consecutive rows whose nonzeros are
// contiguous and every value/column load is coalesced; each warp keeps UNR such row
// groups in flight to hide HBM latency.  Values and columns stream with evict-first loads
// (they are read once per product); x is gathered through the read-only path, where its
// stencil locality turns into L1/L2 hits.  The product can be fused with the residual
// b - A x and with one or two dot products that are reduced deterministically on the
// device.
#include "pb_device.cuh"
#include "pb_epilogue.cuh"
#include <algorithm>
#include <vector>

#include "pb_spmv.cuh"

namespace pb {

int spmv_lanes(int n, int64_t nnz) {
  double avg = n > 0 ? (double)nnz / n : 1.0;
  if (avg <= 2.0) return 2;
  if (avg <= 4.0) return 4;
  if (avg <= 10.0) return 8;
  if (avg <= 20.0) return 16;
  return 32;
}

template <class T> __device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }

template <int LPR, int UNR, class VT, class XT, int ND, bool RES>
__global__ void __launch_bounds__(kRedThreads, 4) k_spmv(int n, const int* __restrict__ rp,
                                                      const int* __restrict__ ci,
                                                      const VT* __restrict__ va, int rbase,
                                                      int cbase, const XT* __restrict__ x,
                                                      XT* __restrict__ y, const XT* __restrict__ b,
                                                      const XT* __restrict__ d, int sa0, int sb0,
                                                      int sa1, int sb1, Red red, const int* gate) {
  if (gated(gate)) return;
  constexpr int G = 32 / LPR;
  constexpr int TILE = G * UNR;
  const int lane = threadIdx.x & 31;
  const int g = lane / LPR, lg = lane % LPR;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int k = 0; k < (ND > 0 ? ND : 1); ++k) acc[k] = 0.0;

  for (int64_t base = warp * TILE; base < n; base += nwarps * TILE) {
    int beg[UNR], len[UNR];
    int maxlen = 0;
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
      int64_t row = base + u * G + g;
      if (row < n) {
        beg[u] = __ldg(rp + row) - rbase;
        len[u] = __ldg(rp + row + 1) - rbase - beg[u];
      } else {
        beg[u] = 0;
        len[u] = 0;
      }
      maxlen = max(maxlen, len[u]);
    }
    XT sum[UNR];
#pragma unroll
    for (int u = 0; u < UNR; ++u) sum[u] = XT(0);
    for (int k = lg; k < maxlen; k += LPR) {
      VT v[UNR];
      int c[UNR];
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        if (k < len[u]) {
          v[u] = ld_stream(va + beg[u] + k);
          c[u] = ld_stream(ci + beg[u] + k) - cbase;
        } else {
          v[u] = VT(0);
          c[u] = -1;
        }
      }
#pragma unroll
      for (int u = 0; u < UNR; ++u)
        if (c[u] >= 0) sum[u] += (XT)v[u] * __ldg(x + c[u]);
    }
#pragma unroll
    for (int u = 0; u < UNR; ++u) {
#pragma unroll
      for (int o = LPR / 2; o > 0; o >>= 1) sum[u] += __shfl_xor_sync(kFull, sum[u], o);
    }
    if (lg == 0) {
#pragma unroll
      for (int u = 0; u < UNR; ++u) {
        int64_t row = base + u * G + g;
        if (row < n) {
          XT yv = RES ? b[row] - sum[u] : sum[u];
          y[row] = yv;
          if constexpr (ND > 0) {
            XT src[3] = {yv, x[row], d ? d[row] : XT(0)};
            acc[0] += (double)(src[sa0] * src[sb0]);
            if (ND > 1) acc[ND > 1 ? 1 : 0] += (double)(src[sa1] * src[sb1]);
          }
        }
      }
    }
  }
  if constexpr (ND > 0) reduce_and_finish<ND>(acc, red);
}

// Sliced-ELLPACK SpMV: one thread per row, all of a row's value/column loads issued
// before its x gathers.
template <class VT, class XT, int ND, bool RES>
__global__ void __launch_bounds__(kRedThreads, 4) k_spmv_sell(int n, int nslices, const int* __restrict__ soff,
                                                           const int* __restrict__ sw,
                                                           const int* __restrict__ ci,
                                                           const VT* __restrict__ va,
                                                           const XT* __restrict__ x, XT* __restrict__ y,
                                                           const XT* __restrict__ b, const XT* __restrict__ d,
                                                           int sa0, int sb0, int sa1, int sb1, Red red,
                                                           const int* gate) {
  if (gated(gate)) return;
  constexpr int U = 8;
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int k = 0; k < (ND > 0 ? ND : 1); ++k) acc[k] = 0.0;
  for (int s = warp; s < nslices; s += nwarps) {
    const int off = __ldg(soff + s) + lane;
    const int w = __ldg(sw + s);
    const int row = s * 32 + lane;
    XT sum = XT(0);
    for (int k0 = 0; k0 < w; k0 += U) {
      VT v[U];
      int c[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u < w) {
          v[u] = __ldcs(va + off + (k0 + u) * 32);
          c[u] = __ldcs(ci + off + (k0 + u) * 32);
        } else {
          v[u] = VT(0);
          c[u] = row < n ? row : 0;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) sum += (XT)v[u] * __ldg(x + c[u]);
    }
    if (row < n) {
      XT yv = RES ? b[row] - sum : sum;
      y[row] = yv;
      if constexpr (ND > 0) {
        XT src[3] = {yv, x[row], d ? d[row] : XT(0)};
        acc[0] += (double)(src[sa0] * src[sb0]);
        if (ND > 1) acc[ND > 1 ? 1 : 0] += (double)(src[sa1] * src[sb1]);
      }
    }
  }
  if constexpr (ND > 0) reduce_and_finish<ND>(acc, red);
}

// Position of row r's entry on diagonal k in the diagonal copy: sliced like the ELLPACK copy
// (32-row slices, the slice's diagonals one after the other, 32 values each), so that a
// warp reads one contiguous run of 32 nd values per slice; only the column indices are
// gone.  (Diagonal-major storage, each diagonal a separate array, ran at half the speed.)
__host__ __device__ __forceinline__ int64_t dia_at(int64_t r, int k, int nd) {
  return (r & ~int64_t(31)) * nd + (int64_t)k * 32 + (r & 31);
}

// Diagonal-format SpMV (natural layout): one thread per row, the diagonals in ascending
// offset order, so a row's products are summed in its CRS column order (an absent entry
// contributes an exact zero).  Values stream coalesced and without column indices; the
// x gathers of neighbouring rows are contiguous.
template <class VT, class XT, int ND, bool RES>
__global__ void __launch_bounds__(kRedThreads, 4) k_spmv_dia(int n, int nd, const int* __restrict__ doff,
                                                       const VT* __restrict__ dval, const XT* __restrict__ x,
                                                       XT* __restrict__ y, const XT* __restrict__ b,
                                                       const XT* __restrict__ d, int sa0, int sb0, int sa1,
                                                       int sb1, Red red, const int* gate) {
  if (gated(gate)) return;
  __shared__ int offs[kDiaMaxDiag];
  if (threadIdx.x < nd) offs[threadIdx.x] = doff[threadIdx.x];
  __syncthreads();
  double acc[ND > 0 ? ND : 1];
#pragma unroll
  for (int k = 0; k < (ND > 0 ? ND : 1); ++k) acc[k] = 0.0;
  // a warp takes whole 32-row slices, the grid's warps consecutive ones, so that all warps
  // together sweep the copy front to back (as the sliced-ELLPACK product does)
  const int lane = threadIdx.x & 31;
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int nslices = (n + 31) >> 5;
  for (int sl = warp; sl < nslices; sl += nwarps) {
    const int row = sl * 32 + lane;
    if (row >= n) continue;
    VT v[kDiaMaxDiag];
#pragma unroll
    for (int k = 0; k < kDiaMaxDiag; ++k)
      if (k < nd) v[k] = __ldcs(dval + dia_at(row, k, nd));
    XT sum = XT(0);
#pragma unroll
    for (int k = 0; k < kDiaMaxDiag; ++k) {
      if (k < nd) {
        int c = row + offs[k];
        c = c < 0 ? 0 : (c >= n ? n - 1 : c);     // out of the matrix: the stored value is zero
        sum += (XT)v[k] * __ldg(x + c);
      }
    }
    XT yv = RES ? b[row] - sum : sum;
    y[row] = yv;
    if constexpr (ND > 0) {
      XT src[3] = {yv, x[row], d ? d[row] : XT(0)};
      acc[0] += (double)(src[sa0] * src[sb0]);
      if (ND > 1) acc[ND > 1 ? 1 : 0] += (double)(src[sa1] * src[sb1]);
    }
  }
  if constexpr (ND > 0) reduce_and_finish<ND>(acc, red);
}

template <class VT, class XT, int ND, bool RES>
static void launch_spmv(const DevMat<VT>& A, const XT* x, XT* y, const XT* b, const XT* d,
                        const int* sa, const int* sb, const Red& red, const int* gate,
                        cudaStream_t st) {
  const int lpr = spmv_lanes(A.n, A.nnz);
  const int grid = red_blocks();
  int a0 = sa ? sa[0] : 0, b0 = sb ? sb[0] : 0, a1 = sa ? sa[1] : 0, b1 = sb ? sb[1] : 0;
  if (A.d_val) {
    k_spmv_dia<VT, XT, ND, RES><<<grid, kRedThreads, 0, st>>>(A.n, A.ndiag, A.d_off, A.d_val, x, y, b, d, a0, b0,
                                                             a1, b1, red, gate);
    PB_CUDA(cudaGetLastError());
    return;
  }
  if (A.s_val) {
    k_spmv_sell<VT, XT, ND, RES><<<grid, kRedThreads, 0, st>>>(A.n, A.nslices, A.s_off, A.s_w, A.s_col,
                                                              A.s_val, x, y, b, d, a0, b0, a1, b1, red,
                                                              gate);
    PB_CUDA(cudaGetLastError());
    return;
  }
#define L(LPR_, UNR_)                                                                         \
  k_spmv<LPR_, UNR_, VT, XT, ND, RES><<<grid, kRedThreads, 0, st>>>(                          \
      A.n, A.rowptr, A.col, A.val, A.rbase, A.cbase, x, y, b, d, a0, b0, a1, b1, red, gate)
  switch (lpr) {
    case 2: L(2, 4); break;
    case 4: L(4, 4); break;
    case 8: L(8, 4); break;
    case 16: L(16, 2); break;
    default: L(32, 1); break;
  }
#undef L
  PB_CUDA(cudaGetLastError());
}

template <class VT, class XT>
void spmv(const DevMat<VT>& A, const XT* x, XT* y, int mode, const XT* b, const int* gate,
          cudaStream_t st) {
  Red red{};
  if (mode == SPMV_RES) launch_spmv<VT, XT, 0, true>(A, x, y, b, nullptr, nullptr, nullptr, red, gate, st);
  else launch_spmv<VT, XT, 0, false>(A, x, y, b, nullptr, nullptr, nullptr, red, gate, st);
}

template <class VT, class XT>
void spmv_dot(const DevMat<VT>& A, const XT* x, XT* y, int mode, const XT* b, const XT* d,
              int nd, const int* sa, const int* sb, const Red& red, const int* gate,
              cudaStream_t st) {
  if (nd == 1) {
    if (mode == SPMV_RES) launch_spmv<VT, XT, 1, true>(A, x, y, b, d, sa, sb, red, gate, st);
    else launch_spmv<VT, XT, 1, false>(A, x, y, b, d, sa, sb, red, gate, st);
  } else {
    if (mode == SPMV_RES) launch_spmv<VT, XT, 2, true>(A, x, y, b, d, sa, sb, red, gate, st);
    else launch_spmv<VT, XT, 2, false>(A, x, y, b, d, sa, sb, red, gate, st);
  }
}

template <class VT>
__global__ void k_fill_sell(int np, const int* __restrict__ rowAt, const int* __restrict__ pos,
                            const int* __restrict__ rp, const int* __restrict__ ci,
                            const double* __restrict__ va, int rbase, int cbase,
                            const int* __restrict__ soff, const int* __restrict__ sw,
                            int* __restrict__ scol, VT* __restrict__ sval) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < ((np + 31) & ~31); q += gridDim.x * blockDim.x) {
    const int s = q >> 5, lane = q & 31;
    const int w = sw[s];
    const int base = soff[s] + lane;
    int i = (q < np) ? (rowAt ? rowAt[q] : q) : -1;
    int a = 0, len = 0;
    if (i >= 0) { a = rp[i] - rbase; len = rp[i + 1] - rbase - a; }
    const int self = q < np ? q : 0;
    for (int k = 0; k < w; ++k) {
      if (k < len) {
        const int c = ci[a + k] - cbase;
        scol[base + 32 * k] = pos ? pos[c] : c;
        sval[base + 32 * k] = (VT)va[a + k];
      } else {
        scol[base + 32 * k] = self;
        sval[base + 32 * k] = VT(0);
      }
    }
  }
}

// Slice widths: the longest of the 32 rows of each slice (warp per slice).
__global__ void k_sell_width(int np, const int* __restrict__ rowAt, const int* __restrict__ rp,
                             int* __restrict__ sw) {
  const int ns = (np + 31) >> 5;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < (ns << 5); q += gridDim.x * blockDim.x) {
    int len = 0;
    if (q < np) {
      const int i = rowAt ? rowAt[q] : q;
      if (i >= 0) len = rp[i + 1] - rp[i];
    }
    len = __reduce_max_sync(kFull, len);
    if ((q & 31) == 0) sw[q >> 5] = len;
  }
}

// Slice offsets off[s] = 32 * (w[0] + ... + w[s-1]) for s = 0..ns, one block; the 64-bit
// total goes to *total so that the host can check it against the int32 range.
constexpr int kSellScanThreads = 1024;
__global__ void __launch_bounds__(kSellScanThreads) k_sell_offsets(int ns, const int* __restrict__ sw,
                                                                   int* __restrict__ off,
                                                                   long long* __restrict__ total) {
  __shared__ long long part[kSellScanThreads];
  const int t = threadIdx.x;
  const int per = (ns + kSellScanThreads - 1) / kSellScanThreads;
  const int a = min(ns, t * per), z = min(ns, a + per);
  long long loc = 0;
  for (int s = a; s < z; ++s) loc += 32LL * sw[s];
  part[t] = loc;
  __syncthreads();
  for (int d = 1; d < kSellScanThreads; d <<= 1) {   // inclusive scan of the per-thread sums
    const long long v = t >= d ? part[t - d] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  long long run = part[t] - loc;
  for (int s = a; s < z; ++s) {
    off[s] = (int)min(run, (long long)INT32_MAX);
    run += 32LL * sw[s];
  }
  if (t == kSellScanThreads - 1) {
    off[ns] = (int)min(part[t], (long long)INT32_MAX);
    *total = part[t];
  }
}

template <class VT>
void build_sell(const DevMat<double>& A, int np, const int* rowAt_d, const int* pos_d, SellBuf<VT>& buf,
                DevMat<VT>& M) {
  cudaStream_t st = stream();
  const int ns = (np + 31) / 32;
  buf.off.alloc(sizeof(int) * (ns + 1));
  buf.w.alloc(sizeof(int) * std::max(ns, 1));
  DBuf tot(sizeof(long long));
  const int grid = (int)std::min<int64_t>(((int64_t)ns * 32 + 255) / 256, 8LL * num_sms());
  k_sell_width<<<std::max(grid, 1), 256, 0, st>>>(np, rowAt_d, A.rowptr, dp<int>(buf.w));
  PB_CUDA(cudaGetLastError());
  k_sell_offsets<<<1, kSellScanThreads, 0, st>>>(ns, dp<int>(buf.w), dp<int>(buf.off), dp<long long>(tot));
  PB_CUDA(cudaGetLastError());
  long long total = 0;
  d2h(&total, tot.p, sizeof(long long));
  PB_CHECK(total < INT32_MAX, PARCEL_B_E_UNSUPPORTED, "matrix too large for int32 SELL");
  total = std::max(total, 1LL);
  buf.col.alloc(sizeof(int) * total);
  buf.val.alloc(sizeof(VT) * total);
  k_fill_sell<VT><<<8 * num_sms(), 256, 0, st>>>(np, rowAt_d, pos_d, A.rowptr, A.col, A.val, A.rbase,
                                                 A.cbase, dp<int>(buf.off), dp<int>(buf.w),
                                                 dp<int>(buf.col), dp<VT>(buf.val));
  PB_CUDA(cudaGetLastError());
  M.nslices = ns;
  M.s_off = dp<int>(buf.off);
  M.s_w = dp<int>(buf.w);
  M.s_col = dp<int>(buf.col);
  M.s_val = dp<VT>(buf.val);
  M.n = np;
}

// Any entry off the candidate diagonals sets *miss.
__global__ void k_dia_check(int n, const int* __restrict__ rp, const int* __restrict__ ci, int rbase, int cbase,
                            int nd, const int* __restrict__ doff, int* __restrict__ miss) {
  __shared__ int offs[kDiaMaxDiag];
  if (threadIdx.x < nd) offs[threadIdx.x] = doff[threadIdx.x];
  __syncthreads();
  bool bad = false;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int e = rp[r] - rbase; e < rp[r + 1] - rbase; ++e) {
      const int o = ci[e] - cbase - r;
      bool hit = false;
      for (int k = 0; k < nd; ++k) hit |= offs[k] == o;
      bad |= !hit;
    }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(miss, 1);
}

template <class VT>
__global__ void k_dia_fill(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                           const double* __restrict__ va, int rbase, int cbase, int nd, const int* __restrict__ doff,
                           VT* __restrict__ dval) {
  __shared__ int offs[kDiaMaxDiag];
  if (threadIdx.x < nd) offs[threadIdx.x] = doff[threadIdx.x];
  __syncthreads();
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (int e = rp[r] - rbase; e < rp[r + 1] - rbase; ++e) {
      const int o = ci[e] - cbase - r;
      for (int k = 0; k < nd; ++k)
        if (offs[k] == o) dval[dia_at(r, k, nd)] = (VT)va[e];
    }
}

// Row t of 64 sample rows scattered over the matrix (a multiplicative hash of t, so that a
// stencil's boundary rows, which lie on regular strides, do not make up the sample):
// out[t][0] = its entry count (more than kDiaMaxDiag: only the count), out[t][1..] = its
// column offsets.
__global__ void k_dia_sample(int n, const int* __restrict__ rp, const int* __restrict__ ci, int rbase, int cbase,
                             int* __restrict__ out) {
  const int t = threadIdx.x;
  const int r = (int)(((uint64_t)(t + 1) * 2654435761ull) % (uint64_t)n);
  int* o = out + t * (kDiaMaxDiag + 1);
  const int b = rp[r] - rbase, e = rp[r + 1] - rbase;
  o[0] = e - b;
  if (e - b <= kDiaMaxDiag)
    for (int k = b; k < e; ++k) o[1 + k - b] = ci[k] - cbase - r;
}

template <class VT>
int build_dia(const DevMat<double>& A, SellBuf<VT>& buf, DevMat<VT>& M) {
  cudaStream_t st = stream();
  const int n = A.n;
  if (n < 2) return 0;
  // candidate diagonals: the offsets found in 64 rows scattered over the matrix (interior
  // rows of a stencil carry all of them, boundary rows a subset), gathered in one launch
  constexpr int kSamples = 64;
  DBuf sm(sizeof(int) * kSamples * (kDiaMaxDiag + 1));
  k_dia_sample<<<1, kSamples, 0, st>>>(n, A.rowptr, A.col, A.rbase, A.cbase, dp<int>(sm));
  PB_CUDA(cudaGetLastError());
  std::vector<int> hs(kSamples * (kDiaMaxDiag + 1));
  d2h(hs.data(), sm.p, sizeof(int) * hs.size());
  std::vector<int> offs;
  for (int t = 0; t < kSamples; ++t) {
    const int len = hs[t * (kDiaMaxDiag + 1)];
    if (len > kDiaMaxDiag) return 0;
    for (int k = 0; k < len; ++k) offs.push_back(hs[t * (kDiaMaxDiag + 1) + 1 + k]);
  }
  std::sort(offs.begin(), offs.end());
  offs.erase(std::unique(offs.begin(), offs.end()), offs.end());
  if ((int)offs.size() > kDiaMaxDiag) return 0;
  if (offs.empty()) return 0;
  const int nd = (int)offs.size();
  if ((double)nd * n > 1.5 * (double)std::max<int64_t>(A.nnz, 1)) return 0;
  buf.doff.alloc(sizeof(int) * kDiaMaxDiag);
  h2d(buf.doff.p, offs.data(), sizeof(int) * nd);
  DBuf miss(sizeof(int));
  PB_CUDA(cudaMemsetAsync(miss.p, 0, sizeof(int), st));
  const int grid = std::max(1, std::min((n + 255) / 256, 8 * num_sms()));
  k_dia_check<<<grid, 256, 0, st>>>(n, A.rowptr, A.col, A.rbase, A.cbase, nd, dp<int>(buf.doff), dp<int>(miss));
  PB_CUDA(cudaGetLastError());
  int m = 0;
  d2h(&m, miss.p, sizeof(int));
  if (m) return 0;
  buf.dval.alloc(sizeof(VT) * (size_t)nd * (((size_t)n + 31) & ~size_t(31)));   // zero-filled
  k_dia_fill<VT><<<grid, 256, 0, st>>>(n, A.rowptr, A.col, A.val, A.rbase, A.cbase, nd, dp<int>(buf.doff),
                                       dp<VT>(buf.dval));
  PB_CUDA(cudaGetLastError());
  M.ndiag = nd;
  M.d_off = dp<int>(buf.doff);
  M.d_val = dp<VT>(buf.dval);
  return nd;
}

template int build_dia<double>(const DevMat<double>&, SellBuf<double>&, DevMat<double>&);
template int build_dia<float>(const DevMat<double>&, SellBuf<float>&, DevMat<float>&);

template void build_sell<double>(const DevMat<double>&, int, const int*, const int*, SellBuf<double>&,
                                 DevMat<double>&);
template void build_sell<float>(const DevMat<double>&, int, const int*, const int*, SellBuf<float>&,
                                DevMat<float>&);

template void spmv<double, double>(const DevMat<double>&, const double*, double*, int,
                                   const double*, const int*, cudaStream_t);
template void spmv<float, float>(const DevMat<float>&, const float*, float*, int, const float*,
                                 const int*, cudaStream_t);
template void spmv_dot<double, double>(const DevMat<double>&, const double*, double*, int,
                                       const double*, const double*, int, const int*, const int*,
                                       const Red&, const int*, cudaStream_t);
template void spmv_dot<float, float>(const DevMat<float>&, const float*, float*, int,
                                     const float*, const float*, int, const int*, const int*,
                                     const Red&, const int*, cudaStream_t);

}  // namespace pb
