// pb_cagmres.cu -- CA-GMRES(s, t) on B200.
//
// Reference: KSP_pCAGMRES (src/pcagmres.f90:1557-2518) with calc_NewtonBasis(Vec)
// (:586-611, 1480-1552), calc_HessenbergMatrix (:879-1052), GivensRotations (:190-242),
// getHessenbergMat_Eigen + modified_leja_ordering (:613-742, src/LejaOrdering.f90:100-322),
// QRDecomposition_ (src/QRDecomposition.f90:1331-1552; R-only TSQR / Cholesky QR, then
// Q = V R^-1) and the update of x (update_xVec, pcagmres.f90:1136-1236).
//
// Device work per block of s basis vectors: s preconditioned SpMVs (the matrix-powers
// step), one tall-skinny product Q^T V (shared-memory tiles, deterministic two-stage sum),
// the block update V -= Q R, an R-only QR of the (s+1)-column panel (warp-level
// structured Householder TSQR with a recursive reduction of the per-warp R factors, or
// Cholesky QR / Cholesky QR2 from the Gram matrix), and Q = V R^-1.  The s x s algebra
// (Hessenberg reconstruction, Givens rotations, Ritz values, Leja ordering) runs on the
// host, as in the reference.
//
// Two deliberate differences from the reference, both documented in the design notes:
// Q is formed for every block (the reference keeps R only for the last block of a cycle
// and corrects the update with R^-1: identical in exact arithmetic), and the Newton
// recurrence for a complex shift pair uses the sign that matches the change-of-basis
// matrix the Hessenberg is built from (the reference's two signs disagree, which detaches
// its residual estimate from the true residual whenever Ritz values are complex).
#include <cmath>

#include "pb_dense.hpp"
#include "pb_mixed.cuh"

namespace pb {

using dense::Mat;

// ------------------------------------------------------------------ device kernels
constexpr int kTsRows = 32;      // rows per shared-memory tile
constexpr int kTsMaxPQ = 1024;   // max p*q of one tall-skinny product

// Partial C = A^T B over this block's row tiles; A: p columns, B: q columns.
__global__ void __launch_bounds__(256) k_tsgemm_atb(int64_t n, const double* __restrict__ A, int64_t lda,
                                                    int p, const double* __restrict__ B, int64_t ldb,
                                                    int q, double* __restrict__ part) {
  extern __shared__ double sh[];
  double* As = sh;                       // [p][kTsRows]
  double* Bs = sh + (size_t)p * kTsRows; // [q][kTsRows]
  const int pq = p * q;
  double acc[kTsMaxPQ / 256];
#pragma unroll
  for (int e = 0; e < kTsMaxPQ / 256; ++e) acc[e] = 0.0;
  for (int64_t r0 = (int64_t)blockIdx.x * kTsRows; r0 < n; r0 += (int64_t)gridDim.x * kTsRows) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < (p + q) * kTsRows; idx += blockDim.x) {
      const int c = idx / kTsRows, rr = idx % kTsRows;
      const int64_t row = r0 + rr;
      double v = 0.0;
      if (row < n) v = (c < p) ? A[(size_t)c * lda + row] : B[(size_t)(c - p) * ldb + row];
      sh[idx] = v;
    }
    __syncthreads();
#pragma unroll
    for (int e = 0; e < kTsMaxPQ / 256; ++e) {
      const int idx = threadIdx.x + e * 256;
      if (idx < pq) {
        const int i = idx % p, j = idx / p;
        const double* a = As + (size_t)i * kTsRows;
        const double* b = Bs + (size_t)j * kTsRows;
        double s = acc[e];
#pragma unroll 8
        for (int rr = 0; rr < kTsRows; ++rr) s += a[rr] * b[rr];
        acc[e] = s;
      }
    }
  }
#pragma unroll
  for (int e = 0; e < kTsMaxPQ / 256; ++e) {
    const int idx = threadIdx.x + e * 256;
    if (idx < pq) part[(size_t)blockIdx.x * pq + idx] = acc[e];
  }
}

// Partial C = A^T B, register-blocked, for p <= 64 and q <= QM: thread (mb, g) accumulates
// the 2 x q outputs of A columns 2 mb, 2 mb + 1 over the rows g, g + G, ... of every tile
// (G = 512 / ceil(p / 2) row groups).  Tiles of R rows (a multiple of 32 chosen so that three
// fill the shared memory) are staged row-major with an odd row stride (the column-wise fills
// and the row-wise reads are both free of bank conflicts) by asynchronous 8-byte copies,
// three deep: two tiles stream in while one is multiplied, which keeps enough bytes in
// flight per SM for HBM speed.  At the end the row groups' sums are added in group order.
// The reads of A and B are the only HBM traffic.
constexpr int kTsRbMaxP = 64;
constexpr int kTsRbStages = 3;
constexpr int kTsRbSmem = 200 * 1024;
constexpr int kTsRbThreads = 512;
constexpr int kTsRbMB = 2;          // A columns per thread

__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int QM>
__global__ void __launch_bounds__(kTsRbThreads, 1) k_tsgemm_rb(int64_t n, const double* __restrict__ A, int64_t lda,
                                                              int p, const double* __restrict__ B, int64_t ldb, int q,
                                                              int R, double* __restrict__ part) {
  extern __shared__ double sh[];
  const int npb = (p + kTsRbMB - 1) / kTsRbMB;
  const int G = kTsRbThreads / npb;
  const int pw = kTsRbMB * npb;
  const int stride = (pw + QM) | 1;                   // odd
  const int tile = R * stride;
  double* out = sh + kTsRbStages * tile;              // [pw][QM] group sums
  const int mb = threadIdx.x % npb, g = threadIdx.x / npb;
  const bool active = g < G;
  for (int i = threadIdx.x; i < kTsRbStages * tile + pw * QM; i += kTsRbThreads) sh[i] = 0.0;
  __syncthreads();
  double acc[kTsRbMB][QM];
#pragma unroll
  for (int k = 0; k < kTsRbMB; ++k)
#pragma unroll
    for (int j = 0; j < QM; ++j) acc[k][j] = 0.0;
  const int64_t step = (int64_t)gridDim.x * R;
  const int64_t first = (int64_t)blockIdx.x * R;
  // copies tile t (rows first + t step ...) into its stage; rows past n become zeros; an
  // empty group is committed past the end so that the group count stays uniform
  auto fill = [&](int64_t t) {
    const int64_t r0 = first + t * step;
    if (r0 < n) {
      double* tb = sh + (t % kTsRbStages) * tile;
      const int cols = p + q;
      for (int idx = threadIdx.x; idx < cols * R; idx += kTsRbThreads) {
        const int c = idx / R, rr = idx - c * R;
        const int64_t row = r0 + rr;
        double* dst = tb + rr * stride + (c < p ? c : pw + (c - p));
        if (row < n) cp_async8(dst, c < p ? A + (size_t)c * lda + row : B + (size_t)(c - p) * ldb + row);
        else *dst = 0.0;   // this stage is not being read: the round that read it ended with a barrier
      }
    }
    cp_async_commit();
  };
  fill(0);
  fill(1);
  for (int64_t t = 0; first + t * step < n; ++t) {
    cp_async_wait<1>();   // tile t has landed (only tile t + 1 may still be in flight)
    __syncthreads();
    const double* tb = sh + (t % kTsRbStages) * tile;
    if (active) {
      for (int rr = g; rr < R; rr += G) {
        const double* rowp = tb + rr * stride;
        double a[kTsRbMB], b[QM];
#pragma unroll
        for (int k = 0; k < kTsRbMB; ++k) a[k] = rowp[kTsRbMB * mb + k];
#pragma unroll
        for (int j = 0; j < QM; ++j) b[j] = rowp[pw + j];
#pragma unroll
        for (int k = 0; k < kTsRbMB; ++k)
#pragma unroll
          for (int j = 0; j < QM; ++j) acc[k][j] += a[k] * b[j];
      }
    }
    __syncthreads();      // stage t % 3 is refilled two rounds later
    fill(t + 2);
  }
  cp_async_wait<0>();
  // row groups' sums, added in group order
  for (int gg = 0; gg < G; ++gg) {
    if (active && g == gg) {
#pragma unroll
      for (int k = 0; k < kTsRbMB; ++k)
#pragma unroll
        for (int j = 0; j < QM; ++j) out[(kTsRbMB * mb + k) * QM + j] += acc[k][j];
    }
    __syncthreads();
  }
  const int pq = p * q;
  for (int idx = threadIdx.x; idx < pq; idx += kTsRbThreads) {
    const int i = idx % p, j = idx / p;
    part[(size_t)blockIdx.x * pq + idx] = out[i * QM + j];
  }
}

// out[idx] = sum over blocks b (in order) of part[b*pq + idx]
__global__ void k_sum_parts(const double* __restrict__ part, int nblk, int pq, double* __restrict__ out) {
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < pq; idx += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)b * pq + idx];
    out[idx] = s;
  }
}

// V(:, c) = V(:, c) - sum_j Q(:, j) R(j, c) for c < q, j < p (CAGMRES_GEMM order).
// V(:, 0..q-1) -= Q(:, 0..p-1) R (R p x q, ld p), one thread per row; QM >= q is a
// compile-time bound, so the row's q values stay in registers.
template <int QM>
__global__ void __launch_bounds__(256) k_block_update(int64_t n, double* __restrict__ V, int64_t ldv, int q,
                                                      const double* __restrict__ Q, int64_t ldq, int p,
                                                      const double* __restrict__ R) {
  extern __shared__ double Rs[];
  for (int i = threadIdx.x; i < p * q; i += blockDim.x) Rs[i] = R[i];
  __syncthreads();
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
    double acc[QM];
#pragma unroll
    for (int c = 0; c < QM; ++c) acc[c] = c < q ? V[(size_t)c * ldv + row] : 0.0;
    for (int j = 0; j < p; ++j) {
      const double qv = Q[(size_t)j * ldq + row];
#pragma unroll
      for (int c = 0; c < QM; ++c)
        if (c < q) acc[c] = acc[c] - qv * Rs[c * p + j];
    }
#pragma unroll
    for (int c = 0; c < QM; ++c)
      if (c < q) V[(size_t)c * ldv + row] = acc[c];
  }
}

// Q(:, k) = sum_{j <= k} V(:, j) Ri(j, k), one thread per row, the row in registers.
template <int CM>
__global__ void __launch_bounds__(256) k_apply_rinv(int64_t n, const double* __restrict__ V, int64_t ldv, int c,
                                                    const double* __restrict__ Ri, double* __restrict__ Q,
                                                    int64_t ldq) {
  __shared__ double Rs[16 * 16];
  for (int i = threadIdx.x; i < c * c; i += blockDim.x) Rs[i] = Ri[i];
  __syncthreads();
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
    double v[CM];
#pragma unroll
    for (int j = 0; j < CM; ++j) v[j] = j < c ? V[(size_t)j * ldv + row] : 0.0;
#pragma unroll
    for (int k = 0; k < CM; ++k) {
      if (k >= c) break;
      double s = 0.0;
#pragma unroll
      for (int j = 0; j <= k; ++j) s += v[j] * Rs[k * c + j];
      Q[(size_t)k * ldq + row] = s;
    }
  }
}

// v0 = sum_{i<m} y_i Q(:, i) (sum_vec_FP64_CPU order: start at 0, add y_i Q_i).
__global__ void k_sum_cols(int64_t n, double* __restrict__ v0, const double* __restrict__ Q, int64_t ldq,
                           int m, const double* __restrict__ y) {
  extern __shared__ double ys[];
  for (int i = threadIdx.x; i < m; i += blockDim.x) ys[i] = y[i];
  __syncthreads();
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < n; row += (int64_t)gridDim.x * blockDim.x) {
    double t = 0.0;
    for (int i = 0; i < m; ++i) t = t + ys[i] * Q[(size_t)i * ldq + row];
    v0[row] = t;
  }
}

// Structured Householder TSQR, R only: each warp folds its rows, 32 at a time, into an
// upper triangular c x c factor (lane k holds row k of R), reflecting the stacked
// [R; X] with reflectors that only touch R's diagonal entry and the 32 new rows.
// Writes the warp's R as rows [w*c, w*c+c) of Rout (column-major, leading dim ldo).
template <int CM>
__global__ void __launch_bounds__(256) k_tsqr_local(int64_t nrows, int c, const double* __restrict__ A,
                                                    int64_t lda, int64_t rows_per_warp,
                                                    double* __restrict__ Rout, int64_t ldo) {
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t r0 = w * rows_per_warp;
  // The grid is rounded up to whole blocks: warps past the last row own no R factor and
  // must not write one (Rout holds exactly ceil(nrows / rows_per_warp) factors).
  if (r0 >= nrows) return;
  const int64_t r1 = min(nrows, r0 + rows_per_warp);
  double R[CM];
#pragma unroll
  for (int j = 0; j < CM; ++j) R[j] = 0.0;
  for (int64_t base = r0; base < r1; base += 32) {
    const int64_t row = base + lane;
    double X[CM];
#pragma unroll
    for (int j = 0; j < CM; ++j) X[j] = (j < c && row < r1) ? A[(size_t)j * lda + row] : 0.0;
#pragma unroll
    for (int k = 0; k < CM; ++k) {
      if (k >= c) break;
      double sig = X[k] * X[k];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sig += __shfl_xor_sync(kFull, sig, o);
      const double alpha = __shfl_sync(kFull, R[k], k);
      if (sig == 0.0) continue;
      const double nrm = sqrt(alpha * alpha + sig);
      const double beta = alpha >= 0.0 ? -nrm : nrm;
      const double v0 = alpha - beta;
      const double tau = (beta - alpha) / beta;
      const double u = X[k] / v0;                  // this lane's part of u (u0 = 1)
#pragma unroll
      for (int j = 0; j < CM; ++j) {
        if (j <= k || j >= c) continue;
        double s = u * X[j];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        const double wj = __shfl_sync(kFull, R[j], k) + s;
        if (lane == k) R[j] -= tau * wj;
        X[j] -= tau * wj * u;
      }
      if (lane == k) R[k] = beta;
      X[k] = 0.0;
    }
  }
  if (lane < c) {
#pragma unroll
    for (int j = 0; j < CM; ++j)
      if (j < c) Rout[(size_t)j * ldo + w * c + lane] = R[j];
  }
}

// ------------------------------------------------------------------ host helpers
namespace {

struct Dev {
  DBuf part, out, small, tmp;
  int parts_blocks = 0;
};

int tsgemm_blocks() { return 2 * num_sms(); }

// C (p x q) = A^T B on the host, A/B device panels of n rows.
Mat tsgemm(Dev& D, int64_t n, const double* A, int64_t lda, int p, const double* B, int64_t ldb, int q) {
  PB_CHECK(p * q <= kTsMaxPQ, PARCEL_B_E_UNSUPPORTED, "block product %dx%d too large", p, q);
  int nb = tsgemm_blocks();
  cudaStream_t st = stream();
  if (p <= kTsRbMaxP && q <= 16) {
    const int pw = kTsRbMB * ((p + kTsRbMB - 1) / kTsRbMB);
    auto launch = [&](auto kern, int QM) {
      const int stride = (pw + QM) | 1;
      int R = (int)((kTsRbSmem - sizeof(double) * pw * QM) / (sizeof(double) * kTsRbStages * stride));
      R = std::max(32, std::min(512, R / 32 * 32));
      const size_t smem = sizeof(double) * ((size_t)kTsRbStages * R * stride + (size_t)pw * QM);
      static bool attr[17] = {};
      if (!attr[QM]) {
        PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, kTsRbSmem));
        attr[QM] = true;
      }
      kern<<<num_sms(), kTsRbThreads, smem, st>>>(n, A, lda, p, B, ldb, q, R, dp<double>(D.part));
      return num_sms();
    };
    int used;
    if (q <= 4) used = launch(k_tsgemm_rb<4>, 4);
    else if (q <= 8) used = launch(k_tsgemm_rb<8>, 8);
    else if (q <= 9) used = launch(k_tsgemm_rb<9>, 9);
    else if (q <= 12) used = launch(k_tsgemm_rb<12>, 12);
    else used = launch(k_tsgemm_rb<16>, 16);
    nb = used;
  } else {
    const size_t smem = sizeof(double) * (size_t)(p + q) * kTsRows;
    k_tsgemm_atb<<<nb, 256, smem, st>>>(n, A, lda, p, B, ldb, q, dp<double>(D.part));
  }
  PB_CUDA(cudaGetLastError());
  k_sum_parts<<<(p * q + 127) / 128, 128, 0, st>>>(dp<double>(D.part), nb, p * q, dp<double>(D.out));
  PB_CUDA(cudaGetLastError());
  Mat C(p, q);
  d2h(C.a.data(), D.out.p, sizeof(double) * p * q);
  return C;
}

// R-only TSQR of an n x c device panel (c <= 16); rows of R normalised to a positive
// diagonal as TSQR_Ronly_ does (src/QRDecomposition.f90:887-1002).
Mat tsqr_r(Dev& D, int64_t n, const double* A, int64_t lda, int c) {
  cudaStream_t st = stream();
  const double* cur = A;
  int64_t curld = lda, rows = n;
  DBuf bufs[2];
  int which = 0;
  while (true) {
    const int64_t warps_max = (int64_t)num_sms() * 16;
    int64_t rpw = std::max<int64_t>(512, (rows + warps_max - 1) / warps_max);
    rpw = (rpw + 31) / 32 * 32;
    const int64_t nw = (rows + rpw - 1) / rpw;
    const int64_t ldo = nw * c;
    bufs[which].alloc(sizeof(double) * (size_t)ldo * c);
    const int threads = 256;
    const int64_t blocks = (nw * 32 + threads - 1) / threads;
    if (c <= 8)
      k_tsqr_local<8><<<(unsigned)blocks, threads, 0, st>>>(rows, c, cur, curld, rpw, dp<double>(bufs[which]), ldo);
    else
      k_tsqr_local<16><<<(unsigned)blocks, threads, 0, st>>>(rows, c, cur, curld, rpw, dp<double>(bufs[which]), ldo);
    PB_CUDA(cudaGetLastError());
    cur = dp<double>(bufs[which]);
    curld = ldo;
    rows = ldo;
    which ^= 1;
    if (nw == 1) break;
  }
  Mat R(c, c);
  std::vector<double> h((size_t)c * c);
  for (int j = 0; j < c; ++j) d2h(&R.a[(size_t)j * c], cur + (size_t)j * curld, sizeof(double) * c);
  for (int i = 0; i < c; ++i)
    for (int j = 0; j < i; ++j) R(i, j) = 0.0;
  for (int i = 0; i < c; ++i)
    if (R(i, i) < 0.0)
      for (int j = i; j < c; ++j) R(i, j) = -R(i, j);
  return R;
}

void apply_rinv(Dev& D, int64_t n, const double* V, int64_t ldv, const Mat& Ri, double* Q, int64_t ldq) {
  const int c = Ri.n;
  D.small.alloc(sizeof(double) * c * c);
  h2d(D.small.p, Ri.a.data(), sizeof(double) * c * c);
  const int grid = std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 8 * num_sms()));
  if (c <= 8) k_apply_rinv<8><<<grid, 256, 0, stream()>>>(n, V, ldv, c, dp<double>(D.small), Q, ldq);
  else k_apply_rinv<16><<<grid, 256, 0, stream()>>>(n, V, ldv, c, dp<double>(D.small), Q, ldq);
  PB_CUDA(cudaGetLastError());
}

// R-only QR of the device panel (c columns): TSQR, Cholesky QR or Cholesky QR2
// (QRDecomposition_, src/QRDecomposition.f90:1331-1552).  MGS / CGS flags use TSQR.
Mat qr_r_only(Dev& D, int64_t n, const double* V, int64_t ldv, int c, int flag) {
  if (flag == PARCEL_B_QR_CHOLQR || flag == PARCEL_B_QR_CHOLQR2) {
    Mat G = tsgemm(D, n, V, ldv, c, V, ldv, c);
    Mat R1;
    if (dense::chol_upper(G, R1)) {
      if (flag == PARCEL_B_QR_CHOLQR) return R1;
      D.tmp.alloc(sizeof(double) * (size_t)ldv * c);
      apply_rinv(D, n, V, ldv, dense::trinv_upper(R1), dp<double>(D.tmp), ldv);
      Mat G2 = tsgemm(D, n, dp<double>(D.tmp), ldv, c, dp<double>(D.tmp), ldv, c);
      Mat R2;
      if (dense::chol_upper(G2, R2)) return dense::gemm(R2, R1);
    }
    // Gram matrix not numerically positive definite: fall back to TSQR
  }
  return tsqr_r(D, n, V, ldv, c);
}

void newton_basis(int s, Mat& B1, const std::vector<double>& er, const std::vector<double>& ei) {
  int i = 1;
  while (i <= s) {
    if (i == s) {
      B1(i - 1, i - 1) = er[i - 1];
    } else if (std::fabs(ei[i - 1]) == 0.0) {
      B1(i - 1, i - 1) = er[i - 1];
    } else {
      B1(i - 1, i - 1) = er[i - 1];
      B1(i, i) = er[i - 1];
      B1(i - 1, i) = -ei[i - 1] * ei[i - 1];
      ++i;
    }
    ++i;
  }
}

// modified_leja_ordering (src/LejaOrdering.f90:100-322), in place on er/ei[0..n).
void leja(int n, std::vector<double>& er, std::vector<double>& ei) {
  for (int i = 1; i < n; ++i) {
    int j = i;
    while (j > 0 && std::sqrt(er[j - 1] * er[j - 1] + ei[j - 1] * ei[j - 1]) <
                        std::sqrt(er[j] * er[j] + ei[j] * ei[j])) {
      std::swap(er[j], er[j - 1]);
      std::swap(ei[j], ei[j - 1]);
      --j;
    }
  }
  std::vector<double> ptmp(n, 1.0), mu(n, 1.0), tr(n, 0.0), ti(n, 0.0), tmp(n, 0.0);
  std::vector<int> out(n, 0);
  double C = 1.0;
  int L;
  if (ei[0] > 0.0) {
    tr[0] = er[0]; ti[0] = ei[0]; tr[1] = er[1]; ti[1] = ei[1];
    out[0] = 0; out[1] = 1;
    L = 2;
  } else {
    tr[0] = er[0]; ti[0] = 0.0; out[0] = 0;
    L = 1;
  }
  while (L < n) {
    const double Cold = C;
    for (int j = 0; j <= L - 2; ++j) {
      const double a = tr[L - 1] - tr[j], b = ti[L - 1] - ti[j];
      ptmp[j + 1] = std::pow(std::sqrt(a * a + b * b), mu[out[j]] / L);
    }
    C = 1.0;
    for (int j = 0; j < n; ++j) C = C * ptmp[j];
    const double f = C / Cold;
    for (int j = 0; j < n; ++j) { er[j] /= f; ei[j] /= f; tr[j] /= f; ti[j] /= f; }
    for (int j = 0; j < n; ++j) tmp[j] = 0.0;
    for (int j = 0; j < n; ++j) {
      bool in = false;
      for (int i = 0; i < L; ++i) if (out[i] == j) in = true;
      if (in) continue;
      double prod = 1.0;
      for (int q = 0; q <= L - 2; ++q) {
        const double a = er[j] - tr[q], b = ei[j] - ti[q];
        prod = prod * std::pow(std::sqrt(a * a + b * b), mu[out[q]]);
      }
      tmp[j] = prod;
    }
    double mx = std::fabs(tmp[0]);
    int k = 0;
    for (int j = 1; j < n; ++j)
      if (std::fabs(tmp[j]) > mx) { mx = std::fabs(tmp[j]); k = j; }
    if (std::fabs(ei[k]) > 0.0) {
      const int a = ei[k] < 0.0 ? k - 1 : k;
      tr[L] = er[a]; ti[L] = ei[a]; tr[L + 1] = er[a + 1]; ti[L + 1] = ei[a + 1];
      out[L] = a; out[L + 1] = a + 1;
      L += 2;
    } else {
      tr[L] = er[k]; ti[L] = 0.0; out[L] = k;
      L += 1;
    }
  }
  for (int i = 0; i < n; ++i) { er[i] = tr[i] * C; ei[i] = ti[i] * C; }
}

void givens_h(Mat& Hg, int i, std::vector<double>& co, std::vector<double>& si, std::vector<double>& ze) {
  for (int k = 1; k <= i - 1; ++k) {
    const double t1 = Hg(k - 1, i - 1) * co[k - 1] - Hg(k, i - 1) * si[k - 1];
    const double t2 = Hg(k - 1, i - 1) * si[k - 1] + Hg(k, i - 1) * co[k - 1];
    Hg(k - 1, i - 1) = t1;
    Hg(k, i - 1) = t2;
  }
  const double t = (Hg(i - 1, i - 1) == 0.0) ? Hg(i, i - 1) / 1.0 - 300.0 : Hg(i, i - 1) / Hg(i - 1, i - 1);
  co[i - 1] = 1.0 / std::sqrt(1.0 + t * t);
  si[i - 1] = -co[i - 1] * t;
  const double t1 = co[i - 1] * ze[i - 1] - si[i - 1] * ze[i];
  const double t2 = si[i - 1] * ze[i - 1] + co[i - 1] * ze[i];
  ze[i - 1] = t1;
  ze[i] = t2;
  Hg(i - 1, i - 1) = co[i - 1] * Hg(i - 1, i - 1) - si[i - 1] * Hg(i, i - 1);
  Hg(i, i - 1) = 0.0;
}

Mat sub(const Mat& A, int i0, int j0, int m, int n) {
  Mat B(m, n);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) B(i, j) = A(i0 + i, j0 + j);
  return B;
}

// calc_HessenbergMatrix (src/pcagmres.f90:879-1052); returns the new hk_pre.
double hessenberg_update(int s, int k, const Mat& B1, Mat& H, const Mat& R1, const Mat& Rk,
                         const Mat& BRup, double hk_pre) {
  if (k == 1) {
    Mat Rinv = dense::trinv_upper(sub(R1, 0, 0, s, s));
    Mat Hes = dense::gemm(dense::gemm(R1, B1), Rinv);
    for (int j = 0; j < s; ++j)
      for (int i = 0; i <= s; ++i) H(i, j) = Hes(i, j);
    return Hes(s, s - 1);
  }
  const int s1 = s * (k - 1);
  Mat Rt0(s + 1, s + 1);
  for (int i = 0; i <= s; ++i) Rt0(0, i) = BRup(s1, i);
  for (int j = 0; j < s; ++j)
    for (int i = 0; i < s; ++i) Rt0(1 + i, 1 + j) = Rk(i, j);
  Mat BRu = sub(BRup, 0, 0, s1, s + 1);
  Mat BR = sub(BRup, 0, 0, s1, s);
  Mat Rinv = dense::trinv_upper(sub(Rt0, 0, 0, s, s));
  Mat BlockHes = sub(H, 0, 0, s1, s1);
  Mat X1 = dense::gemm(BlockHes, BR);
  Mat X2 = dense::gemm(BRu, B1);
  for (size_t i = 0; i < X1.a.size(); ++i) X1.a[i] = -X1.a[i] + X2.a[i];
  Mat X3 = dense::gemm(X1, Rinv);
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s1; ++j) H(j, s1 + i) = X3(j, i);
  const double bk = B1(s, s - 1);
  const double rho_tilde = Rt0(s - 1, s - 1);
  const double rho = Rt0(s, s);
  const double hk = rho / rho_tilde * bk;
  H(s * k, s * k - 1) = hk;
  Mat Hss = dense::gemm(dense::gemm(sub(Rt0, 0, 0, s, s), sub(B1, 0, 0, s, s)), Rinv);
  for (int i = 0; i < s; ++i) Hss(i, s - 1) = Hss(i, s - 1) + bk / rho_tilde * Rt0(i, s);
  Mat e1(s, s);
  for (int i = 0; i < s; ++i) e1(0, i) = BR(s1 - 1, i) * hk_pre;
  Mat H0 = dense::gemm(e1, Rinv);
  for (size_t i = 0; i < Hss.a.size(); ++i) Hss.a[i] = Hss.a[i] - H0.a[i];
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < s; ++j) H(s1 + j, s1 + i) = Hss(j, i);
  return hk;
}

}  // namespace

SolveOut solve_cagmres(const Options& o, System<double>& S, const double* b_nat, double* x_nat,
                       std::vector<double>& hist, double* setup_t) {
  cudaStream_t st = stream();
  const int s = o.sstep, t = o.tstep, stt = s * t;
  PB_CHECK(s >= 1 && s <= 15 && stt <= 64, PARCEL_B_E_UNSUPPORTED,
           "CA-GMRES needs 1 <= s <= 15 and s*t <= 64 (got s=%d, t=%d)", s, t);
  const int64_t np = S.np;
  const int64_t ldv = (np + 31) & ~int64_t(31);
  DBuf bb, xb;
  const double* b = b_nat;
  double* x = x_nat;
  if (S.permuted) {
    bb.alloc(sizeof(double) * np);
    xb.alloc(sizeof(double) * np);
    PB_CUDA(cudaMemsetAsync(bb.p, 0, sizeof(double) * np, st));
    PB_CUDA(cudaMemsetAsync(xb.p, 0, sizeof(double) * np, st));
    scatter_perm<double>(S.n, dp<double>(bb), b_nat, dp<int>(S.pos), st);
    scatter_perm<double>(S.n, dp<double>(xb), x_nat, dp<int>(S.pos), st);
    b = dp<double>(bb);
    x = dp<double>(xb);
  }
  DBuf Vb(sizeof(double) * ldv * (s + 1)), Qb(sizeof(double) * ldv * (stt + 1)), rb(sizeof(double) * np),
      pvb(sizeof(double) * np), v0b(sizeof(double) * np), x0b(sizeof(double) * np), yb(sizeof(double) * (stt + 1));
  PB_CUDA(cudaMemsetAsync(Vb.p, 0, Vb.bytes, st));
  PB_CUDA(cudaMemsetAsync(Qb.p, 0, Qb.bytes, st));
  double* V = dp<double>(Vb);
  double* Q = dp<double>(Qb);
  double* r = dp<double>(rb);
  Dev D;
  D.part.alloc(sizeof(double) * (size_t)tsgemm_blocks() * kTsMaxPQ);
  D.out.alloc(sizeof(double) * kTsMaxPQ);
  sync();
  if (setup_t) *setup_t = now_s();

  auto col = [&](double* base, int j) { return base + (size_t)j * ldv; };
  auto dot = [&](const double* a, const double* c) { return dev_dot<double>(np, a, c); };
  int launches = 0;

  Mat B1(s + 1, s);
  for (int i = 0; i < s; ++i) B1(i + 1, i) = 1.0;
  std::vector<double> er(stt, 0.0), ei(stt, 0.0);
  const double bnorm = std::sqrt(dot(b, b));
  hist.assign(o.itrmax + stt + 2, 0.0);
  int iflag_exit = -1, iflag_basis = -1;
  int itr = 1, itr0 = 0;
  for (itr = 1; itr <= o.itrmax; itr += stt) {
    itr0 = itr;
    std::vector<double> co(stt + 1, 0.0), si(stt + 1, 0.0), ze(stt + 1, 0.0);
    Mat H(stt + 1, stt), Hg(stt + 1, stt), R1, Rk, BRup;
    double hk_pre = 0.0;
    spmv<double, double>(S.A, x, r, SPMV_RES, b, nullptr, st);
    const double rnorm0 = std::sqrt(dot(r, r));
    launches += 2;
    if (rnorm0 < o.abstol || rnorm0 / bnorm < o.rtol) break;
    if (rnorm0 != rnorm0) { SolveOut so; so.niter = itr; so.iret = PARCEL_B_E_BREAKDOWN; return so; }
    if (itr == 1) hist[0] = rnorm0 / bnorm;
    ze[0] = -rnorm0;
    lincomb<double>(np, V, r, cimm(-1.0 / rnorm0), nullptr, cimm(0), nullptr, cimm(0), nullptr, st);
    int mm = 0;
    for (int k = 1; k <= t; ++k) {
      if (o.basis == PARCEL_B_BASIS_NEWTON && iflag_basis == 1) newton_basis(s, B1, er, ei);
      for (int i = 1; i <= s; ++i) {
        S.M.apply(np, col(V, i - 1), dp<double>(pvb), nullptr, st);
        spmv<double, double>(S.A, dp<double>(pvb), col(V, i), SPMV_Y, nullptr, nullptr, st);
        launches += 2;
        if (iflag_basis == 1 && o.basis == PARCEL_B_BASIS_NEWTON) {
          const double alpha = -B1(i - 1, i - 1);
          if (i != 1) {
            const double beta = -B1(i - 2, i - 1);
            lincomb<double>(np, col(V, i), col(V, i - 1), cimm(alpha), col(V, i - 2), cimm(beta), col(V, i),
                            cimm(1.0), nullptr, st);
          } else {
            lincomb<double>(np, col(V, i), col(V, i - 1), cimm(alpha), col(V, i), cimm(1.0), nullptr, cimm(0),
                            nullptr, st);
          }
          ++launches;
        }
      }
      if (k == 1) {
        R1 = qr_r_only(D, np, V, ldv, s + 1, o.qrflag);
        apply_rinv(D, np, V, ldv, dense::trinv_upper(R1), Q, ldv);
      } else {
        const int s1 = s * (k - 1) + 1;
        BRup = tsgemm(D, np, Q, ldv, s1, V, ldv, s + 1);
        // V(:, 1..s) -= Q(:, 0..s1-1) BRup(:, 1..s)
        Mat Rsub = sub(BRup, 0, 1, s1, s);
        D.small.alloc(sizeof(double) * s1 * s);
        h2d(D.small.p, Rsub.a.data(), sizeof(double) * s1 * s);
        const int grid = std::max<int64_t>(1, std::min<int64_t>((np + 255) / 256, 8 * num_sms()));
        if (s <= 8)
          k_block_update<8><<<grid, 256, sizeof(double) * s1 * s, st>>>(np, col(V, 1), ldv, s, Q, ldv, s1,
                                                                        dp<double>(D.small));
        else
          k_block_update<16><<<grid, 256, sizeof(double) * s1 * s, st>>>(np, col(V, 1), ldv, s, Q, ldv, s1,
                                                                         dp<double>(D.small));
        PB_CUDA(cudaGetLastError());
        Rk = qr_r_only(D, np, col(V, 1), ldv, s, o.qrflag);
        apply_rinv(D, np, col(V, 1), ldv, dense::trinv_upper(Rk), col(Q, s1), ldv);
        launches += 4;
      }
      hk_pre = hessenberg_update(s, k, B1, H, R1, Rk, BRup, hk_pre);
      if (k != t) {
        d2d(V, col(Q, s * k), sizeof(double) * np);
      }
      for (int i = s * (k - 1); i < s * k; ++i)
        for (int j = 0; j <= stt; ++j) Hg(j, i) = H(j, i);
      for (int i = s * (k - 1) + 1; i <= s * k; ++i) {
        mm = i;
        givens_h(Hg, i, co, si, ze);
        const double rn = std::fabs(ze[i]);
        itr0 = i + (itr - 1) + 1;
        hist[itr0 - 1] = rn / bnorm;
        if (rn / bnorm < o.rtol || i + (itr - 1) + 1 == o.itrmax) { iflag_exit = 1; break; }
      }
      if (iflag_exit == 1) break;
      if (o.basis == PARCEL_B_BASIS_NEWTON) {
        iflag_basis = 1;
        std::vector<double> wr, wi;
        dense::hessenberg_eigs(sub(H, 0, 0, s * k, s * k), wr, wi);
        leja(s * k, wr, wi);
        for (int i = 0; i < s * k; ++i) { er[i] = wr[i]; ei[i] = wi[i]; }
      }
    }
    // update: y = Hg^-1 ze over mm columns; x += M^-1 (Q y)
    std::vector<double> y(std::max(mm, 1), 0.0);
    for (int i = mm; i >= 1; --i) {
      double v = ze[i - 1];
      for (int j = mm; j >= i + 1; --j) v = v - Hg(i - 1, j - 1) * y[j - 1];
      const double d = Hg(i - 1, i - 1);
      y[i - 1] = (d == 0.0) ? v / 1.0e-300 : v / d;
    }
    h2d(yb.p, y.data(), sizeof(double) * mm);
    const int grid = std::max<int64_t>(1, std::min<int64_t>((np + 255) / 256, 8 * num_sms()));
    k_sum_cols<<<grid, 256, sizeof(double) * std::max(mm, 1), st>>>(np, dp<double>(v0b), Q, ldv, mm, dp<double>(yb));
    PB_CUDA(cudaGetLastError());
    S.M.apply(np, dp<double>(v0b), dp<double>(x0b), nullptr, st);
    lincomb<double>(np, x, dp<double>(x0b), cimm(1.0), x, cimm(1.0), nullptr, cimm(0), nullptr, st);
    launches += 3;
    if (iflag_exit == 1) break;
  }
  if (S.permuted) gather_perm<double>(S.n, x_nat, x, dp<int>(S.pos), st);
  sync();
  SolveOut so;
  so.niter = std::min(o.itrmax, itr0);
  so.iret = (o.itrmax <= itr) ? 1 : 0;
  so.launches = launches;
  hist.resize(std::max(so.niter, 0));
  return so;
}

}  // namespace pb
