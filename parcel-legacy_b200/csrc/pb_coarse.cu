// pb_coarse.cu -- Galerkin coarse-grid operator, grid transfers and the one-cluster coarse
// Jacobi-PCG of the two-level preconditioner stage (no counterpart in the reference).
//
// Kernels:
//   k_galerkin       one CTA per coarse cell: A_c(I, I + d) = sum_f sum_g P(f, I) A(f, g) P(g, I + d)
//                    over the fine cells f whose interpolation involves I; every thread keeps
//                    private sums for the 27 taps in shared memory and the 27 tap owners add
//                    the threads' sums in thread order (deterministic).
//   k_restrict_half  one warp per half cell ((c/2)^3 fine cells that share their two coarse
//                    parents along every axis): the 8 weighted sums of the half cell.
//   k_restrict_sum   one thread per coarse cell: adds the half-cell sums that belong to it,
//                    in a fixed order.
//   k_prolong_add    one thread per iteration-layout position: z += trilinear(y).
//   k_coarse_pcg     one thread-block cluster (8 CTAs x 1024 threads), see pcg().
#include <cooperative_groups.h>

#include "pb_coarse.cuh"
#include "pb_device.cuh"

namespace cg = cooperative_groups;

namespace pb {
namespace coarse {
namespace {

constexpr int kGalThreads = 128;
constexpr int kPcgThreads = 1024;
constexpr int kPcgCluster = 8;
constexpr int kPcgMaxCpt = 8;       // coarse cells per thread
constexpr int kRmsThreads = 1024;

// Interpolation along one axis: fine index i -> coarse parents lo, hi (clamped) and the
// weight w of hi (1 - w of lo).  u = (2 i + 1 - c) / (2 c) exactly.
__host__ __device__ __forceinline__ void lin1(int i, int c, int G, int& lo, int& hi, double& w) {
  const int num = 2 * i + 1 - c, den = 2 * c;
  const int i0 = num >= 0 ? num / den : -((-num + den - 1) / den);
  w = (double)(num - den * i0) / (double)den;
  lo = min(max(i0, 0), G - 1);
  hi = min(max(i0 + 1, 0), G - 1);
}

// Weight of coarse index I in fine index i's interpolation along one axis.
__device__ __forceinline__ double wof(int i, int c, int G, int I) {
  int lo, hi;
  double w;
  lin1(i, c, G, lo, hi, w);
  return (lo == I ? 1.0 - w : 0.0) + (hi == I ? w : 0.0);
}

__global__ void __launch_bounds__(kGalThreads)
    k_galerkin(Grid g, const int* __restrict__ rowptr, const int* __restrict__ col, const double* __restrict__ val,
               int rbase, int cbase, double* __restrict__ ac) {
  __shared__ double acc[kTaps * kGalThreads];
  const int t = threadIdx.x;
  const int64_t I = blockIdx.x;
  const int Ix = (int)(I % g.gx), Iy = (int)((I / g.gx) % g.gy), Iz = (int)(I / ((int64_t)g.gx * g.gy));
#pragma unroll
  for (int s = 0; s < kTaps; ++s) acc[s * kGalThreads + t] = 0.0;
  const int h = g.c / 2;
  const int x0 = max(0, g.c * Ix - h), x1 = min(g.nx - 1, g.c * Ix + g.c + h - 1);
  const int y0 = max(0, g.c * Iy - h), y1 = min(g.ny - 1, g.c * Iy + g.c + h - 1);
  const int z0 = max(0, g.c * Iz - h), z1 = min(g.nz - 1, g.c * Iz + g.c + h - 1);
  const int sx = x1 - x0 + 1, sy = y1 - y0 + 1, sz = z1 - z0 + 1;
  const int tot = sx * sy * sz;
  const int64_t nxy = (int64_t)g.nx * g.ny;
  for (int e = t; e < tot; e += kGalThreads) {
    const int fx = x0 + e % sx, fy = y0 + (e / sx) % sy, fz = z0 + e / (sx * sy);
    const double wI = wof(fx, g.c, g.gx, Ix) * wof(fy, g.c, g.gy, Iy) * wof(fz, g.c, g.gz, Iz);
    if (wI == 0.0) continue;
    const int64_t f = (int64_t)fz * nxy + (int64_t)fy * g.nx + fx;
    const int kb = rowptr[f] - rbase, ke = rowptr[f + 1] - rbase;
    for (int k = kb; k < ke; ++k) {
      const int64_t gc = (int64_t)col[k] - cbase;
      const double a = val[k] * wI;
      const int gx_ = (int)(gc % g.nx), gy_ = (int)((gc / g.nx) % g.ny), gz_ = (int)(gc / nxy);
      int lx, hx, ly, hy, lz, hz;
      double wx, wy, wz;
      lin1(gx_, g.c, g.gx, lx, hx, wx);
      lin1(gy_, g.c, g.gy, ly, hy, wy);
      lin1(gz_, g.c, g.gz, lz, hz, wz);
#pragma unroll
      for (int cz = 0; cz < 2; ++cz) {
        const int dz = (cz ? hz : lz) - Iz;
        const double fz_ = cz ? wz : 1.0 - wz;
        if (dz < -1 || dz > 1 || fz_ == 0.0) continue;
#pragma unroll
        for (int cy = 0; cy < 2; ++cy) {
          const int dy = (cy ? hy : ly) - Iy;
          const double fy_ = cy ? wy : 1.0 - wy;
          if (dy < -1 || dy > 1 || fy_ == 0.0) continue;
#pragma unroll
          for (int cx = 0; cx < 2; ++cx) {
            const int dx = (cx ? hx : lx) - Ix;
            const double fx_ = cx ? wx : 1.0 - wx;
            if (dx < -1 || dx > 1 || fx_ == 0.0) continue;
            acc[(9 * (dz + 1) + 3 * (dy + 1) + (dx + 1)) * kGalThreads + t] += a * fz_ * fy_ * fx_;
          }
        }
      }
    }
  }
  __syncthreads();
  if (t < kTaps) {
    double s = 0.0;
    for (int k = 0; k < kGalThreads; ++k) s += acc[t * kGalThreads + k];
    ac[(int64_t)t * g.Vc() + I] = s;
  }
}

__global__ void k_to_f32(int64_t Vc, const double* __restrict__ ac64, float* __restrict__ ac32,
                         float* __restrict__ dinv32) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Vc) return;
#pragma unroll
  for (int t = 0; t < kTaps; ++t) ac32[t * Vc + i] = (float)ac64[t * Vc + i];
  const double d = ac64[13 * Vc + i];
  dinv32[i] = d != 0.0 ? (float)(1.0 / d) : 0.f;
}

// Half cell H = (hx, hy, hz) covers fine cells [hx c/2, (hx + 1) c/2) along x (and so on);
// all of them interpolate from the same two coarse cells per axis.  hc[8 H + 4 cz + 2 cy + cx]
// = sum over the half cell of v * wz_cz * wy_cy * wx_cx (w_0 = 1 - w, w_1 = w).
template <class T>
__global__ void __launch_bounds__(256)
    k_restrict_half(Grid g, const T* __restrict__ v, const int* __restrict__ pos, float* __restrict__ hc,
                    const int* gate) {
  if (gated(gate)) return;
  const int lane = threadIdx.x & 31;
  const int64_t w = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= g.Vh()) return;
  const int hn = 2 * g.gx, hm = 2 * g.gy;
  const int hx = (int)(w % hn), hy = (int)((w / hn) % hm), hz = (int)(w / ((int64_t)hn * hm));
  const int hs = g.c / 2, n3 = hs * hs * hs;
  double m[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) m[k] = 0.0;
  for (int e = lane; e < n3; e += 32) {
    const int x = hx * hs + e % hs, y = hy * hs + (e / hs) % hs, z = hz * hs + e / (hs * hs);
    const int64_t nat = ((int64_t)z * g.ny + y) * g.nx + x;
    const double val = (double)v[pos ? pos[nat] : nat];
    int l, u;
    double wx, wy, wz;
    lin1(x, g.c, g.gx, l, u, wx);
    lin1(y, g.c, g.gy, l, u, wy);
    lin1(z, g.c, g.gz, l, u, wz);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      m[k] += val * ((k & 4) ? wz : 1.0 - wz) * ((k & 2) ? wy : 1.0 - wy) * ((k & 1) ? wx : 1.0 - wx);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    double s = m[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    m[k] = s;
  }
  if (lane == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) hc[8 * w + k] = (float)m[k];
  }
}

// Half cells along one axis whose corner (0: lower parent, 1: upper parent) is coarse
// index I; returns the count (at most 8), entries h * 2 + corner.
__device__ __forceinline__ int half_list(int I, int G, int* out) {
  int n = 0;
  for (int h = 2 * I - 1; h <= 2 * I + 2; ++h) {
    if (h < 0 || h >= 2 * G) continue;
    const int i0 = (h - 1) >> 1;
    const int lo = min(max(i0, 0), G - 1), hi = min(max(i0 + 1, 0), G - 1);
    if (lo == I) out[n++] = 2 * h;
    if (hi == I) out[n++] = 2 * h + 1;
  }
  return n;
}

__global__ void __launch_bounds__(256)
    k_restrict_sum(Grid g, const float* __restrict__ hc, float* __restrict__ rc, const int* gate) {
  if (gated(gate)) return;
  const int64_t I = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (I >= g.Vc()) return;
  const int Ix = (int)(I % g.gx), Iy = (int)((I / g.gx) % g.gy), Iz = (int)(I / ((int64_t)g.gx * g.gy));
  int lx[8], ly[8], lz[8];
  const int nx = half_list(Ix, g.gx, lx), ny = half_list(Iy, g.gy, ly), nz = half_list(Iz, g.gz, lz);
  const int64_t hn = 2 * g.gx, hm = 2 * g.gy;
  float s = 0.f;
  for (int a = 0; a < nz; ++a)
    for (int b = 0; b < ny; ++b)
      for (int e = 0; e < nx; ++e) {
        const int64_t H = ((int64_t)(lz[a] >> 1) * hm + (ly[b] >> 1)) * hn + (lx[e] >> 1);
        s += __ldg(hc + 8 * H + 4 * (lz[a] & 1) + 2 * (ly[b] & 1) + (lx[e] & 1));
      }
  rc[I] = s;
}

template <class T>
__global__ void __launch_bounds__(256)
    k_prolong_add(Grid g, int64_t np, const float* __restrict__ y, const int* __restrict__ rowAt, T* __restrict__ z,
                  const int* gate) {
  if (gated(gate)) return;
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int64_t nat = rowAt ? (int64_t)rowAt[p] : p;
  if (nat < 0) return;
  const int x = (int)(nat % g.nx), yy = (int)((nat / g.nx) % g.ny), zz = (int)(nat / ((int64_t)g.nx * g.ny));
  int x0, x1, y0, y1, z0, z1;
  double wx, wy, wz;
  lin1(x, g.c, g.gx, x0, x1, wx);
  lin1(yy, g.c, g.gy, y0, y1, wy);
  lin1(zz, g.c, g.gz, z0, z1, wz);
  const float fx = (float)wx, fy = (float)wy, fz = (float)wz;
  auto at = [&](int c, int b, int a) { return __ldg(y + ((int64_t)c * g.gy + b) * g.gx + a); };
  const float c00 = at(z0, y0, x0) * (1.f - fz) + at(z1, y0, x0) * fz;
  const float c01 = at(z0, y0, x1) * (1.f - fz) + at(z1, y0, x1) * fz;
  const float c10 = at(z0, y1, x0) * (1.f - fz) + at(z1, y1, x0) * fz;
  const float c11 = at(z0, y1, x1) * (1.f - fz) + at(z1, y1, x1) * fz;
  const float c0 = c00 * (1.f - fy) + c10 * fy;
  const float c1 = c01 * (1.f - fy) + c11 * fy;
  z[p] += (T)(c0 * (1.f - fx) + c1 * fx);
}

__global__ void __launch_bounds__(kRmsThreads) k_rms(int64_t V, const float* __restrict__ v, float* __restrict__ scal,
                                                    const int* gate) {
  if (gated(gate)) return;
  __shared__ double red[kRmsThreads / 32];
  double s = 0.0;
  for (int64_t i = threadIdx.x; i < V; i += kRmsThreads) s += (double)v[i] * v[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kRmsThreads / 32; ++w) t += red[w];
    const double r = sqrt(t / (double)V);
    scal[0] = r > 0.0 ? (float)(1.0 / r) : 0.f;
    scal[1] = (float)r;
  }
}

// ---------------------------------------------------------------- cluster PCG
struct PcgK {
  PcgArgs a;
  int ppr;      // coarse z-planes per CTA
  int chunk;    // cells per CTA (ppr gx gy)
};

// Sum of N per-thread values over the whole cluster, identical in every thread of every
// CTA: warp shuffles, warps in order, then each CTA's total is written into slot `rank` of
// every CTA's shared table and the ranks are added in order after the cluster barrier.
template <int N>
__device__ __forceinline__ void cluster_sum(double (&v)[N], double* wred, double* slots, cg::cluster_group& cl,
                                            int rank, int ncta) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double s = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
    if (lane == 0) wred[wid * N + k] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[N];
#pragma unroll
    for (int k = 0; k < N; ++k) s[k] = 0.0;
    for (int w = 0; w < kPcgThreads / 32; ++w)
#pragma unroll
      for (int k = 0; k < N; ++k) s[k] += wred[w * N + k];
    for (int q = 0; q < ncta; ++q) {
      double* dst = cl.map_shared_rank(slots, q);
#pragma unroll
      for (int k = 0; k < N; ++k) dst[rank * N + k] = s[k];
    }
  }
  cl.sync();
#pragma unroll
  for (int k = 0; k < N; ++k) {
    double s = 0.0;
    for (int q = 0; q < ncta; ++q) s += slots[q * N + k];
    v[k] = s;
  }
}

template <int CPT>
__global__ void __launch_bounds__(kPcgThreads, 1) k_coarse_pcg(PcgK K) {
  extern __shared__ float p_s[];                   // this CTA's part of the search direction
  __shared__ double wred[2 * kPcgThreads / 32];
  __shared__ double slots[2][2 * kPcgCluster];     // alternating tables of the cluster sums
  __shared__ float* ptab[kPcgCluster];
  const PcgArgs& a = K.a;
  if (gated(a.gate)) return;                      // every CTA reads the same flag
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), ncta = (int)cl.num_blocks();
  const int gx = a.g.gx, gy = a.g.gy, gz = a.g.gz;
  const int64_t Vc = a.g.Vc(), gxy = (int64_t)gx * gy;
  if (threadIdx.x < ncta) ptab[threadIdx.x] = cl.map_shared_rank(p_s, (int)threadIdx.x);
  const int64_t base = (int64_t)rank * K.chunk;
  const int64_t left = Vc - base;
  const int nloc = left <= 0 ? 0 : (int)(left < K.chunk ? left : K.chunk);
  float y[CPT], r[CPT], p[CPT], d[CPT], q[CPT];
  int par = 0;
  auto sum1 = [&](double x) {
    double v[1] = {x};
    cluster_sum<1>(v, wred, slots[par], cl, rank, ncta);
    par ^= 1;
    return v[0];
  };
  // q = A_c p_s over the local cells (p_s of all CTAs complete: caller synchronised).
  auto spmv = [&]() {
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      const int i = threadIdx.x + k * kPcgThreads;
      q[k] = 0.f;
      if (i >= nloc) continue;
      const int64_t I = base + i;
      const int Ix = (int)(I % gx), Iy = (int)((I / gx) % gy), Iz = (int)(I / gxy);
      float s = 0.f;
#pragma unroll
      for (int t = 0; t < kTaps; ++t) {
        const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
        const int jx = Ix + dx, jy = Iy + dy, jz = Iz + dz;
        if (jx < 0 || jx >= gx || jy < 0 || jy >= gy || jz < 0 || jz >= gz) continue;
        const int owner = jz / K.ppr;
        const int64_t loc = (int64_t)(jz - owner * K.ppr) * gxy + (int64_t)jy * gx + jx;
        s += __ldg(a.ac + (int64_t)t * Vc + I) * ptab[owner][loc];
      }
      q[k] = s;
    }
  };
  cl.sync();   // ptab written, and every CTA of the cluster running before any remote access
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = threadIdx.x + k * kPcgThreads;
    const bool in = i < nloc;
    r[k] = in ? a.rc[base + i] : 0.f;
    d[k] = in ? a.dinv[base + i] : 0.f;
    y[k] = (in && a.g0) ? a.g0[base + i] : 0.f;
  }
  if (a.g0) {
    // y = gamma g0 with gamma = <rc, g0> / <g0, A_c g0>; r = rc - gamma A_c g0
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      const int i = threadIdx.x + k * kPcgThreads;
      if (i < nloc) p_s[i] = y[k];
    }
    cl.sync();
    spmv();
    double v[2] = {0.0, 0.0};
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      v[0] += (double)r[k] * y[k];
      v[1] += (double)y[k] * q[k];
    }
    cluster_sum<2>(v, wred, slots[par], cl, rank, ncta);
    par ^= 1;
    const float gam = v[1] != 0.0 && isfinite(v[0] / v[1]) ? (float)(v[0] / v[1]) : 0.f;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      y[k] *= gam;
      r[k] -= gam * q[k];
    }
  }
  double rz = 0.0;
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    p[k] = d[k] * r[k];
    rz += (double)r[k] * p[k];
  }
  rz = sum1(rz);
  for (int it = 0; it < a.steps; ++it) {
    if (!(fabs(rz) > 0.0)) break;               // converged or NaN: the same in every CTA
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      const int i = threadIdx.x + k * kPcgThreads;
      if (i < nloc) p_s[i] = p[k];
    }
    cl.sync();
    spmv();
    double pq = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; ++k) pq += (double)p[k] * q[k];
    pq = sum1(pq);
    if (!(fabs(pq) > 0.0)) break;
    const float alpha = (float)(rz / pq);
    double rz1 = 0.0;
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      y[k] += alpha * p[k];
      r[k] -= alpha * q[k];
      rz1 += (double)r[k] * (d[k] * r[k]);
    }
    rz1 = sum1(rz1);
    const float beta = (float)(rz1 / rz);
#pragma unroll
    for (int k = 0; k < CPT; ++k) p[k] = d[k] * r[k] + beta * p[k];
    rz = rz1;
  }
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = threadIdx.x + k * kPcgThreads;
    if (i < nloc) a.y[base + i] = y[k];
  }
  cl.sync();   // no CTA leaves while another may still read its shared memory
}

int pcg_ppr(const Grid& g) { return (g.gz + kPcgCluster - 1) / kPcgCluster; }

}  // namespace

int64_t max_coarse_cells() { return (int64_t)kPcgCluster * kPcgThreads * kPcgMaxCpt; }

void check_grid(const Grid& g) {
  PB_CHECK(g.c >= 2 && g.c % 2 == 0, PARCEL_B_E_ARG, "the coarse-grid stage needs an even coarsening factor (%d)",
           g.c);
  PB_CHECK(g.nx % g.c == 0 && g.ny % g.c == 0 && g.nz % g.c == 0 && g.gx > 0 && g.gy > 0 && g.gz > 0,
           PARCEL_B_E_ARG, "grid %d x %d x %d is not divisible by the coarsening factor %d", g.nx, g.ny, g.nz, g.c);
  const int64_t chunk = (int64_t)pcg_ppr(g) * g.gx * g.gy;
  PB_CHECK(chunk <= (int64_t)kPcgThreads * kPcgMaxCpt, PARCEL_B_E_UNSUPPORTED,
           "coarse grid %d x %d x %d is too large for the one-cluster coarse solver (at most %d cells per CTA, "
           "%d CTAs over z-planes): use a larger coarsening factor",
           g.gx, g.gy, g.gz, kPcgThreads * kPcgMaxCpt, kPcgCluster);
}

void galerkin(const Grid& g, const DevMat<double>& A, double* ac64, cudaStream_t st) {
  check_grid(g);
  PB_CHECK((int64_t)A.n == (int64_t)g.nx * g.ny * g.nz, PARCEL_B_E_ARG, "matrix has %d rows, the grid %d x %d x %d",
           A.n, g.nx, g.ny, g.nz);
  k_galerkin<<<(unsigned)g.Vc(), kGalThreads, 0, st>>>(g, A.rowptr, A.col, A.val, A.rbase, A.cbase, ac64);
  PB_CUDA(cudaGetLastError());
}

void to_f32(int64_t Vc, const double* ac64, float* ac32, float* dinv32, cudaStream_t st) {
  k_to_f32<<<(unsigned)((Vc + 255) / 256), 256, 0, st>>>(Vc, ac64, ac32, dinv32);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void restrict_fine(const Grid& g, const T* v, const int* pos, float* hc, float* rc, const int* gate,
                   cudaStream_t st) {
  const int64_t warps = g.Vh();
  k_restrict_half<T><<<(unsigned)((warps * 32 + 255) / 256), 256, 0, st>>>(g, v, pos, hc, gate);
  k_restrict_sum<<<(unsigned)((g.Vc() + 255) / 256), 256, 0, st>>>(g, hc, rc, gate);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void prolong_add(const Grid& g, int64_t np, const float* y, const int* rowAt, T* z, const int* gate,
                 cudaStream_t st) {
  k_prolong_add<T><<<(unsigned)((np + 255) / 256), 256, 0, st>>>(g, np, y, rowAt, z, gate);
  PB_CUDA(cudaGetLastError());
}

void rms(int64_t Vc, const float* v, float* scal, const int* gate, cudaStream_t st) {
  k_rms<<<1, kRmsThreads, 0, st>>>(Vc, v, scal, gate);
  PB_CUDA(cudaGetLastError());
}

void pcg(const PcgArgs& a, cudaStream_t st) {
  check_grid(a.g);
  PcgK K;
  K.a = a;
  K.ppr = pcg_ppr(a.g);
  K.chunk = K.ppr * a.g.gx * a.g.gy;
  const int cpt = (K.chunk + kPcgThreads - 1) / kPcgThreads;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kPcgCluster);
  cfg.blockDim = dim3(kPcgThreads);
  cfg.dynamicSmemBytes = sizeof(float) * (size_t)K.chunk;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kPcgCluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cpt <= 1) PB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_pcg<1>, K));
  else if (cpt <= 2) PB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_pcg<2>, K));
  else if (cpt <= 4) PB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_pcg<4>, K));
  else PB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_pcg<8>, K));
}

template void restrict_fine<float>(const Grid&, const float*, const int*, float*, float*, const int*, cudaStream_t);
template void restrict_fine<double>(const Grid&, const double*, const int*, float*, float*, const int*,
                                    cudaStream_t);
template void prolong_add<float>(const Grid&, int64_t, const float*, const int*, float*, const int*, cudaStream_t);
template void prolong_add<double>(const Grid&, int64_t, const float*, const int*, double*, const int*,
                                  cudaStream_t);

}  // namespace coarse
}  // namespace pb
