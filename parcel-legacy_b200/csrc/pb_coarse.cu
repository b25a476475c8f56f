// pb_coarse.cu -- Galerkin coarse-grid operator, grid transfers and the one-cluster coarse
// Jacobi-PCG of the two-level preconditioner stage (no counterpart in the reference).
//
// Kernels:
//   k_galerkin       one CTA per coarse cell: A_c(I, I + d) = sum_f sum_g P(f, I) A(f, g) P(g, I + d)
//                    over the fine cells f whose interpolation involves I; every thread keeps
//                    private sums for the 27 taps in shared memory and the 27 tap owners add
//                    the threads' sums in thread order (deterministic).
//   k_restrict_half  one thread per half cell ((c/2)^3 fine cells that share their two
//                    coarse parents along every axis): the 8 weighted sums of the half cell.
//   k_restrict_sum   one thread per coarse cell: adds the half-cell sums that belong to it,
//                    in a fixed order.
//   k_prolong_add    one thread per iteration-layout position: z += trilinear(y), the fine
//                    cell's coordinates read from a packed per-position code (k_pack_coords).
//   k_coarse_pcg     one thread-block cluster (8 CTAs x 512 threads), see pcg().
#include <cooperative_groups.h>

#include "pb_coarse.cuh"
#include "pb_device.cuh"

namespace cg = cooperative_groups;

namespace pb {
namespace coarse {
namespace {

constexpr int kGalThreads = 128;
constexpr int kPcgThreads = 512;
constexpr int kPcgCluster = 8;
constexpr int kPcgMaxCpt = 16;      // coarse cells per thread
constexpr int64_t kMaxCoarseCells = 49152;   // the prolongation stages the coarse vector in shared memory
constexpr int kRmsThreads = 1024;
constexpr int kProlongThreads = 1024;

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
// all of them interpolate from the same two coarse cells per axis, and the weight of the
// upper one for local offset l is (2 l + 1) / (2 c), plus 1/2 when hx is even.
// hc[8 H + 4 cz + 2 cy + cx] = sum over the half cell of v * wz_cz * wy_cy * wx_cx
// (w_0 = 1 - w, w_1 = w), one thread per half cell, summed in z, y, x order.
template <class T>
__global__ void __launch_bounds__(256)
    k_restrict_half(Grid g, const T* __restrict__ v, const int* __restrict__ pos, float* __restrict__ hc,
                    const int* gate) {
  if (gated(gate)) return;
  const int64_t H = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (H >= g.Vh()) return;
  const int hn = 2 * g.gx, hm = 2 * g.gy;
  const int hx = (int)(H % hn), hy = (int)((H / hn) % hm), hz = (int)(H / ((int64_t)hn * hm));
  const int hs = g.c / 2;
  const float inv2c = 0.5f / (float)g.c;
  const float ox = (hx & 1) ? 0.f : 0.5f, oy = (hy & 1) ? 0.f : 0.5f, oz = (hz & 1) ? 0.f : 0.5f;
  float m[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) m[k] = 0.f;
  for (int lz = 0; lz < hs; ++lz) {
    const float wz = oz + (float)(2 * lz + 1) * inv2c;
    for (int ly = 0; ly < hs; ++ly) {
      const float wy = oy + (float)(2 * ly + 1) * inv2c;
      const float wyz[4] = {(1.f - wy) * (1.f - wz), wy * (1.f - wz), (1.f - wy) * wz, wy * wz};
      const int64_t row = ((int64_t)(hz * hs + lz) * g.ny + (hy * hs + ly)) * g.nx + (int64_t)hx * hs;
      for (int lx = 0; lx < hs; ++lx) {
        const float wx = ox + (float)(2 * lx + 1) * inv2c;
        const int64_t nat = row + lx;
        const float val = (float)v[pos ? pos[nat] : nat];
        const float a0 = val * (1.f - wx), a1 = val * wx;
#pragma unroll
        for (int k = 0; k < 8; ++k) m[k] = fmaf((k & 1) ? a1 : a0, wyz[k >> 1], m[k]);
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) hc[8 * H + k] = m[k];
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

// Interpolation along one axis in FP32 (c even: u is never an integer, so the rounding of
// (i + 1/2) / c cannot move floor(u)).
__device__ __forceinline__ void lin1f(int i, float inv_c, int G, int& lo, int& hi, float& w) {
  const float u = ((float)i + 0.5f) * inv_c - 0.5f;
  const float f = floorf(u);
  w = u - f;
  const int i0 = (int)f;
  lo = min(max(i0, 0), G - 1);
  hi = min(max(i0 + 1, 0), G - 1);
}

// code[p] = x | y << 10 | z << 20 of the natural row at iteration position p, -1 for padding.
__global__ void __launch_bounds__(256)
    k_pack_coords(Grid g, int64_t np, const int* __restrict__ rowAt, int* __restrict__ code) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int64_t nat = rowAt ? (int64_t)rowAt[p] : p;
  if (nat < 0) { code[p] = -1; return; }
  const int x = (int)(nat % g.nx), y = (int)((nat / g.nx) % g.ny), z = (int)(nat / ((int64_t)g.nx * g.ny));
  code[p] = x | (y << 10) | (z << 20);
}

// One CTA per SM over a grid-stride range of positions; the coarse vector is first copied
// into shared memory (the trilinear gathers of neighbouring positions hit scattered coarse
// cells, which from L1 costs a wavefront per distinct line).
template <class T>
__global__ void __launch_bounds__(kProlongThreads)
    k_prolong_add(Grid g, int64_t np, const float* __restrict__ y, const int* __restrict__ code, T* __restrict__ z,
                  const int* gate) {
  if (gated(gate)) return;
  extern __shared__ float ys[];
  const int64_t V = g.Vc();
  for (int64_t i = threadIdx.x; i < V; i += kProlongThreads) ys[i] = __ldg(y + i);
  __syncthreads();
  const float inv_c = 1.f / (float)g.c;
  const int gxy = g.gx * g.gy;
  for (int64_t p = (int64_t)blockIdx.x * kProlongThreads + threadIdx.x; p < np;
       p += (int64_t)gridDim.x * kProlongThreads) {
    const int cd = code[p];
    if (cd < 0) continue;
    int x0, x1, y0, y1, z0, z1;
    float fx, fy, fz;
    lin1f(cd & 1023, inv_c, g.gx, x0, x1, fx);
    lin1f((cd >> 10) & 1023, inv_c, g.gy, y0, y1, fy);
    lin1f(cd >> 20, inv_c, g.gz, z0, z1, fz);
    const float* p0 = ys + z0 * gxy;
    const float* p1 = ys + z1 * gxy;
    const float c00 = p0[y0 * g.gx + x0] * (1.f - fz) + p1[y0 * g.gx + x0] * fz;
    const float c01 = p0[y0 * g.gx + x1] * (1.f - fz) + p1[y0 * g.gx + x1] * fz;
    const float c10 = p0[y1 * g.gx + x0] * (1.f - fz) + p1[y1 * g.gx + x0] * fz;
    const float c11 = p0[y1 * g.gx + x1] * (1.f - fz) + p1[y1 * g.gx + x1] * fz;
    const float c0 = c00 * (1.f - fy) + c10 * fy;
    const float c1 = c01 * (1.f - fy) + c11 * fy;
    z[p] += (T)(c0 * (1.f - fx) + c1 * fx);
  }
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

// pe holds this CTA's ppr coarse planes of the search direction between one halo plane
// below and one above: exchange() publishes the CTA's planes, waits for the cluster and
// copies the neighbours' boundary planes into the halos (zero at the grid's ends), so the
// product reads shared memory only.
template <int CPT>
__global__ void __launch_bounds__(kPcgThreads, 1) k_coarse_pcg(PcgK K) {
  extern __shared__ float pe[];                    // (ppr + 2) planes
  __shared__ double wred[2 * kPcgThreads / 32];
  __shared__ double slots[2][2 * kPcgCluster];     // alternating tables of the cluster sums
  const PcgArgs& a = K.a;
  if (gated(a.gate)) return;                      // every CTA reads the same flag
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), ncta = (int)cl.num_blocks();
  const int gx = a.g.gx, gy = a.g.gy;
  const int gxy = gx * gy;
  const int64_t Vc = a.g.Vc();
  const int64_t base = (int64_t)rank * K.chunk;
  const int64_t left = Vc - base;
  const int nloc = left <= 0 ? 0 : (int)(left < K.chunk ? left : K.chunk);
  const int64_t left_next = Vc - base - K.chunk;
  const bool has_prev = rank > 0 && nloc > 0;
  const bool has_next = rank + 1 < ncta && left_next > 0;
  float y[CPT], r[CPT], p[CPT], d[CPT], q[CPT];
  int cxy[CPT];                                    // x | y << 10 | local plane << 20
  const int halo_hi = (K.ppr + 1) * gxy;
  for (int i = threadIdx.x; i < gxy; i += kPcgThreads) {
    pe[i] = 0.f;
    pe[halo_hi + i] = 0.f;
  }
  int par = 0;
  auto sum1 = [&](double x) {
    double v[1] = {x};
    cluster_sum<1>(v, wred, slots[par], cl, rank, ncta);
    par ^= 1;
    return v[0];
  };
  auto exchange = [&](const float (&src)[CPT]) {
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      const int i = threadIdx.x + k * kPcgThreads;
      if (i < nloc) pe[gxy + i] = src[k];
    }
    cl.sync();
    if (has_prev) {
      const float* rp = cl.map_shared_rank(pe, rank - 1) + (size_t)K.ppr * gxy;   // its last plane
      for (int i = threadIdx.x; i < gxy; i += kPcgThreads) pe[i] = rp[i];
    }
    if (has_next) {
      const float* rn = cl.map_shared_rank(pe, rank + 1) + gxy;                    // its first plane
      for (int i = threadIdx.x; i < gxy; i += kPcgThreads) pe[halo_hi + i] = rn[i];
    }
    __syncthreads();
  };
  // q = A_c (the exchanged vector) over the local cells
  auto spmv = [&]() {
#pragma unroll
    for (int k = 0; k < CPT; ++k) {
      const int i = threadIdx.x + k * kPcgThreads;
      q[k] = 0.f;
      if (i >= nloc) continue;
      const int64_t I = base + i;
      const int x = cxy[k] & 1023, yy = (cxy[k] >> 10) & 1023, lz = cxy[k] >> 20;
      const float* c0 = pe + (lz + 1) * gxy + yy * gx + x;
      float s = 0.f;
#pragma unroll
      for (int t = 0; t < kTaps; ++t) {
        const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
        if ((dx < 0 && x == 0) || (dx > 0 && x == gx - 1) || (dy < 0 && yy == 0) || (dy > 0 && yy == gy - 1))
          continue;
        s += __ldg(a.ac + (int64_t)t * Vc + I) * c0[dz * gxy + dy * gx + dx];
      }
      q[k] = s;
    }
  };
#pragma unroll
  for (int k = 0; k < CPT; ++k) {
    const int i = threadIdx.x + k * kPcgThreads;
    const bool in = i < nloc;
    cxy[k] = in ? ((i % gx) | (((i / gx) % gy) << 10) | ((i / gxy) << 20)) : 0;
    r[k] = in ? a.rc[base + i] : 0.f;
    d[k] = in ? a.dinv[base + i] : 0.f;
    y[k] = (in && a.g0) ? a.g0[base + i] : 0.f;
  }
  cl.sync();   // halos zeroed, and every CTA of the cluster running before any remote access
  if (a.g0) {
    // y = gamma g0 with gamma = <rc, g0> / <g0, A_c g0>; r = rc - gamma A_c g0
    exchange(y);
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
    exchange(p);
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

int64_t max_coarse_cells() { return kMaxCoarseCells; }

void check_grid(const Grid& g) {
  PB_CHECK(g.c >= 2 && g.c % 2 == 0, PARCEL_B_E_ARG, "the coarse-grid stage needs an even coarsening factor (%d)",
           g.c);
  PB_CHECK(g.nx % g.c == 0 && g.ny % g.c == 0 && g.nz % g.c == 0 && g.gx > 0 && g.gy > 0 && g.gz > 0,
           PARCEL_B_E_ARG, "grid %d x %d x %d is not divisible by the coarsening factor %d", g.nx, g.ny, g.nz, g.c);
  PB_CHECK(g.nx <= 1024 && g.ny <= 1024 && g.nz <= 1024, PARCEL_B_E_UNSUPPORTED,
           "the coarse-grid stage supports at most 1024 cells per axis (grid %d x %d x %d)", g.nx, g.ny, g.nz);
  PB_CHECK(g.Vc() <= kMaxCoarseCells, PARCEL_B_E_UNSUPPORTED,
           "coarse grid %d x %d x %d has more than %lld cells: use a larger coarsening factor", g.gx, g.gy, g.gz,
           (long long)kMaxCoarseCells);
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
  k_restrict_half<T><<<(unsigned)((g.Vh() + 255) / 256), 256, 0, st>>>(g, v, pos, hc, gate);
  k_restrict_sum<<<(unsigned)((g.Vc() + 255) / 256), 256, 0, st>>>(g, hc, rc, gate);
  PB_CUDA(cudaGetLastError());
}

void pack_coords(const Grid& g, int64_t np, const int* rowAt, int* code, cudaStream_t st) {
  k_pack_coords<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(g, np, rowAt, code);
  PB_CUDA(cudaGetLastError());
}

template <class T>
void prolong_add(const Grid& g, int64_t np, const float* y, const int* code, T* z, const int* gate,
                 cudaStream_t st) {
  const size_t smem = sizeof(float) * (size_t)g.Vc();
  static bool attr_set[2] = {false, false};
  if (!attr_set[sizeof(T) == 8]) {   // before any stream capture: the stage's constructor calls this first
    PB_CUDA(cudaFuncSetAttribute(k_prolong_add<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(float) * kMaxCoarseCells)));
    attr_set[sizeof(T) == 8] = true;
  }
  k_prolong_add<T><<<num_sms(), kProlongThreads, smem, st>>>(g, np, y, code, z, gate);
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
  cfg.dynamicSmemBytes = sizeof(float) * (size_t)(K.ppr + 2) * a.g.gx * a.g.gy;
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
  else if (cpt <= 8) PB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_pcg<8>, K));
  else PB_CUDA(cudaLaunchKernelEx(&cfg, k_coarse_pcg<16>, K));
}

template void restrict_fine<float>(const Grid&, const float*, const int*, float*, float*, const int*, cudaStream_t);
template void restrict_fine<double>(const Grid&, const double*, const int*, float*, float*, const int*,
                                    cudaStream_t);
template void prolong_add<float>(const Grid&, int64_t, const float*, const int*, float*, const int*, cudaStream_t);
template void prolong_add<double>(const Grid&, int64_t, const float*, const int*, double*, const int*,
                                  cudaStream_t);

}  // namespace coarse
}  // namespace pb
