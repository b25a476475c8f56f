// pb_cnn.cu -- kernels of the learned coarse-grid preconditioner stage.
//
// The four 32 -> 32 convolutions and their transposes (backward pass) run on the
// 5th-generation tensor cores (tcgen05.mma, BF16 operands in shared memory, FP32
// accumulators in TMEM; k_conv32_tc).  The weight gradient is the voxel-axis contraction
// on warp-level MMAs (ldmatrix.trans operands, m16n8k16 BF16 -> FP32); every CTA writes a
// partial and a second kernel sums the partials in CTA order, so gradients are
// deterministic.  The 2 -> 32 input layer and the 32 -> 1 output layer have too few MACs
// per voxel for the tensor cores and run on the CUDA cores.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "pb_cnn.cuh"
#include "pb_device.cuh"

namespace pb {
namespace cnn {

namespace {

typedef __nv_bfloat16 bf16;

constexpr int TX = 32, TY = 4, TZ = 2;                 // output tile of one CTA
constexpr int BX = TX + 2, BY = TY + 2, BZ = TZ + 2;   // halo brick
constexpr int kBrickRows = BX * BY * BZ;               // 816 voxels
constexpr int kTileVox = TX * TY * TZ;                 // 256 voxels
constexpr int kBrickBytes = kBrickRows * 64;           // 52,224 B
constexpr int kWgSmem = kBrickBytes + kTileVox * 64;
constexpr int kWgThreads = 288;                        // 9 warps: 3 taps each
constexpr int kWgPart = kTaps * kCh * kCh + kCh;       // W then b of one 32 -> 32 layer
constexpr int kL1Part = kTaps * kCin * kCh + kCh;      // 1,760
constexpr int kL6Part = kTaps * kCh + 1;               // 865

struct Tiles {
  int ntx, nty, ntz;
  int64_t per_sample, total;
};
__host__ __device__ inline Tiles tiles_of(const Geo& g, int batch) {
  Tiles t;
  t.ntx = (g.gx + TX - 1) / TX;
  t.nty = (g.gy + TY - 1) / TY;
  t.ntz = (g.gz + TZ - 1) / TZ;
  t.per_sample = (int64_t)t.ntx * t.nty * t.ntz;
  t.total = t.per_sample * batch;
  return t;
}

// Hidden activations and their gradients are stored chunk-planar: channel group c / 8 of
// sample b is a plane [gz][gy][gx][8 channels], planes ordered (b, c / 8).  A line of
// voxels is then 16 contiguous bytes per voxel within a plane, so the tensor copies of the
// tensor-core convolution move 512-byte rows.
__host__ __device__ __forceinline__ int64_t aoff(int64_t b, int64_t v, int c, int64_t V) {
  return ((b * 4 + (c >> 3)) * V + v) * 8 + (c & 7);
}

// 64-byte rows (32 BF16 channels) of four 16-byte chunks; the chunk index is XORed with
// bits 1..2 of the row so that ldmatrix over any 8 consecutive rows is conflict-free.
__device__ __forceinline__ uint32_t swz(int row, int chunk) {
  return (uint32_t)row * 64u + ((uint32_t)(chunk ^ ((row >> 1) & 3)) << 4);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}
__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr) : "memory");
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], uint32_t addr) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(addr) : "memory");
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Keeps each BF16 half of v where the matching half of m is > 0 (ReLU derivative).
__device__ __forceinline__ uint32_t mask_pairs(uint32_t v, uint32_t m) {
  const uint32_t lo = ((int16_t)(m & 0xFFFFu) > 0) ? 0x0000FFFFu : 0u;
  const uint32_t hi = ((int16_t)(m >> 16) > 0) ? 0xFFFF0000u : 0u;
  return v & (lo | hi);
}

__device__ __forceinline__ void tile_origin(const Tiles& T, int64_t tile, int64_t& b, int& x0, int& y0, int& z0) {
  b = tile / T.per_sample;
  const int64_t rem = tile - b * T.per_sample;
  x0 = (int)(rem % T.ntx) * TX;
  y0 = (int)((rem / T.ntx) % T.nty) * TY;
  z0 = (int)(rem / ((int64_t)T.ntx * T.nty)) * TZ;
}

// Halo brick of 32-channel BF16 voxels (zero outside the grid) into shared memory.
__device__ __forceinline__ void load_brick(uint32_t sb, const bf16* in, const Geo& g, int64_t b, int x0,
                                           int y0, int z0) {
  for (int idx = threadIdx.x; idx < kBrickRows * 4; idx += blockDim.x) {
    const int row = idx >> 2, ch = idx & 3;
    const int bx = row % BX, r2 = row / BX, by = r2 % BY, bz = r2 / BY;
    const int x = x0 + bx - 1, y = y0 + by - 1, z = z0 + bz - 1;
    const bool ok = (unsigned)x < (unsigned)g.gx && (unsigned)y < (unsigned)g.gy && (unsigned)z < (unsigned)g.gz;
    const bf16* src = ok ? in + aoff(b, ((int64_t)z * g.gy + y) * g.gx + x, ch * 8, g.V()) : in;
    cp_async16(sb + swz(row, ch), src, ok);
  }
}

// ---------------------------------------------------------------- 32 -> 32 convolution
// out = relu(conv3(in, W) + b)                          (forward)
// out = conv3(in, W') where mask > 0, else 0            (transposed convolution, W' mirrored)
// ---------------------------------------------------------------- tcgen05 32 -> 32 convolution
// The same convolution on the 5th-generation tensor cores.  A CTA of 4 warps owns an output
// tile of 32 (x) x 4 (y) x 2 (z) voxels.  Shared memory holds three copies of the halo brick
// shifted by dx = -1, 0, +1 (zero outside the grid), each in the canonical K-major
// no-swizzle layout: for every 8-channel K chunk, the brick's rows (voxels) of 16 bytes one
// after another.  Lines are 32 rows apart, so for any tap (dz, dy, dx) the 128 A rows of
// 4 consecutive output lines form 16 core matrices 128 bytes apart (SBO = 128) and the two
// K chunks of one MMA lie one chunk plane apart (LBO).  The packed weights of all 27 taps
// use the same layout with N = 32 rows.  One thread issues M=128 N=32 K=16 BF16 MMAs into
// FP32 accumulators in TMEM: per z plane the taps are dealt round-robin to 4 accumulators
// (32 columns each), so 8 independent MMA chains are in flight; tcgen05.commit arrives on
// an mbarrier; each warp then reads its 32 TMEM lanes (one voxel per thread, all 32
// channels), sums the 4 partial accumulators and applies the bias + ReLU (or ReLU-mask)
// epilogue with 64-byte stores.  The bricks arrive by tensor copies (TMA).
constexpr int kTcLinesY = TY + 2, kTcLinesZ = TZ + 2;               // 6 x 4 brick lines
constexpr int kTcRows = kTcLinesY * kTcLinesZ * TX;                  // 768 rows per copy
constexpr int kTcPlane = kTcRows * 16;                              // 12,288 B per K chunk
constexpr int kTcCopy = 4 * kTcPlane;                               // 49,152 B per shifted copy
constexpr int kTcWTap = 4 * kCh * 16;                               // 2,048 B per tap
constexpr int kTcWBytes = kTaps * kTcWTap;                          // 55,296 B
constexpr int kTcSmem = 3 * kTcCopy + kTcWBytes + 256;              // + barrier, TMEM address, bias
constexpr int kTcThreads = 160;                                     // issuer warp + 4 epilogue warps
constexpr int kTcSplit = 2;                                         // accumulators per z plane
constexpr int kTcCols = 2 * TZ * kTcSplit * kCh;                    // two buffers: 256 TMEM columns
constexpr unsigned kTcWaitLimit = 1u << 24;
// kind::f16 instruction descriptor: D FP32 (bits 4-5 = 1), A BF16 (7-9 = 1), B BF16
// (10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCh >> 3) << 17) | ((128u >> 4) << 24);

// Shared-memory matrix descriptor, no swizzle: start >> 4 (bits 0-13), LBO >> 4 (16-29),
// SBO >> 4 (32-45), descriptor version 1 (bits 46-47), layout type 0 (bits 61-63).
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// Tensor copy of one box {8 channels, 32 x, 6 y, 4 z, 1 sample} (12,288 bytes) into shared
// memory; coordinates outside the tensor read zeros.  The innermost coordinate (channel)
// is a multiple of 8 elements = 16 bytes.
__device__ __forceinline__ void tma_box5(uint32_t dst, const CUtensorMap* map, int c, int x, int y, int z, int b,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
      ::"r"(dst), "l"(map), "r"(c), "r"(x), "r"(y), "r"(z), "r"(b), "r"(smem_u32(bar)) : "memory");
}

template <bool DGRAD>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_conv32_tc(const __grid_constant__ CUtensorMap tmap, Geo g, int batch, const bf16* __restrict__ wpk,
                const float* __restrict__ bias, const bf16* __restrict__ mask, bf16* __restrict__ out,
                int* err, const int* gate) {
  if (gated(gate)) return;
  extern __shared__ __align__(128) unsigned char smem[];
  const uint32_t sbase = smem_u32(smem);
  const uint32_t wsm = sbase + 3 * kTcCopy;
  unsigned char* ctl = smem + 3 * kTcCopy + kTcWBytes;
  uint64_t* lbar = reinterpret_cast<uint64_t*>(ctl);        // [2] brick halves landed (K chunks 0-1, 2-3)
  uint64_t* abar = lbar + 2;                                 // MMAs on chunks 0-1 done
  uint64_t* mbar = lbar + 3;                                 // [2] all MMAs of a tile done, per TMEM buffer
  uint64_t* ebar = lbar + 5;                                 // [2] TMEM buffer read by the epilogue
  uint32_t* tslot = reinterpret_cast<uint32_t*>(ctl + 64);
  float* sbias = reinterpret_cast<float*>(ctl + 128);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // weights of all taps, canonical layout: tap t, K chunk c, row n at t*2048 + c*512 + n*16
  for (int idx = threadIdx.x; idx < kTaps * kCh * 4; idx += kTcThreads) {
    const int c = idx & 3, n = (idx >> 2) & 31, t = idx >> 7;
    cp_async16(wsm + t * kTcWTap + c * (kCh * 16) + n * 16, wpk + (t * kCh + n) * kCh + c * 8, true);
  }
  if (threadIdx.x < kCh) sbias[threadIdx.x] = DGRAD ? 0.f : bias[threadIdx.x];
  if (threadIdx.x == 0) {
    for (int i = 0; i < 5; ++i) mbar_init(lbar + i, 1);
    mbar_init(ebar, 4);
    mbar_init(ebar + 1, 4);
    mbar_fence_init();
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  cp_async_wait_all();
  fence_async_shared();   // the weights came through the generic proxy; the MMAs read async
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tslot;
  const Tiles T = tiles_of(g, batch);
  const int64_t V = g.V();

  if (warp == 0) {
    // ---------------- issuer: tensor copies and MMAs (one elected lane)
    if (lane == 0) {
      auto load_half = [&](int64_t tile, int h) {   // K chunks 2h, 2h+1 of all three copies
        int64_t b;
        int x0, y0, z0;
        tile_origin(T, tile, b, x0, y0, z0);
        mbar_arrive_expect_tx(lbar + h, 6u * (unsigned)kTcPlane);
        for (int sh = 0; sh < 3; ++sh)
          for (int c = 2 * h; c < 2 * h + 2; ++c)
            tma_box5(sbase + sh * kTcCopy + c * kTcPlane, &tmap, 0, x0 + sh - 1, y0 - 1, z0 - 1, (int)(b * 4 + c),
                     lbar + h);
      };
      // Descriptors of the brick copies and of the weights at offset 0; every operand of the
      // unrolled loop is that base plus a compile-time offset (>> 4 in the start field).
      const uint64_t a_base = tc_desc(sbase, kTcPlane, 128);
      const uint64_t b_base = tc_desc(wsm, kCh * 16, 128);
      auto mmas = [&](int buf, int ks) {
        const uint32_t tbuf = tmem + (uint32_t)(buf * TZ * kTcSplit * kCh);
#pragma unroll
        for (int t = 0; t < kTaps; ++t) {
          const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
          const uint64_t bd = b_base + (uint64_t)((t * kTcWTap + 2 * ks * (kCh * 16)) >> 4);
#pragma unroll
          for (int zz = 0; zz < TZ; ++zz) {
            const int row0 = ((zz + 1 + dz) * kTcLinesY + (1 + dy)) * TX;
            const uint64_t ad = a_base + (uint64_t)(((dx + 1) * kTcCopy + 2 * ks * kTcPlane + row0 * 16) >> 4);
            // tap t accumulates into chain t % kTcSplit of its z plane
            tc_mma(tbuf + (uint32_t)((zz * kTcSplit + t % kTcSplit) * kCh), ad, bd, (ks > 0 || t >= kTcSplit) ? 1u : 0u);
          }
        }
      };
      bool ok = true;
      int i = 0;
      int64_t tile = blockIdx.x;
      if (tile < T.total) { load_half(tile, 0); load_half(tile, 1); }
      for (; tile < T.total && ok; tile += gridDim.x, ++i) {
        const int buf = i & 1;
        const unsigned par = (unsigned)i & 1u, bpar = (unsigned)(i >> 1) & 1u;
        ok = mbar_wait(lbar, par, kTcWaitLimit);
        if (ok && i >= 2) ok = mbar_wait(ebar + buf, bpar ^ 1u, kTcWaitLimit);
        if (!ok) break;
        tc_fence_after();
        mmas(buf, 0);
        tc_commit(abar);
        ok = mbar_wait(lbar + 1, par, kTcWaitLimit);
        if (!ok) break;
        mmas(buf, 1);
        tc_commit(mbar + buf);
        const int64_t next = tile + gridDim.x;
        ok = mbar_wait(abar, par, kTcWaitLimit);             // chunks 0-1 no longer read
        if (ok && next < T.total) load_half(next, 0);
        if (ok) ok = mbar_wait(mbar + buf, bpar, kTcWaitLimit);   // chunks 2-3 no longer read
        if (ok && next < T.total) load_half(next, 1);
      }
      if (!ok) atomicExch(err, 4);
    }
    __syncwarp();
  } else {
    // ---------------- epilogue warps 1-4: TMEM lanes 32 (warp % 4) .. + 31 = output line
    const int q = warp & 3;
    int i = 0;
    for (int64_t tile = blockIdx.x; tile < T.total; tile += gridDim.x, ++i) {
      const int buf = i & 1;
      const unsigned bpar = (unsigned)(i >> 1) & 1u;
      if (!mbar_wait(mbar + buf, bpar, kTcWaitLimit)) {
        atomicExch(err, 6);
        break;
      }
      tc_fence_after();
      int64_t b;
      int x0, y0, z0;
      tile_origin(T, tile, b, x0, y0, z0);
      float acc[TZ][32];
#pragma unroll
      for (int zz = 0; zz < TZ; ++zz) {
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[zz][j] = 0.f;
#pragma unroll 1
        for (int k = 0; k < kTcSplit; ++k) {
          uint32_t r[32];
          tc_ld32(tmem + ((uint32_t)(32 * q) << 16) + ((buf * TZ + zz) * kTcSplit + k) * kCh, r);
#pragma unroll
          for (int j = 0; j < 32; ++j) acc[zz][j] += __uint_as_float(r[j]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(ebar + buf);   // this warp's lanes of the buffer are free
      const int y = y0 + q, x = x0 + lane;
#pragma unroll
      for (int zz = 0; zz < TZ; ++zz) {
        const int z = z0 + zz;
        if (x < g.gx && y < g.gy && z < g.gz) {
          const int64_t vox = ((int64_t)z * g.gy + y) * g.gx + x;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            uint32_t w4[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int co = k * 8 + j * 2;
              float v0 = acc[zz][co], v1 = acc[zz][co + 1];
              if (!DGRAD) {
                v0 = fmaxf(v0 + sbias[co], 0.f);
                v1 = fmaxf(v1 + sbias[co + 1], 0.f);
              }
              __nv_bfloat162 pk = __floats2bfloat162_rn(v0, v1);
              w4[j] = *reinterpret_cast<uint32_t*>(&pk);
            }
            const int64_t o = aoff(b, vox, k * 8, V);
            if (DGRAD) {
              const uint4 m = *reinterpret_cast<const uint4*>(mask + o);
              w4[0] = mask_pairs(w4[0], m.x);
              w4[1] = mask_pairs(w4[1], m.y);
              w4[2] = mask_pairs(w4[2], m.z);
              w4[3] = mask_pairs(w4[3], m.w);
            }
            *reinterpret_cast<uint4*>(out + o) = make_uint4(w4[0], w4[1], w4[2], w4[3]);
          }
        }
      }
    }
  }
  // every copy and MMA the issuer started has completed or been waited for (bounded) above
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
}

// ---------------------------------------------------------------- 32 -> 32 weight gradient
// part[cta] = ( dW[t][ci][co] = sum_v a[v + d_t][ci] g[v][co],  db[co] = sum_v g[v][co] )
// over the tiles of this CTA.  Warp w owns taps w, w + 9, w + 18.
__global__ void __launch_bounds__(kWgThreads, 1)
    k_wgrad32(Geo g, int batch, const bf16* __restrict__ a_in, const bf16* __restrict__ gout, float* __restrict__ part) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ float sdb[kWgThreads / 32][kCh];
  const uint32_t sb = smem_u32(smem), sg = sb + kBrickBytes;
  const Tiles T = tiles_of(g, batch);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = lane >> 3, rr = lane & 7, gq = lane >> 2, tq = lane & 3;
  const int64_t V = g.V();
  float acc[3][2][4][4];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int l = 0; l < 4; ++l) acc[i][j][k][l] = 0.f;
  float db = 0.f;
  for (int64_t tile = blockIdx.x; tile < T.total; tile += gridDim.x) {
    int64_t b;
    int x0, y0, z0;
    tile_origin(T, tile, b, x0, y0, z0);
    load_brick(sb, a_in, g, b, x0, y0, z0);
    for (int idx = threadIdx.x; idx < kTileVox * 4; idx += kWgThreads) {
      const int tv = idx >> 2, ch = idx & 3;
      const int x = x0 + tv % TX, y = y0 + (tv / TX) % TY, z = z0 + tv / (TX * TY);
      const bool ok = x < g.gx && y < g.gy && z < g.gz;
      const bf16* src = ok ? gout + aoff(b, ((int64_t)z * g.gy + y) * g.gx + x, ch * 8, V) : gout;
      cp_async16(sg + swz(tv, ch), src, ok);
    }
    cp_async_wait_all();
    __syncthreads();
    {
      const int co = threadIdx.x & 31;
      for (int v = warp; v < kTileVox; v += kWgThreads / 32)
        db += __bfloat162float(*reinterpret_cast<const bf16*>(smem + kBrickBytes + swz(v, co >> 3) + (co & 7) * 2));
    }
#pragma unroll 1
    for (int L = 0; L < TY * TZ; ++L) {
      const int wy = L % TY, wz = L / TY;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int tvb = L * TX + h * 16;
        uint32_t bq[4][2];
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          uint32_t r[4];
          ldsm_x4_t(r, sg + swz(tvb + (q & 1) * 8 + rr, np * 2 + (q >> 1)));
          bq[np * 2][0] = r[0];
          bq[np * 2][1] = r[1];
          bq[np * 2 + 1][0] = r[2];
          bq[np * 2 + 1][1] = r[3];
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) {
          const int t = warp + 9 * i;
          const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
          const int rbase = ((wz + 1 + dz) * BY + (wy + 1 + dy)) * BX + 1 + dx + h * 16;
#pragma unroll
          for (int mt = 0; mt < 2; ++mt) {
            uint32_t a[4];
            ldsm_x4_t(a, sb + swz(rbase + (q >> 1) * 8 + rr, mt * 2 + (q & 1)));
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[i][mt][nt], a, bq[nt][0], bq[nt][1]);
          }
        }
      }
    }
    __syncthreads();
  }
  float* P = part + (size_t)blockIdx.x * kWgPart;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int t = warp + 9 * i;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
          const int ci = mt * 16 + gq + (r >> 1) * 8, co = nt * 8 + tq * 2 + (r & 1);
          P[(t * kCh + ci) * kCh + co] = acc[i][mt][nt][r];
        }
  }
  sdb[warp][threadIdx.x & 31] = db;
  __syncthreads();
  if (threadIdx.x < kCh) {
    float s = 0.f;
    for (int w = 0; w < kWgThreads / 32; ++w) s += sdb[w][threadIdx.x];
    P[kTaps * kCh * kCh + threadIdx.x] = s;
  }
}

// Sums `nparts` partials of `count` floats (stride `stride`) in partial order.
__global__ void k_reduce_parts(const float* __restrict__ part, int nparts, int stride, int count, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  double s = 0.0;
  for (int c = 0; c < nparts; ++c) s += part[(size_t)c * stride + i];
  out[i] = (float)s;
}

__device__ __forceinline__ void voxel_xyz(const Geo& g, int64_t v, int& x, int& y, int& z) {
  x = (int)(v % g.gx);
  y = (int)((v / g.gx) % g.gy);
  z = (int)(v / ((int64_t)g.gx * g.gy));
}
__device__ __forceinline__ bool nb_of(const Geo& g, int x, int y, int z, int t, int sgn, int64_t& nb) {
  const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
  const int xx = x + sgn * dx, yy = y + sgn * dy, zz = z + sgn * dz;
  if ((unsigned)xx >= (unsigned)g.gx || (unsigned)yy >= (unsigned)g.gy || (unsigned)zz >= (unsigned)g.gz) return false;
  nb = ((int64_t)zz * g.gy + yy) * g.gx + xx;
  return true;
}

// ---------------------------------------------------------------- input layer 2 -> 32
__global__ void __launch_bounds__(256) k_l1_fwd(Geo g, int batch, const __nv_bfloat162* __restrict__ u,
                                                const float* __restrict__ w0, const float* __restrict__ b0,
                                                bf16* __restrict__ out, const int* gate) {
  if (gated(gate)) return;
  __shared__ float sw[kTaps * kCin * kCh];
  __shared__ float sbv[kCh];
  for (int i = threadIdx.x; i < kTaps * kCin * kCh; i += blockDim.x) sw[i] = w0[i];
  if (threadIdx.x < kCh) sbv[threadIdx.x] = b0[threadIdx.x];
  __syncthreads();
  const int64_t V = g.V();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * batch) return;
  const int64_t b = i / V, v = i - b * V;
  int x, y, z;
  voxel_xyz(g, v, x, y, z);
  float acc[kCh];
#pragma unroll
  for (int c = 0; c < kCh; ++c) acc[c] = sbv[c];
  for (int t = 0; t < kTaps; ++t) {
    int64_t nb;
    if (!nb_of(g, x, y, z, t, 1, nb)) continue;
    const float2 uv = __bfloat1622float2(u[b * V + nb]);
#pragma unroll
    for (int c = 0; c < kCh; ++c) {
      acc[c] = fmaf(uv.x, sw[(t * kCin + 0) * kCh + c], acc[c]);
      acc[c] = fmaf(uv.y, sw[(t * kCin + 1) * kCh + c], acc[c]);
    }
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      __nv_bfloat162 p = __floats2bfloat162_rn(fmaxf(acc[k * 8 + j * 2], 0.f), fmaxf(acc[k * 8 + j * 2 + 1], 0.f));
      w[j] = *reinterpret_cast<uint32_t*>(&p);
    }
    *reinterpret_cast<uint4*>(out + aoff(b, v, k * 8, V)) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// The 32 channels of voxel v of sample b (chunk-planar layout).
__device__ __forceinline__ void unpack32(const bf16* act, int64_t b, int64_t v, int64_t V, float (&a)[kCh]) {
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const uint4 q = *reinterpret_cast<const uint4*>(act + aoff(b, v, k * 8, V));
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[j]));
      a[k * 8 + j * 2] = f.x;
      a[k * 8 + j * 2 + 1] = f.y;
    }
  }
}

// ---------------------------------------------------------------- output layer 32 -> 1
__global__ void __launch_bounds__(256) k_l6_fwd(Geo g, int batch, const bf16* __restrict__ a5,
                                                const float* __restrict__ w5, const float* __restrict__ b5,
                                                float* __restrict__ y, const int* gate) {
  if (gated(gate)) return;
  __shared__ float sw[kTaps * kCh];
  for (int i = threadIdx.x; i < kTaps * kCh; i += blockDim.x) sw[i] = w5[i];
  __syncthreads();
  const int64_t V = g.V();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * batch) return;
  const int64_t b = i / V, v = i - b * V;
  int x, yy, z;
  voxel_xyz(g, v, x, yy, z);
  float acc = b5[0];
  for (int t = 0; t < kTaps; ++t) {
    int64_t nb;
    if (!nb_of(g, x, yy, z, t, 1, nb)) continue;
    float a[kCh];
    unpack32(a5, b, nb, V, a);
#pragma unroll
    for (int c = 0; c < kCh; ++c) acc = fmaf(a[c], sw[t * kCh + c], acc);
  }
  y[i] = acc;
}

// g5[u][ci] = (sum_t W5[t][ci] gy[u - d_t]) where a5[u][ci] > 0
__global__ void __launch_bounds__(256) k_l6_dgrad(Geo g, int batch, const float* __restrict__ gy,
                                                  const float* __restrict__ w5, const bf16* __restrict__ a5,
                                                  bf16* __restrict__ g5) {
  __shared__ float sw[kTaps * kCh];
  for (int i = threadIdx.x; i < kTaps * kCh; i += blockDim.x) sw[i] = w5[i];
  __syncthreads();
  const int64_t V = g.V();
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V * batch) return;
  const int64_t b = i / V, v = i - b * V;
  int x, y, z;
  voxel_xyz(g, v, x, y, z);
  float acc[kCh];
#pragma unroll
  for (int c = 0; c < kCh; ++c) acc[c] = 0.f;
  for (int t = 0; t < kTaps; ++t) {
    int64_t nb;
    if (!nb_of(g, x, y, z, t, -1, nb)) continue;
    const float gv = gy[b * V + nb];
#pragma unroll
    for (int c = 0; c < kCh; ++c) acc[c] = fmaf(sw[t * kCh + c], gv, acc[c]);
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int64_t off = aoff(b, v, k * 8, V);
    const uint4 mk = *reinterpret_cast<const uint4*>(a5 + off);
    const uint32_t mw[4] = {mk.x, mk.y, mk.z, mk.w};
    uint32_t w[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      __nv_bfloat162 p = __floats2bfloat162_rn(acc[k * 8 + j * 2], acc[k * 8 + j * 2 + 1]);
      w[j] = mask_pairs(*reinterpret_cast<uint32_t*>(&p), mw[j]);
    }
    *reinterpret_cast<uint4*>(g5 + off) = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// part[blk] = (dW5[t][ci] = sum_v a5[v + d_t][ci] gy[v],  db5 = sum_v gy[v]) over a
// contiguous range of voxels.  Thread (w, ci) owns taps w, w + 9, w + 18.
__global__ void __launch_bounds__(kWgThreads) k_wgrad_l6(Geo g, int batch, const bf16* __restrict__ a5,
                                                         const float* __restrict__ gy, float* __restrict__ part) {
  const int64_t V = g.V(), M = V * batch;
  const int64_t per = (M + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(M, i0 + per);
  const int ci = threadIdx.x & 31, w = threadIdx.x >> 5;
  float acc[3] = {0.f, 0.f, 0.f};
  float db = 0.f;
  for (int64_t i = i0; i < i1; ++i) {
    const int64_t b = i / V, v = i - b * V;
    int x, y, z;
    voxel_xyz(g, v, x, y, z);
    const float gv = gy[i];
    db += gv;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      int64_t nb;
      if (nb_of(g, x, y, z, w + 9 * k, 1, nb)) acc[k] = fmaf(__bfloat162float(a5[aoff(b, nb, ci, V)]), gv, acc[k]);
    }
  }
  float* P = part + (size_t)blockIdx.x * kL6Part;
#pragma unroll
  for (int k = 0; k < 3; ++k) P[(w + 9 * k) * kCh + ci] = acc[k];
  if (threadIdx.x == 0) P[kTaps * kCh] = db;
}

// part[blk] = (dW0[t][ci][co] = sum_v u[v + d_t][ci] g1[v][co],  db0[co] = sum_v g1[v][co]).
__global__ void __launch_bounds__(kWgThreads) k_wgrad_l1(Geo g, int batch, const __nv_bfloat162* __restrict__ u,
                                                         const bf16* __restrict__ g1, float* __restrict__ part) {
  const int64_t V = g.V(), M = V * batch;
  const int64_t per = (M + gridDim.x - 1) / gridDim.x;
  const int64_t i0 = (int64_t)blockIdx.x * per, i1 = min(M, i0 + per);
  const int co = threadIdx.x & 31, w = threadIdx.x >> 5;
  float acc[3][2] = {{0.f, 0.f}, {0.f, 0.f}, {0.f, 0.f}};
  float db = 0.f;
  for (int64_t i = i0; i < i1; ++i) {
    const int64_t b = i / V, v = i - b * V;
    int x, y, z;
    voxel_xyz(g, v, x, y, z);
    const float gv = __bfloat162float(g1[aoff(b, v, co, V)]);
    db += gv;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      int64_t nb;
      if (nb_of(g, x, y, z, w + 9 * k, 1, nb)) {
        const float2 uv = __bfloat1622float2(u[b * V + nb]);
        acc[k][0] = fmaf(uv.x, gv, acc[k][0]);
        acc[k][1] = fmaf(uv.y, gv, acc[k][1]);
      }
    }
  }
  float* P = part + (size_t)blockIdx.x * kL1Part;
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int c = 0; c < 2; ++c) P[((w + 9 * k) * kCin + c) * kCh + co] = acc[k][c];
  if (w == 0) P[kTaps * kCin * kCh + co] = db;
}

// gy = (y - s t) / M and per-block sums of (y - s t)^2 (fixed grid: deterministic).
__global__ void __launch_bounds__(256) k_loss(int64_t M, const float* __restrict__ y, const float* __restrict__ tgt,
                                              float s, float invM, float* __restrict__ gy, double* __restrict__ part) {
  __shared__ double red[256 / 32];
  double acc = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < M; i += (int64_t)gridDim.x * blockDim.x) {
    const float d = y[i] - s * tgt[i];
    gy[i] = d * invM;
    acc += (double)d * d;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s2 = 0.0;
    for (int w = 0; w < 256 / 32; ++w) s2 += red[w];
    part[blockIdx.x] = s2;
  }
}
__global__ void k_loss_final(const double* __restrict__ part, int n, double half_invM, double* __restrict__ loss) {
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += part[i];
  *loss = s * half_invM;
}

__global__ void k_adam(int64_t n, float* __restrict__ p, const float* __restrict__ gr, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float c1, float c2, float eps) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = gr[i];
  const float mi = b1 * m[i] + (1.f - b1) * g;
  const float vi = b2 * v[i] + (1.f - b2) * g * g;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / c1, vh = vi / c2;
  p[i] = p[i] - lr * mh / (sqrtf(vh) + eps);
}

struct PackPtrs {
  bf16* fwd[4];
  bf16* bwd[4];
};
__global__ void k_pack(const float* __restrict__ master, float* __restrict__ w0, float* __restrict__ w5, PackPtrs pp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kTaps * kCin * kCh) w0[i] = __bfloat162float(__float2bfloat16_rn(master[layer_off(0) + i]));
  if (i < kTaps * kCh) w5[i] = __bfloat162float(__float2bfloat16_rn(master[layer_off(5) + i]));
  if (i < 4 * kTaps * kCh * kCh) {
    const int l = i / (kTaps * kCh * kCh), r = i % (kTaps * kCh * kCh);
    const int t = r / (kCh * kCh), ci = (r / kCh) % kCh, co = r % kCh;
    const bf16 w = __float2bfloat16_rn(master[layer_off(l + 1) + r]);
    pp.fwd[l][(t * kCh + co) * kCh + ci] = w;
    pp.bwd[l][((kTaps - 1 - t) * kCh + ci) * kCh + co] = w;
  }
}

// ---------------------------------------------------------------- coarse-grid transfer
__global__ void __launch_bounds__(256) k_prep(int64_t V, const float* __restrict__ tc, const float* __restrict__ dhat,
                                              const float* __restrict__ scal, __nv_bfloat162* __restrict__ u,
                                              const int* gate) {
  if (gated(gate)) return;
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= V) return;
  u[i] = __floats2bfloat162_rn(tc[i] * scal[0], dhat[i]);
}

__global__ void k_to_bf16(size_t n, const float* __restrict__ in, bf16* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

__global__ void k_scale_by(int64_t n, const float* __restrict__ in, const float* __restrict__ scal,
                           float* __restrict__ out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[i] * scal[0];
}

__global__ void __launch_bounds__(256)
    k_coarse_logdiag(int nx, int ny, int nz, int c, const int* __restrict__ rowptr, const int* __restrict__ col,
                     const double* __restrict__ val, int rbase, int cbase, float* __restrict__ out) {
  const int gx = nx / c, gy = ny / c, gz = nz / c;
  const int64_t V = (int64_t)gx * gy * gz;
  const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= V) return;
  const int cx = (int)(v % gx), cy = (int)((v / gx) % gy), cz = (int)(v / ((int64_t)gx * gy));
  double s = 0.0;
  for (int k = 0; k < c; ++k)
    for (int j = 0; j < c; ++j)
      for (int i = 0; i < c; ++i) {
        const int64_t r = ((int64_t)(cz * c + k) * ny + (cy * c + j)) * nx + (int64_t)cx * c + i;
        double d = 0.0;
        for (int e = rowptr[r] - rbase; e < rowptr[r + 1] - rbase; ++e)
          if (col[e] - cbase == r) d = val[e];
        s += log(fmax(fabs(d), 1e-300));
      }
  out[v] = (float)(s / ((double)c * c * c));
}

inline int blocks_for(int64_t n, int t = 256) { return (int)std::max<int64_t>(1, (n + t - 1) / t); }

}  // namespace

// ================================================================ host side
void Net::init(uint64_t seed) {
  std::vector<float> h((size_t)kNumParams, 0.f);
  std::mt19937_64 rng(seed);
  std::normal_distribution<double> nd(0.0, 1.0);
  for (int l = 0; l < kLayers; ++l) {
    const int ci = l == 0 ? kCin : kCh;
    const double sd = std::sqrt(2.0 / (kTaps * ci));
    float* W = h.data() + layer_off(l);
    for (int64_t i = 0; i < layer_w(l); ++i) W[i] = (float)(nd(rng) * sd);
  }
  err.alloc(sizeof(int));
  master.alloc(sizeof(float) * kNumParams);
  grad.alloc(sizeof(float) * kNumParams);
  adam_m.alloc(sizeof(float) * kNumParams);
  adam_v.alloc(sizeof(float) * kNumParams);
  h2d(master.p, h.data(), sizeof(float) * kNumParams);
  cudaStream_t st = stream();
  PB_CUDA(cudaMemsetAsync(adam_m.p, 0, sizeof(float) * kNumParams, st));
  PB_CUDA(cudaMemsetAsync(adam_v.p, 0, sizeof(float) * kNumParams, st));
  PB_CUDA(cudaMemsetAsync(grad.p, 0, sizeof(float) * kNumParams, st));
  adam_t = 0;
  pk.w0.alloc(sizeof(float) * kTaps * kCin * kCh);
  pk.w5.alloc(sizeof(float) * kTaps * kCh);
  for (int l = 0; l < 4; ++l) {
    pk.fwd[l].alloc(sizeof(bf16) * kTaps * kCh * kCh);
    pk.bwd[l].alloc(sizeof(bf16) * kTaps * kCh * kCh);
  }
  repack(st);
}

void Net::repack(cudaStream_t st) {
  PackPtrs pp;
  for (int l = 0; l < 4; ++l) {
    pp.fwd[l] = dp<bf16>(pk.fwd[l]);
    pp.bwd[l] = dp<bf16>(pk.bwd[l]);
  }
  k_pack<<<blocks_for(4 * kTaps * kCh * kCh), 256, 0, st>>>(dp<float>(master), dp<float>(pk.w0), dp<float>(pk.w5), pp);
  PB_CUDA(cudaGetLastError());
}

void Acts::ensure(const Geo& gg, int b, bool training) {
  const bool same = gg.gx == g.gx && gg.gy == g.gy && gg.gz == g.gz && b <= cap;
  if (same && (!training || gy.p)) {
    batch = b;
    return;
  }
  g = gg;
  batch = b;
  cap = b;
  const size_t M = (size_t)g.V() * b;
  u.alloc(sizeof(__nv_bfloat162) * M);
  for (int l = 0; l < 5; ++l) a[l].alloc(sizeof(bf16) * kCh * M);
  y.alloc(sizeof(float) * M);
  if (training) {
    gA.alloc(sizeof(bf16) * kCh * M);
    gB.alloc(sizeof(bf16) * kCh * M);
    gy.alloc(sizeof(float) * M);
    const Tiles T = tiles_of(g, b);
    const int nwg = (int)std::min<int64_t>(T.total, num_sms());
    const size_t pf = std::max<size_t>((size_t)nwg * kWgPart, (size_t)2 * num_sms() * kL1Part);
    part.alloc(sizeof(float) * pf);
    lossp.alloc(sizeof(double) * red_blocks());
  }
}

static void set_smem_attrs() {
  static bool done = false;   // attributes are per device function; one device per process
  if (done) return;
  PB_CUDA(cudaFuncSetAttribute(k_wgrad32, cudaFuncAttributeMaxDynamicSharedMemorySize, kWgSmem));
  PB_CUDA(cudaFuncSetAttribute(k_conv32_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
  PB_CUDA(cudaFuncSetAttribute(k_conv32_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTcSmem));
  done = true;
}

// Tensor map over the chunk-planar BF16 activations, dims {8 channels, gx, gy, gz,
// 4 B planes}, with the brick box {8, 32, 6, 4, 1}: each box row is 16 bytes of one voxel
// and the 32 voxels of a line are contiguous (512 bytes).  Base and strides are multiples
// of 16 bytes.
static CUtensorMap act_map(const bf16* base, const Geo& g, int batch) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    PB_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", reinterpret_cast<void**>(&encode), cudaEnableDefault, &q));
    PB_CHECK(q == cudaDriverEntryPointSuccess && encode, PARCEL_B_E_CUDA, "cuTensorMapEncodeTiled not available");
  }
  CUtensorMap m;
  const cuuint64_t dims[5] = {8, (cuuint64_t)g.gx, (cuuint64_t)g.gy, (cuuint64_t)g.gz, (cuuint64_t)batch * 4};
  const cuuint64_t strides[4] = {16, (cuuint64_t)g.gx * 16, (cuuint64_t)g.gx * g.gy * 16, (cuuint64_t)g.V() * 16};
  const cuuint32_t box[5] = {8, (cuuint32_t)TX, (cuuint32_t)kTcLinesY, (cuuint32_t)kTcLinesZ, 1};
  const cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = encode(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<bf16*>(base), dims, strides, box, es,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  PB_CHECK(r == CUDA_SUCCESS, PARCEL_B_E_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return m;
}

static int tc_grid(const Geo& g, int batch) {   // one CTA per SM (203 KB of shared memory)
  const Tiles T = tiles_of(g, batch);
  return (int)std::min<int64_t>(T.total, (int64_t)num_sms());
}

void init_kernels() { set_smem_attrs(); }

void to_bf16(size_t n, const float* in, __nv_bfloat16* out, cudaStream_t st) {
  k_to_bf16<<<blocks_for((int64_t)n), 256, 0, st>>>(n, in, out);
  PB_CUDA(cudaGetLastError());
}

void scale_by(int64_t n, const float* in, const float* scal, float* out, cudaStream_t st) {
  k_scale_by<<<blocks_for(n), 256, 0, st>>>(n, in, scal, out);
  PB_CUDA(cudaGetLastError());
}

void forward(const Net& net, Acts& A, const int* gate, cudaStream_t st) {
  set_smem_attrs();
  const Geo& g = A.g;
  const int64_t M = g.V() * A.batch;
  const float* mp = dp<float>(net.master);
  k_l1_fwd<<<blocks_for(M), 256, 0, st>>>(g, A.batch, dp<__nv_bfloat162>(A.u), dp<float>(net.pk.w0),
                                          mp + layer_off(0) + layer_w(0), dp<bf16>(A.a[0]), gate);
  const int tg = tc_grid(g, A.batch);
  for (int l = 1; l <= 4; ++l)
    k_conv32_tc<false><<<tg, kTcThreads, kTcSmem, st>>>(act_map(dp<bf16>(A.a[l - 1]), g, A.batch), g, A.batch,
                                                        dp<bf16>(net.pk.fwd[l - 1]),
                                                        mp + layer_off(l) + layer_w(l), nullptr, dp<bf16>(A.a[l]),
                                                        dp<int>(net.err), gate);
  k_l6_fwd<<<blocks_for(M), 256, 0, st>>>(g, A.batch, dp<bf16>(A.a[4]), dp<float>(net.pk.w5),
                                          mp + layer_off(5) + layer_w(5), dp<float>(A.y), gate);
  PB_CUDA(cudaGetLastError());
}

void loss_grad(Net& net, Acts& A, const float* target, float target_scale, double* loss_dev, cudaStream_t st) {
  forward(net, A, nullptr, st);   // also sets the kernels' shared-memory limits
  const Geo& g = A.g;
  const int64_t M = g.V() * A.batch;
  const int rb = red_blocks();
  k_loss<<<rb, 256, 0, st>>>(M, dp<float>(A.y), target, target_scale, (float)(1.0 / (double)M), dp<float>(A.gy),
                             dp<double>(A.lossp));
  k_loss_final<<<1, 32, 0, st>>>(dp<double>(A.lossp), rb, 0.5 / (double)M, loss_dev);
  float* gr = dp<float>(net.grad);
  float* part = dp<float>(A.part);
  const int nsm = num_sms();
  // output layer
  k_wgrad_l6<<<2 * nsm, kWgThreads, 0, st>>>(g, A.batch, dp<bf16>(A.a[4]), dp<float>(A.gy), part);
  k_reduce_parts<<<blocks_for(kL6Part), 256, 0, st>>>(part, 2 * nsm, kL6Part, kL6Part, gr + layer_off(5));
  k_l6_dgrad<<<blocks_for(M), 256, 0, st>>>(g, A.batch, dp<float>(A.gy), dp<float>(net.pk.w5), dp<bf16>(A.a[4]),
                                            dp<bf16>(A.gA));
  // hidden layers, last to first
  bf16* gcur = dp<bf16>(A.gA);
  bf16* gnext = dp<bf16>(A.gB);
  const Tiles T = tiles_of(g, A.batch);
  const int nwg = (int)std::min<int64_t>(T.total, nsm);
  const int tg = tc_grid(g, A.batch);
  for (int l = 4; l >= 1; --l) {
    k_wgrad32<<<nwg, kWgThreads, kWgSmem, st>>>(g, A.batch, dp<bf16>(A.a[l - 1]), gcur, part);
    k_reduce_parts<<<blocks_for(kWgPart), 256, 0, st>>>(part, nwg, kWgPart, kWgPart, gr + layer_off(l));
    k_conv32_tc<true><<<tg, kTcThreads, kTcSmem, st>>>(act_map(gcur, g, A.batch), g, A.batch, dp<bf16>(net.pk.bwd[l - 1]),
                                                       nullptr,
                                                       dp<bf16>(A.a[l - 1]), gnext, dp<int>(net.err), nullptr);
    std::swap(gcur, gnext);
  }
  // input layer
  k_wgrad_l1<<<2 * nsm, kWgThreads, 0, st>>>(g, A.batch, dp<__nv_bfloat162>(A.u), gcur, part);
  k_reduce_parts<<<blocks_for(kL1Part), 256, 0, st>>>(part, 2 * nsm, kL1Part, kL1Part, gr + layer_off(0));
  PB_CUDA(cudaGetLastError());
}

void adam(Net& net, float lr, cudaStream_t st) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  net.adam_t += 1;
  const float c1 = (float)(1.0 - std::pow(0.9, net.adam_t));
  const float c2 = (float)(1.0 - std::pow(0.999, net.adam_t));
  k_adam<<<blocks_for(kNumParams), 256, 0, st>>>(kNumParams, dp<float>(net.master), dp<float>(net.grad),
                                                 dp<float>(net.adam_m), dp<float>(net.adam_v), lr, b1, b2, c1, c2, eps);
  PB_CUDA(cudaGetLastError());
  net.repack(st);
}

void prep_input(const Geo& g, const float* tc, const float* dhat, const float* scal, __nv_bfloat16* u,
                const int* gate, cudaStream_t st) {
  k_prep<<<blocks_for(g.V()), 256, 0, st>>>(g.V(), tc, dhat, scal, reinterpret_cast<__nv_bfloat162*>(u), gate);
  PB_CUDA(cudaGetLastError());
}

void coarse_log_diag(int nx, int ny, int nz, int c, const int* rowptr, const int* col, const double* val,
                     int cbase, float* out, cudaStream_t st) {
  const int64_t V = (int64_t)(nx / c) * (ny / c) * (nz / c);
  k_coarse_logdiag<<<blocks_for(V), 256, 0, st>>>(nx, ny, nz, c, rowptr, col, val, 1, cbase, out);
  PB_CUDA(cudaGetLastError());
}

}  // namespace cnn
}  // namespace pb
