// pb_device.cuh -- device-side helpers shared by the kernels of libparcelb:
// deterministic block reductions, mbarrier / bulk-copy (TMA) wrappers, double-double
// arithmetic and the solver epilogues run by the last block of a reduction.
#pragma once

#include "pb_common.cuh"

namespace pb {

constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------------ epilogue arguments
// Passed by value to every reduction kernel.  `epi` selects what the last block does
// with the reduced sums (see epilogue() in pb_blas.cu).
struct EpiArgs {
  KState* st = nullptr;
  double* hist = nullptr;    // reshistory, itrmax entries (device)
  double* h = nullptr;       // GMRES Hessenberg, (m+1) x m column major
  double* e = nullptr;       // GMRES rhs of the least-squares problem, m+1
  double* cs = nullptr;
  double* sn = nullptr;
  double* out = nullptr;     // EPI_STORE destination
  int m = 0;
  int itrmax = 0;
  double rtol = 0.0;
  double abstol = 0.0;
  int k = 0, j = 0;          // MGS indices of the value being reduced
};

enum Epi : int {
  EPI_STORE = 0,     // out[0..K-1] = sums
  EPI_CG_INIT,       // <b,b>, <r,r>, <s,r>
  EPI_CG_GAMMA,      // <p,q>
  EPI_CG_DOT2,       // <s,r>, <r,r>, then the stop test
  EPI_BICG_INIT,     // <b,b>, <r,r>
  EPI_BICG_C2,       // <r0,q>
  EPI_BICG_C3,       // <e,v>, <v,v>
  EPI_BICG_END,      // <r,r0>, <r,r>, then the stop test
  EPI_GM_RESTART,    // <r,r> at the top of a restart cycle
  EPI_GM_H,          // one MGS coefficient h(k,j)
  EPI_GM_HCGS,       // j CGS coefficients h(1..j, j)
  EPI_GM_NORM,       // ||w|| = h(j+1,j), then Givens and the stop test
  EPI_NORM2,         // out[0] = sqrt(sum0)
};

struct Red {
  double* part;
  unsigned* ticket;
  EpiArgs ea;
  int epi;
};

// ------------------------------------------------------------------ gating
__device__ __forceinline__ bool gated(const int* gate) {
  return gate && *(volatile const int*)gate != 0;
}

// ------------------------------------------------------------------ mbarrier / TMA
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes) : "memory");
}
// Adds to the transaction count of the current phase without arriving.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Bounded parity wait: returns false if the barrier did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned limit) {
  uint32_t addr = smem_u32(bar);
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok) : "r"(addr), "r"(parity) : "memory");
    if (ok) return true;
  }
  return false;
}
// Bulk (non-tensor) global -> shared copy completing on an mbarrier; 16-byte aligned
// addresses, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_shared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async_global() {
  asm volatile("fence.proxy.async.global;" ::: "memory");
}
__device__ __forceinline__ void named_bar_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// ------------------------------------------------------------------ double-double
// The reference's dd arithmetic (src/dd_func.f90:5-98; macro forms ddadd.h / ddmul.h):
// "sloppy" add = two-sum of the high parts, low parts added, renormalised; mul = Dekker
// split with 134217729 = 2^27 + 1.  Every operation is an explicitly rounded intrinsic so
// the compiler can neither contract nor reassociate.
struct dd { double hi, lo; };

__device__ __forceinline__ dd dd_add(dd a, dd b) {
  double p1 = __dadd_rn(a.hi, b.hi);
  double p2 = __dsub_rn(p1, a.hi);
  double t1l = __dadd_rn(__dsub_rn(a.hi, __dsub_rn(p1, p2)), __dsub_rn(b.hi, p2));
  double t1h = p1;
  t1l = __dadd_rn(__dadd_rn(t1l, a.lo), b.lo);
  double s1 = __dadd_rn(t1h, t1l);
  t1l = __dsub_rn(t1l, __dsub_rn(s1, t1h));
  return dd{s1, t1l};
}

__device__ __forceinline__ dd dd_sub(dd a, dd b) {
  double p1 = __dsub_rn(a.hi, b.hi);
  double p2 = __dsub_rn(p1, a.hi);
  double t1l = __dsub_rn(__dsub_rn(a.hi, __dsub_rn(p1, p2)), __dadd_rn(b.hi, p2));
  double t1h = p1;
  t1l = __dsub_rn(__dadd_rn(t1l, a.lo), b.lo);
  double s1 = __dadd_rn(t1h, t1l);
  t1l = __dsub_rn(t1l, __dsub_rn(s1, t1h));
  return dd{s1, t1l};
}

__device__ __forceinline__ dd dd_mul(dd a, dd b) {
  double t1h = __dmul_rn(a.hi, b.hi);
  double u1 = __dmul_rn(134217729.0, a.hi);
  double p1 = __dsub_rn(u1, __dsub_rn(u1, a.hi));
  double p2 = __dsub_rn(a.hi, p1);
  u1 = __dmul_rn(134217729.0, b.hi);
  double r1 = __dsub_rn(u1, __dsub_rn(u1, b.hi));
  double r2 = __dsub_rn(b.hi, r1);
  double t1l = __dadd_rn(__dadd_rn(__dadd_rn(__dsub_rn(__dmul_rn(p1, r1), t1h), __dmul_rn(p1, r2)),
                                   __dmul_rn(p2, r1)),
                         __dmul_rn(p2, r2));
  t1l = __dadd_rn(t1l, __dadd_rn(__dmul_rn(a.hi, b.lo), __dmul_rn(a.lo, b.hi)));
  double s1 = __dadd_rn(t1h, t1l);
  t1l = __dsub_rn(t1l, __dsub_rn(s1, t1h));
  return dd{s1, t1l};
}

// dd_div (dd_func.f90:99-142): q1 = a.hi / b.hi, the product b * q1 formed exactly with
// the Dekker split, one correction q2 = (a - b q1) / b.hi, renormalised.
__device__ __forceinline__ dd dd_div(dd a, dd b) {
  const double q1 = __ddiv_rn(a.hi, b.hi);
  double t1h = __dmul_rn(b.hi, q1);
  double u1 = __dmul_rn(134217729.0, b.hi);
  const double p1 = __dsub_rn(u1, __dsub_rn(u1, b.hi));
  const double p2 = __dsub_rn(b.hi, p1);
  u1 = __dmul_rn(134217729.0, q1);
  double r1 = __dsub_rn(u1, __dsub_rn(u1, q1));
  const double r2 = __dsub_rn(q1, r1);
  double t1l = __dadd_rn(__dadd_rn(__dadd_rn(__dsub_rn(__dmul_rn(p1, r1), t1h), __dmul_rn(p1, r2)),
                                   __dmul_rn(p2, r1)),
                         __dmul_rn(p2, r2));
  t1l = __dadd_rn(t1l, __dmul_rn(b.lo, q1));
  double s1 = __dadd_rn(t1h, t1l);
  t1l = __dsub_rn(t1l, __dsub_rn(s1, t1h));
  t1h = s1;
  s1 = __dsub_rn(a.hi, t1h);
  r1 = __dsub_rn(s1, a.hi);
  double s2 = __dsub_rn(__dsub_rn(a.hi, __dsub_rn(s1, r1)), __dadd_rn(t1h, r1));
  s2 = __dsub_rn(s2, t1l);
  s2 = __dadd_rn(s2, a.lo);
  const double q2 = __ddiv_rn(__dadd_rn(s1, s2), b.hi);
  const double h = __dadd_rn(q1, q2);
  return dd{h, __dsub_rn(q2, __dsub_rn(h, q1))};
}

// dd_sqrt (dd_func.f90:143-239): x = 1 / sqrt(a.hi), then one correction in dd.  A zero
// argument falls through to the general formula as in the reference; a negative one gives 0.
__device__ __forceinline__ dd dd_sqrt(dd a) {
  if (a.hi < 0.0 || (a.hi == 0.0 && a.lo < 0.0)) return dd{0.0, 0.0};
  const double x = __ddiv_rn(1.0, __dsqrt_rn(a.hi));
  const double ax = __dmul_rn(a.hi, x);
  const dd y = dd_mul(dd{x, 0.0}, dd{0.5, 0.0});
  const dd z = dd_mul(dd{ax, 0.0}, dd{ax, 0.0});
  const dd t2 = dd_sub(a, z);
  const dd t1 = dd_mul(t2, y);
  return dd_add(t1, dd{ax, 0.0});
}

}  // namespace pb
