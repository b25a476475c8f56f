// pb_common.cuh -- shared declarations of libparcelb (B200 / sm_100a).
//
// Library-internal header: device buffers, error handling, the persistent context that
// PARCEL_Init/PARCEL_Free manage (src/c_krylov_wrapper.f90:6-23 in the reference), the
// deterministic-reduction workspace and the device-side solver state.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/parcel_b.h"

namespace pb {

// ------------------------------------------------------------------ errors
struct Error {
  int code;
  std::string msg;
};

void set_last_error(int code, const char* fmt, ...);

#define PB_CUDA(call)                                                             \
  do {                                                                            \
    cudaError_t e__ = (call);                                                     \
    if (e__ != cudaSuccess) {                                                     \
      ::pb::set_last_error(PARCEL_B_E_CUDA, "%s:%d %s: %s", __FILE__, __LINE__,   \
                           #call, cudaGetErrorString(e__));                       \
      throw ::pb::Error{PARCEL_B_E_CUDA, cudaGetErrorString(e__)};                \
    }                                                                             \
  } while (0)

#define PB_CHECK(cond, code, ...)                                                 \
  do {                                                                            \
    if (!(cond)) {                                                                \
      ::pb::set_last_error((code), __VA_ARGS__);                                  \
      throw ::pb::Error{(code), "check failed: " #cond};                          \
    }                                                                             \
  } while (0)

// ------------------------------------------------------------------ buffers
// Owning device buffer.  Allocation goes through the context's cache so that repeated
// solves of the same size reuse memory instead of calling cudaMalloc every time.
struct DBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DBuf() = default;
  explicit DBuf(size_t b) { alloc(b); }
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
  DBuf& operator=(DBuf&& o) noexcept {
    if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
    return *this;
  }
  ~DBuf() { release(); }
  void alloc(size_t b);    // zero-filled on the library stream; bytes may be rounded up
  void zero_fill();
  void release();          // returns the buffer to the library's cache
};

// Frees every cached buffer (after draining the library stream).
void release_buffer_cache();
// Page-locked host staging area of at least `bytes`, kept between calls (one user at a
// time: the set-up of one system).
void* pinned_staging(size_t bytes);

// Set-up tracing: with PARCEL_B_TRACE=1 in the environment, trace_mark(label) drains the
// library stream and prints the wall time since the previous mark to stderr.  Off by
// default (no synchronisation is added then).
bool trace_on();
void trace_mark(const char* label);

template <class T> inline T* dp(const DBuf& b) { return reinterpret_cast<T*>(b.p); }

// ------------------------------------------------------------------ launch shapes
constexpr int kRedThreads = 256;     // threads of every reduction kernel
int num_sms();
int red_blocks();                    // fixed grid of the deterministic reductions

// Deterministic multi-value reduction workspace: every reduction kernel writes one
// partial per block and value, the last block to finish (ticket) sums them in block
// order.  One workspace per solve; kernels on one stream never overlap.
constexpr int kMaxRed = 128;
struct RedWs {
  double* part = nullptr;            // red_blocks() * kMaxRed
  unsigned* ticket = nullptr;        // 1 counter, reset by the last block
};

// ------------------------------------------------------------------ device solver state
// Scalars that the reference keeps on the host (pcg.f90:224-892 etc.) live on the device
// so that no iteration needs a host round trip; the host reads `done` once per chunk.
struct KState {
  double bnorm, rnorm, rnorm0;
  double rho0, rho1, gamma, alpha, beta;   // CG
  double c1, c2, c3, ev, vv;               // BiCGStab
  double tmp[4];
  int itr;                                 // reference iteration counter (1-based)
  int inner;                               // GMRES inner index
  int done;                                // 1 once the reference loop has exited
  int niter;
  int iret;
  int diverged;
  int breakdown;
  int mm;                                  // GMRES columns used in the last cycle
  int skip_inner;                          // GMRES: inner loop has exited this cycle
  int stop_after_update;                   // GMRES: exit the solve after update_xVec
  int last_inner;                          // GMRES: Fortran `inner` after the last cycle
  int pad[5];
  __host__ __device__ int mm_prev_inner() const { return last_inner; }
};

// ------------------------------------------------------------------ context
struct Context {
  int device = -1;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  bool initialised = false;
};

Context& ctx();
void ensure_init();
cudaStream_t stream();

// Copy helpers on the library stream.
void h2d(void* dst, const void* src, size_t bytes);
void d2h(void* dst, const void* src, size_t bytes);
void d2d(void* dst, const void* src, size_t bytes);
void sync();

bool is_device_ptr(const void* p);

}  // namespace pb
