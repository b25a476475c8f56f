// pb_context.cu -- library context, device memory, copies and error reporting.
//
// Replaces PARCEL_Init / PARCEL_Free (src/c_krylov_wrapper.f90:6-23), which select the
// GPU (`set_GPU`, cu_common.cu:489-520) and create global cuBLAS/cuSPARSE handles.  This
// library needs no vendor handles: it selects the device, owns one stream and reports
// errors as status codes instead of exiting (cu_common.h:119-124 exits on malloc failure).
#include <chrono>
#include <cstdarg>
#include <cstdlib>
#include <map>
#include <mutex>

#include "pb_common.cuh"

namespace pb {

namespace {
thread_local int g_last_code = 0;
thread_local char g_last_msg[512] = {0};
Context g_ctx;
std::mutex g_mu;
int g_sms = 0;
}  // namespace

void set_last_error(int code, const char* fmt, ...) {
  g_last_code = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_msg, sizeof(g_last_msg), fmt, ap);
  va_end(ap);
}

Context& ctx() { return g_ctx; }

void ensure_init() {
  std::lock_guard<std::mutex> lk(g_mu);
  if (g_ctx.initialised) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) {
    set_last_error(PARCEL_B_E_CUDA, "no CUDA device: %s", cudaGetErrorString(e));
    throw Error{PARCEL_B_E_CUDA, "no CUDA device"};
  }
  PB_CUDA(cudaSetDevice(dev));
  g_ctx.device = dev;
  if (!g_ctx.stream) {
    PB_CUDA(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking));
    g_ctx.own_stream = true;
  }
  cudaDeviceProp prop;
  PB_CUDA(cudaGetDeviceProperties(&prop, dev));
  g_sms = prop.multiProcessorCount;
  g_ctx.initialised = true;
}

cudaStream_t stream() { ensure_init(); return g_ctx.stream; }

bool trace_on() {
  static const int on = [] {
    const char* e = getenv("PARCEL_B_TRACE");
    return (e && e[0] == '1') ? 1 : 0;
  }();
  return on != 0;
}

void trace_mark(const char* label) {
  if (!trace_on()) return;
  static double last = 0.0;
  cudaStreamSynchronize(g_ctx.stream);
  const double t = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  if (last > 0.0 && label) fprintf(stderr, "[parcel_b] %-28s %9.3f ms\n", label, (t - last) * 1e3);
  last = t;
}

int num_sms() { ensure_init(); return g_sms; }

int red_blocks() { return 4 * num_sms(); }

// ------------------------------------------------------------------ buffer cache
// Released buffers are kept, keyed by their rounded size, and handed to the next request
// of that size: a solve repeated on the same problem allocates nothing after the first,
// and no cudaFree (which waits for the whole device) sits inside a solve.  Reuse is safe
// because every kernel, copy and memset of the library runs on the one library stream,
// in order (parcel_b_set_stream drains the old stream before switching).  The cache holds
// at most kCacheMax bytes, is emptied when cudaMalloc fails (then retried) and by
// parcel_free_c_.
namespace {
std::mutex g_cache_mu;
std::multimap<size_t, void*> g_cache;
size_t g_cache_bytes = 0;
constexpr size_t kCacheMax = size_t(16) << 30;

size_t round_size(size_t b) {
  const size_t g = b < (size_t(1) << 20) ? 512 : (size_t(2) << 20);
  return (b + g - 1) / g * g;
}

void cache_trim_locked() {
  for (auto& kv : g_cache) cudaFree(kv.second);
  g_cache.clear();
  g_cache_bytes = 0;
}
}  // namespace

namespace {
void* g_pin = nullptr;
size_t g_pin_bytes = 0;
}  // namespace

void* pinned_staging(size_t bytes) {
  if (bytes > g_pin_bytes) {
    if (g_pin) cudaFreeHost(g_pin);
    g_pin = nullptr;
    g_pin_bytes = 0;
    PB_CUDA(cudaMallocHost(&g_pin, bytes));
    g_pin_bytes = bytes;
  }
  return g_pin;
}

void release_buffer_cache() {
  std::lock_guard<std::mutex> lk(g_cache_mu);
  if (g_ctx.stream) cudaStreamSynchronize(g_ctx.stream);
  cache_trim_locked();
  if (g_pin) cudaFreeHost(g_pin);
  g_pin = nullptr;
  g_pin_bytes = 0;
}

void DBuf::alloc(size_t b) {
  release();
  if (b == 0) return;
  ensure_init();
  const size_t rb = round_size(b);
  {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = g_cache.find(rb);
    if (it != g_cache.end()) {
      p = it->second;
      g_cache.erase(it);
      g_cache_bytes -= rb;
    }
  }
  if (p) {
    bytes = rb;
    zero_fill();
    return;
  }
  cudaError_t e = cudaMalloc(&p, rb);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    {
      std::lock_guard<std::mutex> lk(g_cache_mu);
      if (g_ctx.stream) cudaStreamSynchronize(g_ctx.stream);
      cache_trim_locked();
    }
    e = cudaMalloc(&p, rb);
  }
  if (e != cudaSuccess) {
    p = nullptr;
    (void)cudaGetLastError();
    set_last_error(PARCEL_B_E_NOMEM, "cudaMalloc(%zu) failed: %s", rb, cudaGetErrorString(e));
    throw Error{PARCEL_B_E_NOMEM, "cudaMalloc failed"};
  }
  bytes = rb;
  zero_fill();
}

// Every buffer starts zeroed (stream-ordered): layout padding positions that no kernel
// writes (rows of the iteration layout that belong to no matrix row) must hold zeros, not
// a previous solve's values.
void DBuf::zero_fill() {
  cudaError_t e = cudaMemsetAsync(p, 0, bytes, g_ctx.stream);
  if (e != cudaSuccess) {
    set_last_error(PARCEL_B_E_CUDA, "cudaMemsetAsync: %s", cudaGetErrorString(e));
    throw Error{PARCEL_B_E_CUDA, "cudaMemsetAsync failed"};
  }
}

void DBuf::release() {
  if (p) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    if (g_cache_bytes + bytes <= kCacheMax) {
      g_cache.emplace(bytes, p);
      g_cache_bytes += bytes;
    } else {
      cudaFree(p);
    }
  }
  p = nullptr;
  bytes = 0;
}

void h2d(void* dst, const void* src, size_t bytes) {
  if (bytes) PB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream()));
}
void d2h(void* dst, const void* src, size_t bytes) {
  if (bytes) PB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream()));
  PB_CUDA(cudaStreamSynchronize(stream()));
}
void d2d(void* dst, const void* src, size_t bytes) {
  if (bytes) PB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, stream()));
}
void sync() { PB_CUDA(cudaStreamSynchronize(stream())); }

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  cudaError_t e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) { (void)cudaGetLastError(); return false; }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace pb

extern "C" {

void parcel_init_c_(int* myrank) {
  (void)myrank;   // one process per GPU: the caller's rank picks no device here
  try { pb::ensure_init(); } catch (...) {}
}

void parcel_free_c_(void) {
  pb::release_buffer_cache();
  std::lock_guard<std::mutex> lk(pb::g_mu);
  if (pb::g_ctx.initialised && pb::g_ctx.own_stream && pb::g_ctx.stream) {
    cudaStreamSynchronize(pb::g_ctx.stream);
    cudaStreamDestroy(pb::g_ctx.stream);
  }
  pb::g_ctx = pb::Context{};
}

int parcel_b_set_stream(void* s) {
  try {
    pb::ensure_init();
    std::lock_guard<std::mutex> lk(pb::g_mu);
    // drain the old stream: cached buffers may still be read by work queued on it
    if (pb::g_ctx.stream) cudaStreamSynchronize(pb::g_ctx.stream);
    if (pb::g_ctx.own_stream && pb::g_ctx.stream && s) {
      cudaStreamDestroy(pb::g_ctx.stream);
      pb::g_ctx.own_stream = false;
    }
    if (s) pb::g_ctx.stream = (cudaStream_t)s;
    return 0;
  } catch (const pb::Error& e) { return e.code; }
}

void* parcel_b_get_stream(void) {
  try { return (void*)pb::stream(); } catch (...) { return nullptr; }
}

int parcel_b_last_error(char* buf, int buflen) {
  if (buf && buflen > 0) {
    strncpy(buf, pb::g_last_msg, buflen - 1);
    buf[buflen - 1] = 0;
  }
  return pb::g_last_code;
}

}  // extern "C"
