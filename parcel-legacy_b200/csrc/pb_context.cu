// pb_context.cu -- library context, device memory, copies and error reporting.
//
// Replaces PARCEL_Init / PARCEL_Free (src/c_krylov_wrapper.f90:6-23), which select the
// GPU (`set_GPU`, cu_common.cu:489-520) and create global cuBLAS/cuSPARSE handles.  This
// library needs no vendor handles: it selects the device, owns one stream and reports
// errors as status codes instead of exiting (cu_common.h:119-124 exits on malloc failure).
#include <cstdarg>
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

int num_sms() { ensure_init(); return g_sms; }

int red_blocks() { return 4 * num_sms(); }

void DBuf::alloc(size_t b) {
  release();
  if (b == 0) return;
  ensure_init();
  cudaError_t e = cudaMalloc(&p, b);
  if (e != cudaSuccess) {
    p = nullptr;
    (void)cudaGetLastError();
    set_last_error(PARCEL_B_E_NOMEM, "cudaMalloc(%zu) failed: %s", b, cudaGetErrorString(e));
    throw Error{PARCEL_B_E_NOMEM, "cudaMalloc failed"};
  }
  bytes = b;
}

void DBuf::release() {
  if (p) cudaFree(p);
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
    if (pb::g_ctx.own_stream && pb::g_ctx.stream && s) {
      cudaStreamSynchronize(pb::g_ctx.stream);
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
