// pb_cnn.cuh -- the learned coarse-grid preconditioner stage (BF16 3D CNN).
//
// No counterpart in the reference: PARCEL has no learned component.  The network works on
// the coarse grid of the two-level preconditioner stage (pb_coarse.cuh): from the coarse
// residual rc = P^T v and the coefficient channel it predicts the coarse error
// A_c^-1 rc, which starts the stage's coarse Jacobi-PCG:
//
//     y0 = Net([rc / sigma, dhat])   (6 conv layers, 3^3 taps, BF16, FP32 sums), sigma = rms(rc)
//
// dhat is the normalised coarse mean of log(diag A): the network sees the operator's
// local coefficient through the matrix itself.  Training targets are scaled by s, fixed
// from the training set (the coarse solve rescales the guess, so s needs no inverse).  Network layout: channels last, voxel v = (z gy + y) gx + x on the coarse
// grid, samples contiguous; hidden activations BF16 [V][32].
//
// Parameters (FP32 master copy, Adam state alongside): layer l = 0..5 stores
// W_l[27][C_in][C_out] (tap t = 9 (dz+1) + 3 (dy+1) + (dx+1)) followed by b_l[C_out];
// (C_in, C_out) = (2,32), (32,32) x 4, (32,1).
#pragma once

#include <cuda_bf16.h>

#include "pb_common.cuh"

namespace pb {
namespace cnn {

constexpr int kCin = 2;
constexpr int kCh = 32;
constexpr int kTaps = 27;
constexpr int kLayers = 6;

constexpr int64_t layer_w(int l) {
  return (int64_t)kTaps * (l == 0 ? kCin : kCh) * (l == kLayers - 1 ? 1 : kCh);
}
constexpr int64_t layer_b(int l) { return l == kLayers - 1 ? 1 : kCh; }
constexpr int64_t layer_off(int l) {
  int64_t o = 0;
  for (int i = 0; i < l; ++i) o += layer_w(i) + layer_b(i);
  return o;
}
constexpr int64_t kNumParams = layer_off(kLayers);   // 113,345

struct Geo {
  int gx = 0, gy = 0, gz = 0;   // coarse grid
  __host__ __device__ int64_t V() const { return (int64_t)gx * gy * gz; }
};

// Packed weights consumed by the kernels (rebuilt from the master copy after each update).
struct Packed {
  DBuf w0;        // float [27][2][32], values rounded to BF16
  DBuf w5;        // float [27][32],   values rounded to BF16
  DBuf fwd[4];    // bf16 [27][32 n=co][32 k=ci]          layers 1..4, forward
  DBuf bwd[4];    // bf16 [27][32 n=ci][32 k=co], taps mirrored: transposed convolution
};

// Network: parameters, optimiser state and kernel-side packed weights.
struct Net {
  DBuf master, grad, adam_m, adam_v;
  DBuf err;                                 // nonzero: a tensor-core wait timed out
  Packed pk;
  int adam_t = 0;
  void init(uint64_t seed);                 // He-normal weights, zero biases
  void repack(cudaStream_t st);
};

// Activation buffers for a batch of samples on grid g.
struct Acts {
  int batch = 0;   // samples of the current pass
  int cap = 0;     // samples the buffers hold
  Geo g;
  DBuf u;          // bf16 [B][V][2]
  DBuf a[5];       // bf16 [B][V][32]  (post-ReLU a1..a5)
  DBuf y;          // float [B][V]
  DBuf gA, gB;     // bf16 [B][V][32]  gradient ping-pong
  DBuf gy;         // float [B][V]
  DBuf part;       // float partial sums of the weight-gradient kernels
  DBuf lossp;      // double loss partials
  void ensure(const Geo& g, int batch, bool training);
};

// Sets the shared-memory limits of the tensor-core kernels (once; call before any stream
// capture that launches them).
void init_kernels();
// Forward pass: acts.u must hold the inputs; writes acts.a[*] and acts.y.
void forward(const Net& net, Acts& A, const int* gate, cudaStream_t st);
// Loss 1/(2M) sum (y - s*target)^2 and all parameter gradients into net.grad
// (runs forward first).  loss_dev receives the loss (device double).
void loss_grad(Net& net, Acts& A, const float* target, float target_scale, double* loss_dev,
               cudaStream_t st);
// Adam update of the master weights from net.grad, then repack.
void adam(Net& net, float lr, cudaStream_t st);

// out[i] = bf16(in[i])
void to_bf16(size_t n, const float* in, __nv_bfloat16* out, cudaStream_t st);
// out[i] = in[i] * scal[0]
void scale_by(int64_t n, const float* in, const float* scal, float* out, cudaStream_t st);
// Input preparation: u[v] = (bf16(tc[v] * scal[0]), bf16(dhat[v])) for one sample.
void prep_input(const Geo& g, const float* tc, const float* dhat, const float* scal, __nv_bfloat16* u,
                const int* gate, cudaStream_t st);

// Coarse mean of log|diag A| over c^3 blocks (natural CRS on the device, 1-based row
// pointers, column base cbase).  Host normalisation follows.
void coarse_log_diag(int nx, int ny, int nz, int c, const int* rowptr, const int* col, const double* val,
                     int cbase, float* out, cudaStream_t st);

}  // namespace cnn
}  // namespace pb
