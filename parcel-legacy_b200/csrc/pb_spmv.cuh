// pb_spmv.cuh -- CRS sparse matrix-vector product (pb_spmv.cu).
#pragma once

#include "pb_device.cuh"
#include "pb_ilu.cuh"

namespace pb {

enum SpmvMode : int {
  SPMV_Y = 0,       // y = A x
  SPMV_RES = 1,     // y = b - A x
};

// Lanes of a warp cooperating on one row, chosen from the mean row length.
int spmv_lanes(int n, int64_t nnz);

// y = A x (or b - A x), optionally fused with one or two dot products reduced on the
// device: dot k multiplies y (sel 0), x (sel 1) or d (sel 2) by y / x / d.
template <class VT, class XT>
void spmv(const DevMat<VT>& A, const XT* x, XT* y, int mode, const XT* b, const int* gate,
          cudaStream_t st);
template <class VT, class XT>
void spmv_dot(const DevMat<VT>& A, const XT* x, XT* y, int mode, const XT* b, const XT* d,
              int nd, const int* sa, const int* sb, const Red& red, const int* gate,
              cudaStream_t st);

}  // namespace pb
