// pb_mgs.cuh -- one-launch modified Gram-Schmidt of a GMRES column (pb_mgs.cu).
#pragma once

#include "pb_device.cuh"

namespace pb {

constexpr int kMgsThreads = 256;

template <class T>
struct MgsArgs {
  int64_t np = 0;         // vector length
  int j = 0;              // column (1-based)
  T* w = nullptr;         // A M^-1 v_j (the streaming variant updates it in place)
  const T* V = nullptr;   // basis, column stride ldv
  int64_t ldv = 0;
  T* vnext = nullptr;     // v_{j+1} destination (null for the last column of a cycle)
  double* parts = nullptr;   // 2 * grid partial sums
  unsigned* ctr = nullptr;   // j+1 zeroed barrier counters
  int* err = nullptr;
  const int* gate = nullptr;
  Red red;                // EPI_GM_NORM epilogue arguments
};

template <class T> bool mgs_supported(int64_t np);
template <class T> void mgs_column(const MgsArgs<T>& a, cudaStream_t st);
template <class T> int mgs_grid();

}  // namespace pb
