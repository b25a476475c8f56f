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
  double* slots = nullptr;   // staged variant: (j+1) x num_sms() partial-sum slots and
  double* totals = nullptr;  // j+1 total slots, all preset to all-ones bytes (mgs_staged)
  int* err = nullptr;
  const int* gate = nullptr;
  Red red;                // EPI_GM_NORM epilogue arguments
};

template <class T> bool mgs_supported(int64_t np);
template <class T> void mgs_column(const MgsArgs<T>& a, cudaStream_t st);
template <class T> int mgs_grid();
// True when mgs_column runs the shared-memory-staged variant for this length; it then
// uses MgsArgs::slots (j+1 rows of num_sms() doubles) and MgsArgs::totals (j+1 doubles),
// every byte 0xFF before the launch, instead of ctr / parts.
template <class T> bool mgs_staged(int64_t np);

}  // namespace pb
