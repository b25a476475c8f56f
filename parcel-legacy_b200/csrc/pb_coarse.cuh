// pb_coarse.cuh -- Galerkin coarse-grid correction on a structured grid (pb_coarse.cu).
//
// No counterpart in the reference (PARCEL's preconditioners are one-level: point Jacobi,
// block-Jacobi ILU / D-ILU, additive Schwarz).  The preconditioner stage of the learned
// FGMRES path is additive two-level:
//
//     z = M_ILU^-1 v + P y,   y ~ A_c^-1 P^T v,   A_c = P^T A P
//
// P is the cell-centred trilinear interpolation from the coarse grid (gx, gy, gz) =
// (nx, ny, nz) / c to the fine grid (natural row = (z ny + y) nx + x), clamped at the
// boundary: along one axis fine cell i sits at u = (i + 1/2) / c - 1/2 in coarse units and
// takes weight 1 - w from coarse cell clamp(floor(u)) and w = u - floor(u) from
// clamp(floor(u) + 1).  A_c keeps the couplings of each coarse cell to its 27 neighbours
// (offsets in {-1, 0, 1}^3); the couplings two cells apart that the exact product also
// has (weights below 1/c^2 of the rest for c = 8) are dropped.  y comes from `steps`
// iterations of Jacobi-preconditioned CG on A_c, started from zero or from a guess g
// scaled by gamma = <rc, g> / <g, A_c g> (the A_c-energy-optimal multiple).
#pragma once

#include "pb_common.cuh"
#include "pb_ilu.cuh"

namespace pb {
namespace coarse {

constexpr int kTaps = 27;   // tap t = 9 (dz + 1) + 3 (dy + 1) + (dx + 1)

struct Grid {
  int nx = 0, ny = 0, nz = 0, c = 2;
  int gx = 0, gy = 0, gz = 0;
  Grid() = default;
  Grid(int nx_, int ny_, int nz_, int c_)
      : nx(nx_), ny(ny_), nz(nz_), c(c_), gx(nx_ / c_), gy(ny_ / c_), gz(nz_ / c_) {}
  __host__ __device__ int64_t Vc() const { return (int64_t)gx * gy * gz; }
  __host__ __device__ int64_t Vh() const { return (int64_t)8 * gx * gy * gz; }   // half cells
};

// Throws unless the grid suits the transfer operators (c even, dims divisible by c, at most
// 1024 cells per axis) and the coarse problem has at most max_coarse_cells() cells (49,152:
// the prolongation keeps the coarse vector in shared memory) and fits one thread-block
// cluster of the coarse solver.
void check_grid(const Grid& g);
int64_t max_coarse_cells();

// A_c = P^T A P as [27][Vc] FP64 (zero where the neighbour lies outside the coarse grid),
// deterministic.  A: natural CRS on the device with n = nx ny nz.
void galerkin(const Grid& g, const DevMat<double>& A, double* ac64, cudaStream_t st);
// FP32 copy of A_c and the inverse of its diagonal (0 where the diagonal is 0).
void to_f32(int64_t Vc, const double* ac64, float* ac32, float* dinv32, cudaStream_t st);

// rc = P^T v for a fine vector v in iteration layout (pos maps natural rows to iteration
// positions; NULL: natural layout).  hc: Vh() * 8 floats of scratch.
template <class T>
void restrict_fine(const Grid& g, const T* v, const int* pos, float* hc, float* rc, const int* gate,
                   cudaStream_t st);
// code[p] = x | y << 10 | z << 20 of the natural row rowAt[p] (rowAt NULL: p itself), -1
// where rowAt[p] < 0 (layout padding).
void pack_coords(const Grid& g, int64_t np, const int* rowAt, int* code, cudaStream_t st);
// z[p] += (P y)(fine cell code[p]) for p < np; code[p] < 0 is left untouched.
template <class T>
void prolong_add(const Grid& g, int64_t np, const float* y, const int* code, T* z, const int* gate,
                 cudaStream_t st);
// scal[0] = 1 / rms(v), scal[1] = rms(v) over Vc entries (0, 0 for v == 0); one CTA.
void rms(int64_t Vc, const float* v, float* scal, const int* gate, cudaStream_t st);

// `steps` Jacobi-PCG iterations on A_c y = rc, from zero (g0 NULL) or from gamma g0.  One
// thread-block cluster: coarse z-planes are split over its CTAs, the search direction is
// exchanged through distributed shared memory and the dot products are reduced in rank
// order, so the result does not depend on timing.
struct PcgArgs {
  Grid g;
  const float* ac = nullptr;     // [27][Vc]
  const float* dinv = nullptr;   // [Vc]
  const float* rc = nullptr;     // [Vc]
  const float* g0 = nullptr;     // [Vc] or NULL
  float* y = nullptr;            // [Vc]
  int steps = 0;
  const int* gate = nullptr;
};
void pcg(const PcgArgs& a, cudaStream_t st);

}  // namespace coarse
}  // namespace pb
