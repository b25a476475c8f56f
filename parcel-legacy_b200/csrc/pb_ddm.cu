// pb_ddm.cu -- DDM stencil-format input: parcel_b_solve_ddm / parcel_b_ddsolve_ddm and the
// parcel_d*_ddm shims.
//
// Reference: parcel_ddm_main / parcel_ddm_main_dd (src/src_DDM/ddm_kernel.f90:463-1899) and
// their C-callable forms (src/example/c2fortran_kernel.f90:2964-3691).  A DDM matrix is one
// process's box of a structured grid, padded by `margin` cells on both sides of each axis,
// x fastest: m = prod(n_d + 2 margin) cells (set_grids_decompostion,
// src/example/ddm_setup.f90:66-125).  Stencil point k couples interior cell j with cell
// j + offset(k), value diaA(k m + j) (make_poisson_3D_DDM, ddm_setup.f90:127-345).  The
// Krylov solvers are the generic KSP_pCG / pBiCG / pGMRES / pCAGMRES over the interior
// cells.  Block Jacobi is D-ILU on boxes of the interior:
//   * CPU build: one box per OpenMP thread, the interior cut into slabs along axis
//     div_direc_th (aslu_ddm and ilu_ddm_case_{x,y,z}div, src/src_DDM/aslu_ddm.f90:8-1558;
//     the diagonal in as_ddm_init, src/src_DDM/init_ddm_mod.f90:370-642; the slabs from
//     set_region_for_threads, src/common.f90:266-303);
//   * CUDA build (DDM_CUDA_BJ): n_d / 4 boxes per axis (init_DILU_DDM / get_DILU_DDM,
//     src/src_DDM/precon_ddm_GPU.f90:2646-3097, chosen at ddm_kernel.f90:1009-1017).
// The D-ILU diagonal recurrence keeps only couplings inside the box, and the sweeps walk a
// box's cells in padded-index (lexicographic) order, dropping the other slabs' cells and
// reading zeros from the margin of their output vector.  The preconditioner is therefore
// the CRS block-Jacobi D-ILU of the matrix renumbered box by box (each box's cells in
// lexicographic order) with the boxes as the blocks, and that is how it runs here: the
// cells are renumbered once (host plan, device build of the CRS rows), and the CRS solvers
// solve the renumbered system with the boxes as explicit blocks.  The reference's stored
// DDM outputs (template_cpu/STDOUT_run_ddm: 4 processes x 20 x-slabs, 261 CG iterations;
// template_gpu/STDOUT_run_ddm: 4^3 boxes, 345) are reproduced by this construction.
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstring>
#include <memory>
#include <vector>

#include "pb_api.cuh"

namespace pb {
namespace {

constexpr int kDdmThreads = 256;
constexpr int kDdmMaxNnd = 32;

inline int ddm_grid(int64_t n) {
  return (int)std::max<int64_t>(1, std::min<int64_t>((n + kDdmThreads - 1) / kDdmThreads, 8LL * num_sms()));
}

// Box geometry: interior sizes, padded sizes and strides per axis (axes beyond ndim have one
// cell and no margin).
struct DdmGeo {
  int ndim = 3;
  int n[3] = {1, 1, 1};
  int pad[3] = {1, 1, 1};
  int mg[3] = {0, 0, 0};
  int64_t stride[3] = {1, 1, 1};
  int64_t m = 1;
  int64_t nint = 1;
};

DdmGeo ddm_geometry(const parcel_b_ddm* A) {
  PB_CHECK(A != nullptr, PARCEL_B_E_ARG, "matrix is NULL");
  PB_CHECK(A->ndim >= 1 && A->ndim <= 3, PARCEL_B_E_ARG, "ndim = %d (1..3)", A->ndim);
  PB_CHECK(A->margin >= 1, PARCEL_B_E_ARG, "margin = %d", A->margin);
  DdmGeo g;
  g.ndim = A->ndim;
  for (int d = 0; d < A->ndim; ++d) {
    PB_CHECK(A->n_grids[d] >= 1, PARCEL_B_E_ARG, "n_grids[%d] = %d", d, A->n_grids[d]);
    g.n[d] = A->n_grids[d];
    g.mg[d] = A->margin;
    g.pad[d] = A->n_grids[d] + 2 * A->margin;
  }
  g.stride[0] = 1;
  g.stride[1] = g.pad[0];
  g.stride[2] = (int64_t)g.pad[0] * g.pad[1];
  g.m = g.stride[2] * g.pad[2];
  g.nint = (int64_t)g.n[0] * g.n[1] * g.n[2];
  PB_CHECK(A->m == g.m, PARCEL_B_E_ARG, "m = %lld, the padded box holds %lld cells", (long long)A->m,
           (long long)g.m);
  PB_CHECK(g.m < (int64_t)INT32_MAX && g.nint * A->nnd < (int64_t)INT32_MAX, PARCEL_B_E_UNSUPPORTED,
           "%lld cells x %d points: the renumbered matrix is indexed by int32", (long long)g.m, A->nnd);
  return g;
}

struct Box {
  int lo[3], hi[3];
};

// The block-Jacobi boxes of the interior, in the order their rows are numbered.
std::vector<Box> ddm_boxes(const DdmGeo& g, int mode, int div_dir, int nthreads) {
  std::vector<Box> out;
  if (mode == PARCEL_B_DDM_BOXES_THREADS) {
    PB_CHECK(div_dir >= 1 && div_dir <= 3, PARCEL_B_E_UNSUPPORTED,
             "div_direc_th = %d: the block-Jacobi slabs are cut along x (1), y (2) or z (3)", div_dir);
    const int d = div_dir - 1;
    const int nt = std::max(1, nthreads);
    const int n1 = g.n[d] / nt;   // set_region_for_threads: the last thread takes the rest
    for (int t = 0; t < nt; ++t) {
      Box b;
      for (int e = 0; e < 3; ++e) { b.lo[e] = 0; b.hi[e] = g.n[e]; }
      b.lo[d] = n1 * t;
      b.hi[d] = (t == nt - 1) ? g.n[d] : b.lo[d] + n1;
      if (b.hi[d] > b.lo[d]) out.push_back(b);
    }
  } else {
    PB_CHECK(mode == PARCEL_B_DDM_BOXES_CUBES, PARCEL_B_E_ARG, "boxes = %d", mode);
    // init_DILU_DDM with n_d / 4 divisions: ceil(n_d / div) cells per box, the last shorter
    int div[3], len[3];
    for (int e = 0; e < 3; ++e) {
      div[e] = std::max(g.n[e] / 4, 1);
      len[e] = g.n[e] / div[e] + (g.n[e] % div[e] ? 1 : 0);
    }
    for (int bz = 0; bz < div[2]; ++bz)
      for (int by = 0; by < div[1]; ++by)
        for (int bx = 0; bx < div[0]; ++bx) {
          const int bi[3] = {bx, by, bz};
          Box b;
          bool empty = false;
          for (int e = 0; e < 3; ++e) {
            b.lo[e] = len[e] * bi[e];
            b.hi[e] = std::min(g.n[e], len[e] * (bi[e] + 1));
            empty |= b.hi[e] <= b.lo[e];
          }
          if (!empty) out.push_back(b);
        }
  }
  return out;
}

// perm[r] = padded index of the interior cell numbered r; starts[b] = first row of box b.
void ddm_order(const DdmGeo& g, const std::vector<Box>& boxes, std::vector<int>* perm, std::vector<int>& starts) {
  starts.assign(boxes.size() + 1, 0);
  if (perm) perm->resize((size_t)g.nint);
  int64_t r = 0;
  for (size_t b = 0; b < boxes.size(); ++b) {
    const Box& B = boxes[b];
    starts[b] = (int)r;
    for (int z = B.lo[2]; z < B.hi[2]; ++z)
      for (int y = B.lo[1]; y < B.hi[1]; ++y) {
        const int64_t row = (int64_t)(y + g.mg[1]) * g.stride[1] + (int64_t)(z + g.mg[2]) * g.stride[2];
        for (int x = B.lo[0]; x < B.hi[0]; ++x, ++r)
          if (perm) (*perm)[r] = (int)(row + x + g.mg[0]);
      }
  }
  starts[boxes.size()] = (int)r;
}

// ---- renumbered CRS, built on the device
__device__ __forceinline__ bool ddm_keep(const double* vh, const double* vl, int64_t q) {
  return fabs(vh[q]) > 0.0 || (vl != nullptr && fabs(vl[q]) > 0.0);
}

// Entries of row r: stencil points whose neighbour is an interior cell, nonzero.
__global__ void k_ddm_count(int nint, int nnd, int64_t m, const int* __restrict__ perm, const int* __restrict__ inv,
                            const int* __restrict__ off, const double* __restrict__ vh,
                            const double* __restrict__ vl, int* __restrict__ cnt) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nint; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = perm[r];
    int c = 0;
    for (int k = 0; k < nnd; ++k) {
      const int64_t q = j + off[k];
      if (q >= 0 && q < m && inv[q] >= 0 && ddm_keep(vh, vl, (int64_t)k * m + j)) ++c;
    }
    cnt[r] = c;
  }
}

// Row r's entries sorted by their new column (1-based), values and low parts.  rp holds
// the 0-based row starts.
__global__ void k_ddm_fill(int nint, int nnd, int64_t m, const int* __restrict__ perm, const int* __restrict__ inv,
                           const int* __restrict__ off, const double* __restrict__ vh, const double* __restrict__ vl,
                           const int* __restrict__ rp, int* __restrict__ col_out, double* __restrict__ vh_out,
                           double* __restrict__ vl_out) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nint; r += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = perm[r];
    int cols[kDdmMaxNnd], pts[kDdmMaxNnd];
    int c = 0;
    for (int k = 0; k < nnd; ++k) {
      const int64_t q = j + off[k];
      if (q >= 0 && q < m && inv[q] >= 0 && ddm_keep(vh, vl, (int64_t)k * m + j)) {
        int t = c++;   // insertion by new column
        while (t > 0 && cols[t - 1] > inv[q]) {
          cols[t] = cols[t - 1];
          pts[t] = pts[t - 1];
          --t;
        }
        cols[t] = inv[q];
        pts[t] = k;
      }
    }
    const int p0 = rp[r];
    for (int t = 0; t < c; ++t) {
      const int64_t src = (int64_t)pts[t] * m + j;
      col_out[p0 + t] = cols[t] + 1;
      vh_out[p0 + t] = vh[src];
      if (vl_out) vl_out[p0 + t] = vl ? vl[src] : 0.0;
    }
  }
}

__global__ void k_ddm_rowptr(int64_t n1, int* __restrict__ a) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n1; i += (int64_t)gridDim.x * blockDim.x)
    a[i] += 1;
}

// perm[r] = padded index of interior cell r and inv[perm[r]] = r (inv holds -1 elsewhere,
// set before).  Box b's cells are rows starts[b] .. starts[b + 1] - 1, x fastest inside the
// box; bx holds each box's lo[3], hi[3].  Boxes are never empty, so starts is strictly
// increasing and the search finds the one box that holds r.
__global__ void k_ddm_perm(int nint, int nb, const int* __restrict__ starts, const int* __restrict__ bx, int mg0,
                           int mg1, int mg2, int64_t s1, int64_t s2, int* __restrict__ perm, int* __restrict__ inv) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nint; r += (int64_t)gridDim.x * blockDim.x) {
    int a = 0, z = nb;   // starts[a] <= r < starts[z]
    while (z - a > 1) {
      const int h = (a + z) >> 1;
      if (starts[h] <= r) a = h;
      else z = h;
    }
    const int* B = bx + 6 * (int64_t)a;
    const int ex = B[3] - B[0], ey = B[4] - B[1];
    const int loc = (int)r - starts[a];
    const int x = B[0] + loc % ex, y = B[1] + (loc / ex) % ey, zc = B[2] + loc / (ex * ey);
    const int64_t j = (int64_t)(x + mg0) + (int64_t)(y + mg1) * s1 + (int64_t)(zc + mg2) * s2;
    perm[r] = (int)j;
    inv[j] = (int)r;
  }
}

// dst[r] = src[perm[r]] (to the renumbered order) or dst[perm[r]] = src[r] (back).
__global__ void k_ddm_move(int nint, const int* __restrict__ perm, const double* __restrict__ src,
                           double* __restrict__ dst, int to_box) {
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nint; r += (int64_t)gridDim.x * blockDim.x) {
    if (to_box) dst[r] = src[perm[r]];
    else dst[perm[r]] = src[r];
  }
}

// The renumbered system on the device.
struct DdmCrs {
  DdmGeo g;
  std::vector<int> starts;
  DBuf perm, rowptr, col, vh, vl;
  parcel_b_crs crs;
  const double* lo() const { return vl.p ? dp<double>(vl) : nullptr; }
};

void ddm_build(const parcel_b_ddm* A, int precon_thblock, const double* val_lo, DdmCrs& out) {
  DdmGeo g = ddm_geometry(A);
  PB_CHECK(A->nnd >= 1 && A->nnd <= kDdmMaxNnd, PARCEL_B_E_UNSUPPORTED, "nnd = %d (1..%d stencil points)", A->nnd,
           kDdmMaxNnd);
  PB_CHECK(A->val && A->offset && A->offset_dim, PARCEL_B_E_ARG, "DDM arrays must not be NULL");
  const int nnd = A->nnd;
  std::vector<int> off(nnd), od((size_t)nnd * A->ndim);
  if (is_device_ptr(A->offset)) d2h(off.data(), A->offset, sizeof(int) * nnd);
  else std::memcpy(off.data(), A->offset, sizeof(int) * nnd);
  if (is_device_ptr(A->offset_dim)) d2h(od.data(), A->offset_dim, sizeof(int) * od.size());
  else std::memcpy(od.data(), A->offset_dim, sizeof(int) * od.size());
  for (int k = 0; k < nnd; ++k) {
    int64_t lin = 0;
    for (int d = 0; d < A->ndim; ++d) {
      const int o = od[(size_t)k + (size_t)nnd * d];
      PB_CHECK(o >= -A->margin && o <= A->margin, PARCEL_B_E_ARG,
               "offset_dim(%d, %d) = %d reaches beyond the margin %d", k + 1, d + 1, o, A->margin);
      lin += (int64_t)o * g.stride[d];
    }
    PB_CHECK(lin == off[k], PARCEL_B_E_ARG, "offset(%d) = %d, its offset_dim gives %lld", k + 1, off[k],
             (long long)lin);
    for (int k2 = 0; k2 < k; ++k2)
      PB_CHECK(off[k2] != off[k], PARCEL_B_E_ARG, "offset %d appears twice", off[k]);
  }
  const std::vector<Box> boxes = ddm_boxes(g, A->boxes, A->div_direc_th, precon_thblock);
  ddm_order(g, boxes, nullptr, out.starts);
  const int nbox = (int)boxes.size();
  std::vector<int> bx((size_t)6 * nbox);
  for (int b = 0; b < nbox; ++b)
    for (int e = 0; e < 3; ++e) {
      bx[(size_t)6 * b + e] = boxes[b].lo[e];
      bx[(size_t)6 * b + 3 + e] = boxes[b].hi[e];
    }

  cudaStream_t st = stream();
  const int nint = (int)g.nint;
  const size_t nv = (size_t)nnd * (size_t)g.m;
  // the numbering and its inverse, built on the device from the boxes
  out.perm.alloc(sizeof(int) * (size_t)nint);
  DBuf dinv(sizeof(int) * (size_t)g.m), doff(sizeof(int) * nnd), dbx(sizeof(int) * bx.size()),
      dst(sizeof(int) * out.starts.size());
  h2d(dbx.p, bx.data(), sizeof(int) * bx.size());
  h2d(dst.p, out.starts.data(), sizeof(int) * out.starts.size());
  h2d(doff.p, off.data(), sizeof(int) * nnd);
  PB_CUDA(cudaMemsetAsync(dinv.p, 0xFF, sizeof(int) * (size_t)g.m, st));   // -1: margin cells
  k_ddm_perm<<<ddm_grid(nint), kDdmThreads, 0, st>>>(nint, nbox, dp<int>(dst), dp<int>(dbx), g.mg[0], g.mg[1],
                                                     g.mg[2], g.stride[1], g.stride[2], dp<int>(out.perm),
                                                     dp<int>(dinv));
  PB_CUDA(cudaGetLastError());
  DBuf hv, lv;
  const double* vh = A->val;
  const double* vl = val_lo;
  if (!is_device_ptr(vh)) {
    hv.alloc(sizeof(double) * nv);
    h2d(hv.p, vh, sizeof(double) * nv);
    vh = dp<double>(hv);
  }
  if (vl && !is_device_ptr(vl)) {
    lv.alloc(sizeof(double) * nv);
    h2d(lv.p, vl, sizeof(double) * nv);
    vl = dp<double>(lv);
  }
  out.rowptr.alloc(sizeof(int) * ((size_t)nint + 1));   // zero-filled: rowptr[0] = 0
  int* rp = dp<int>(out.rowptr);
  const int grid = ddm_grid(nint);
  DBuf cnt(sizeof(int) * (size_t)nint);
  k_ddm_count<<<grid, kDdmThreads, 0, st>>>(nint, nnd, g.m, dp<int>(out.perm), dp<int>(dinv), dp<int>(doff), vh, vl,
                                            dp<int>(cnt));
  PB_CUDA(cudaGetLastError());
  size_t tmp_bytes = 0;
  PB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tmp_bytes, dp<int>(cnt), rp + 1, nint, st));
  DBuf tmp(std::max<size_t>(tmp_bytes, 16));
  PB_CUDA(cub::DeviceScan::InclusiveSum(tmp.p, tmp_bytes, dp<int>(cnt), rp + 1, nint, st));
  int nnz = 0;
  PB_CUDA(cudaMemcpyAsync(&nnz, rp + nint, sizeof(int), cudaMemcpyDeviceToHost, st));
  pb::sync();
  PB_CHECK(nnz > 0, PARCEL_B_E_ARG, "the DDM matrix has no nonzero coupling between interior cells");
  out.col.alloc(sizeof(int) * (size_t)nnz);
  out.vh.alloc(sizeof(double) * (size_t)nnz);
  if (val_lo) out.vl.alloc(sizeof(double) * (size_t)nnz);
  k_ddm_fill<<<grid, kDdmThreads, 0, st>>>(nint, nnd, g.m, dp<int>(out.perm), dp<int>(dinv), dp<int>(doff), vh, vl,
                                           rp, dp<int>(out.col), dp<double>(out.vh),
                                           val_lo ? dp<double>(out.vl) : nullptr);
  k_ddm_rowptr<<<ddm_grid(nint + 1), kDdmThreads, 0, st>>>((int64_t)nint + 1, rp);
  PB_CUDA(cudaGetLastError());
  pb::sync();   // the uploaded arrays are released on return
  out.g = g;
  out.crs.n = nint;
  out.crs.gn = nint;
  out.crs.nnz = nnz;
  out.crs.istart = 1;
  out.crs.rowptr = rp;
  out.crs.col = dp<int>(out.col);
  out.crs.val = dp<double>(out.vh);
}

// A vector of the padded box (host or device, m entries) in the renumbered order, on the
// device, and back.
struct BoxVec {
  DBuf box, full;
  const double* src = nullptr;
  BoxVec(const DdmCrs& C, const double* v) {
    const int nint = (int)C.g.nint;
    box.alloc(sizeof(double) * (size_t)std::max(nint, 1));
    if (!v) return;
    src = v;
    const double* d = v;
    if (!is_device_ptr(v)) {
      full.alloc(sizeof(double) * (size_t)C.g.m);
      h2d(full.p, v, sizeof(double) * (size_t)C.g.m);
      d = dp<double>(full);
    }
    k_ddm_move<<<ddm_grid(nint), kDdmThreads, 0, stream()>>>(nint, dp<int>(C.perm), d, dp<double>(box), 1);
    PB_CUDA(cudaGetLastError());
  }
  double* p() { return dp<double>(box); }
  // Writes the interior cells back into the caller's array (margin untouched).
  void store(const DdmCrs& C, double* v) {
    const int nint = (int)C.g.nint;
    double* d = v;
    if (!is_device_ptr(v)) {
      if (!full.p) {
        full.alloc(sizeof(double) * (size_t)C.g.m);
        h2d(full.p, v, sizeof(double) * (size_t)C.g.m);
      }
      d = dp<double>(full);
    }
    k_ddm_move<<<ddm_grid(nint), kDdmThreads, 0, stream()>>>(nint, dp<int>(C.perm), dp<double>(box), d, 0);
    PB_CUDA(cudaGetLastError());
    if (d != v) d2h(v, d, sizeof(double) * (size_t)C.g.m);
    pb::sync();
  }
};

// The DDM options as the CRS solvers take them: D-ILU blocks, independ_nvec at its default.
parcel_b_input ddm_input(const parcel_b_input* prm) {
  parcel_b_input p;
  if (prm) p = *prm;
  else parcel_b_input_init(&p);
  PB_CHECK(p.ipreflag <= 2, PARCEL_B_E_UNSUPPORTED,
           "ipreflag = %d: the DDM path provides none (0), point Jacobi (1) and block-Jacobi D-ILU (2)", p.ipreflag);
  PB_CHECK(p.independ_nvec != 1, PARCEL_B_E_UNSUPPORTED,
           "independ_nvec = 1 (the x-line-independent DDM D-ILU) is not provided");
  p.ILU_method = PARCEL_B_ILUD;
  p.independ_nvec = -1;
  return p;
}

void add_ddm_setup_time(double secs) {
  parcel_b_stats s;
  if (parcel_b_last_stats(&s) != 0) return;
  s.setup_s += secs;
  s.total_s += secs;
  set_stats(s);
}

int ddm_fail(int rc, int* niter, int* iret) {
  if (iret) *iret = rc;
  if (niter) *niter = 0;
  return rc;
}

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" int parcel_b_ddm_order(const parcel_b_ddm* A, int precon_thblock, int32_t* perm, int32_t* starts,
                                  int32_t* nblocks) {
  return guarded([&]() -> int {
    PB_CHECK(nblocks != nullptr, PARCEL_B_E_ARG, "nblocks is NULL");
    DdmGeo g = ddm_geometry(A);
    const std::vector<Box> boxes = ddm_boxes(g, A->boxes, A->div_direc_th, precon_thblock);
    const int cap = *nblocks;
    *nblocks = (int)boxes.size();
    PB_CHECK(starts == nullptr || cap >= (int)boxes.size(), PARCEL_B_E_ARG,
             "starts holds %d + 1 entries, the box has %d blocks", cap, (int)boxes.size());
    std::vector<int> pv, sv;
    ddm_order(g, boxes, perm ? &pv : nullptr, sv);
    if (perm) std::memcpy(perm, pv.data(), sizeof(int) * pv.size());
    if (starts) std::memcpy(starts, sv.data(), sizeof(int) * sv.size());
    return 0;
  });
}

extern "C" int parcel_b_solve_ddm(const parcel_b_input* prm, const parcel_b_ddm* A, const double* b, double* x,
                                  double* reshistory, int* niter, int* iret) {
  DdmCrs C;
  parcel_b_input p;
  std::unique_ptr<BoxVec> bv, xv;
  double conv = 0.0;
  int rc = guarded([&]() -> int {
    ensure_init();
    PB_CHECK(b && x, PARCEL_B_E_ARG, "b and x must not be NULL");
    p = ddm_input(prm);
    const double t0 = now_s();
    ddm_build(A, p.precon_thblock, nullptr, C);
    bv.reset(new BoxVec(C, b));
    xv.reset(new BoxVec(C, x));
    pb::sync();
    conv = now_s() - t0;
    return 0;
  });
  if (rc < 0) return ddm_fail(rc, niter, iret);
  {
    ScopedBlockStarts blocks(&C.starts);
    rc = parcel_b_solve(&p, &C.crs, bv->p(), xv->p(), reshistory, niter, iret);
  }
  add_ddm_setup_time(conv);
  const int rc2 = guarded([&]() -> int {
    xv->store(C, x);
    return 0;
  });
  return rc < 0 ? rc : rc2;
}

extern "C" int parcel_b_ddsolve_ddm(const parcel_b_input* prm, const parcel_b_ddm* A, const double* val_lo,
                                    int precision_A, int precision_b, int precision_x, int precision_precondition,
                                    const double* b_hi, const double* b_lo, double* x_hi, double* x_lo,
                                    double* reshistory, int* niter, int* iret) {
  DdmCrs C;
  parcel_b_input p;
  std::unique_ptr<BoxVec> bh, bl, xh, xl;
  const int solver = prm && prm->solver > 0 ? prm->solver : PARCEL_B_SOLVER_CG;
  int rc = guarded([&]() -> int {
    ensure_init();
    PB_CHECK(b_hi && x_hi, PARCEL_B_E_ARG, "b_hi and x_hi must not be NULL");
    PB_CHECK(solver == PARCEL_B_SOLVER_CG || solver == PARCEL_B_SOLVER_BICG || solver == PARCEL_B_SOLVER_GMRES,
             PARCEL_B_E_UNSUPPORTED, "solver=%d: the dd solvers are CG (1), BiCGStab (2) and GMRES (3)", solver);
    p = ddm_input(prm);
    ddm_build(A, p.precon_thblock, precision_A == 2 ? val_lo : nullptr, C);
    bh.reset(new BoxVec(C, b_hi));
    bl.reset(new BoxVec(C, b_lo));
    xh.reset(new BoxVec(C, x_hi));
    xl.reset(new BoxVec(C, x_lo));
    pb::sync();
    return 0;
  });
  if (rc < 0) return ddm_fail(rc, niter, iret);
  auto fn = solver == PARCEL_B_SOLVER_BICG ? parcel_b_ddbicgstab
                                           : (solver == PARCEL_B_SOLVER_GMRES ? parcel_b_ddgmres : parcel_b_ddcg);
  {
    ScopedBlockStarts blocks(&C.starts);
    rc = fn(&p, &C.crs, C.lo(), precision_A, precision_b, precision_x, precision_precondition, bh->p(),
            b_lo ? bl->p() : nullptr, xh->p(), x_lo ? xl->p() : nullptr, reshistory, niter, iret);
  }
  const int rc2 = guarded([&]() -> int {
    xh->store(C, x_hi);
    if (x_lo) xl->store(C, x_lo);
    return 0;
  });
  return rc < 0 ? rc : rc2;
}

extern "C" int parcel_b_bench_kernels_ddm(const parcel_b_input* prm, const parcel_b_ddm* A, int reps,
                                          double* ms_spmv, double* ms_precon) {
  DdmCrs C;
  parcel_b_input p;
  const int rc = guarded([&]() -> int {
    ensure_init();
    p = ddm_input(prm);
    ddm_build(A, p.precon_thblock, nullptr, C);
    return 0;
  });
  if (rc < 0) return rc;
  ScopedBlockStarts blocks(&C.starts);
  return parcel_b_bench_kernels(&p, &C.crs, reps, ms_spmv, ms_precon);
}

// ---- drop-in shims (src/example/c2fortran_kernel.f90:2964-3691) --------------------------
namespace {

// One process: the box is the whole grid (npe_dim all 1, no neighbour ranks).
int ddm_desc(parcel_b_ddm* A, int32_t* n, int* nnd, const int32_t* offset, const double* diaA, int* num_neighbor_ranks,
             const int* neighbor_ranks, int* margin, int* ndim, const int* npe_dim, const int* n_grids,
             const int* offset_dim, int* div_direc_th, int boxes) {
  std::memset(A, 0, sizeof(*A));
  A->ndim = *ndim;
  int procs = 1;
  for (int d = 0; d < *ndim && d < 3; ++d) {
    A->n_grids[d] = n_grids[d];
    procs *= npe_dim[d];
  }
  int neighbours = 0;
  for (int i = 0; i < *num_neighbor_ranks; ++i)
    if (neighbor_ranks[i] >= 0) ++neighbours;
  if (procs != 1 || neighbours != 0) {
    set_last_error(PARCEL_B_E_UNSUPPORTED,
                   "a DDM box split over %d processes (%d neighbour ranks) runs through parcel_b.ddm "
                   "(torch.distributed); these entry points take one process's whole grid", procs, neighbours);
    return PARCEL_B_E_UNSUPPORTED;
  }
  A->margin = *margin;
  A->m = *n;
  A->nnd = *nnd;
  A->offset = offset;
  A->offset_dim = offset_dim;
  A->val = diaA;
  A->div_direc_th = *div_direc_th;
  A->boxes = boxes;
  return 0;
}

void ddm_params(parcel_b_input* p, int solver, int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock) {
  parcel_b_input_init(p);
  p->solver = solver;
  p->ipreflag = *ipreflag;
  p->addL = *addl;
  p->iflagAS = *iflagas;
  p->itrmax = *niter;
  p->rtolmax = *rtolmax;
  p->abstolmax = 0.0;
  p->iovlflag = *iovlflag;
  p->precon_thblock = *precon_thblock;
  p->Neuman_itr = *neuman_itr;
  p->independ_nvec = *independ_nvec;
  p->nBlock = *nblock;
}

void ddm_run(parcel_b_input* p, int boxes, int32_t* n, int* nnd, int32_t* offset, double* diaA,
             int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim, int* npe_dim, int* n_grids,
             int* offset_dim, int* div_direc_th, double* vecb, double* vecx, double* reshistory, int* niter,
             int* iret) {
  parcel_b_ddm A;
  int rc = ddm_desc(&A, n, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim, n_grids,
                    offset_dim, div_direc_th, boxes);
  int used = 0, ir = rc;
  if (rc == 0) parcel_b_solve_ddm(p, &A, vecb, vecx, reshistory, &used, &ir);
  *niter = used;
  *iret = ir;
}

void dd_ddm_run(parcel_b_input* p, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                int* nnd, int32_t* offset, double* diaA, double* diaA_lo, int* num_neighbor_ranks,
                int* neighbor_ranks, int* margin, int* ndim, int* npe_dim, int* n_grids, int* offset_dim,
                int* div_direc_th, double* reshistory, int* pa, int* pb, int* px, int* pm, int* niter, int* iret) {
  parcel_b_ddm A;
  int rc = ddm_desc(&A, n, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim, npe_dim, n_grids,
                    offset_dim, div_direc_th, PARCEL_B_DDM_BOXES_THREADS);
  int used = 0, ir = rc;
  if (rc == 0)
    parcel_b_ddsolve_ddm(p, &A, diaA_lo, *pa, *pb, *px, *pm, vecb, vecb_lo, vecx, vecx_lo, reshistory, &used, &ir);
  *niter = used;
  *iret = ir;
}

}  // namespace

extern "C" {

void parcel_dcg_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                       double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim,
                       int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag,
                       int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                       int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                       int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_CG, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock, neuman_itr,
             independ_nvec, nblock);
  ddm_run(&p, PARCEL_B_DDM_BOXES_THREADS, n, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim,
          npe_dim, n_grids, offset_dim, div_direc_th, vecb, vecx, reshistory, niter, iret);
}

void parcel_dbicgstab_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                             double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                             int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                             int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                             double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                             int* independ_nvec, int* nblock, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_BICG, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  ddm_run(&p, PARCEL_B_DDM_BOXES_THREADS, n, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim,
          npe_dim, n_grids, offset_dim, div_direc_th, vecb, vecx, reshistory, niter, iret);
}

void parcel_dgmres_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                          double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                          int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                          int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                          double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                          int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_GMRES, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  p.GMRES_m = *restart;
  p.GMRES_GSflag = *gmres_gsflag;
  ddm_run(&p, PARCEL_B_DDM_BOXES_THREADS, n, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim,
          npe_dim, n_grids, offset_dim, div_direc_th, vecb, vecx, reshistory, niter, iret);
}

void parcel_dcagmres_ddm_c_(int* icomm, double* vecx, double* vecb, int32_t* n, int* nnd, int32_t* offset,
                            double* diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                            int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                            int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                            double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                            int* independ_nvec, int* nblock, int* cagmres_sstep, int* cagmres_tstep,
                            int* cagmres_basis, int* cagmres_qrflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_CAGMRES, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  p.CAGMRES_sstep = *cagmres_sstep;
  p.CAGMRES_tstep = *cagmres_tstep;
  p.CAGMRES_basis = *cagmres_basis;
  p.CAGMRES_QRflag = *cagmres_qrflag;
  ddm_run(&p, PARCEL_B_DDM_BOXES_THREADS, n, nnd, offset, diaA, num_neighbor_ranks, neighbor_ranks, margin, ndim,
          npe_dim, n_grids, offset_dim, div_direc_th, vecb, vecx, reshistory, niter, iret);
}

void parcel_ddcg_ddm_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                        int* nnd, int32_t* offset, double* diaA, double* diaA_lo, int* num_neighbor_ranks,
                        int* neighbor_ranks, int* margin, int* ndim, int* npe_dim, int* n_grids,
                        int* offset_dim, int* div_direc_th, int* ipreflag, int* addl, int* iflagas, int* niter,
                        double* rtolmax, double* reshistory, int* iovlflag, int* precon_thblock,
                        int* neuman_itr, int* independ_nvec, int* nblock, int* precision_A, int* precision_b,
                        int* precision_x, int* precision_precondition, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_CG, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock, neuman_itr,
             independ_nvec, nblock);
  dd_ddm_run(&p, vecx, vecx_lo, vecb, vecb_lo, n, nnd, offset, diaA, diaA_lo, num_neighbor_ranks, neighbor_ranks,
             margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, reshistory, precision_A, precision_b,
             precision_x, precision_precondition, niter, iret);
}

void parcel_ddbicgstab_ddm_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo,
                              int32_t* n, int* nnd, int32_t* offset, double* diaA, double* diaA_lo,
                              int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim,
                              int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag,
                              int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                              int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                              int* nblock, int* precision_A, int* precision_b, int* precision_x,
                              int* precision_precondition, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_BICG, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  dd_ddm_run(&p, vecx, vecx_lo, vecb, vecb_lo, n, nnd, offset, diaA, diaA_lo, num_neighbor_ranks, neighbor_ranks,
             margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, reshistory, precision_A, precision_b,
             precision_x, precision_precondition, niter, iret);
}

void parcel_ddgmres_ddm_c_(int* icomm, double* vecx, double* vecx_lo, double* vecb, double* vecb_lo, int32_t* n,
                           int* nnd, int32_t* offset, double* diaA, double* diaA_lo, int* num_neighbor_ranks,
                           int* neighbor_ranks, int* margin, int* ndim, int* npe_dim, int* n_grids,
                           int* offset_dim, int* div_direc_th, int* ipreflag, int* addl, int* iflagas,
                           int* niter, double* rtolmax, double* reshistory, int* iovlflag,
                           int* precon_thblock, int* neuman_itr, int* independ_nvec, int* nblock,
                           int* restart, int* gmres_gsflag, int* precision_A, int* precision_b,
                           int* precision_x, int* precision_precondition, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_GMRES, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  p.GMRES_m = *restart;
  p.GMRES_GSflag = *gmres_gsflag;
  dd_ddm_run(&p, vecx, vecx_lo, vecb, vecb_lo, n, nnd, offset, diaA, diaA_lo, num_neighbor_ranks, neighbor_ranks,
             margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, reshistory, precision_A, precision_b,
             precision_x, precision_precondition, niter, iret);
}

// CUDA-build forms: device arrays behind devicemem handles, n_d / 4 boxes per axis.
void parcel_dcg_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                           void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin, int* ndim,
                           int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th, int* ipreflag,
                           int* addl, int* iflagas, int* niter, double* rtolmax, double* reshistory,
                           int* iovlflag, int* precon_thblock, int* neuman_itr, int* independ_nvec,
                           int* nblock, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_CG, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock, neuman_itr,
             independ_nvec, nblock);
  ddm_run(&p, PARCEL_B_DDM_BOXES_CUBES, n, nnd, (int32_t*)*offset, (double*)*diaA, num_neighbor_ranks,
          neighbor_ranks, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, (double*)*vecb,
          (double*)*vecx, reshistory, niter, iret);
}

void parcel_dbicgstab_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                                 void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                                 int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                                 int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                                 double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                                 int* independ_nvec, int* nblock, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_BICG, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  ddm_run(&p, PARCEL_B_DDM_BOXES_CUBES, n, nnd, (int32_t*)*offset, (double*)*diaA, num_neighbor_ranks,
          neighbor_ranks, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, (double*)*vecb,
          (double*)*vecx, reshistory, niter, iret);
}

void parcel_dgmres_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                              void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                              int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                              int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                              double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                              int* independ_nvec, int* nblock, int* restart, int* gmres_gsflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_GMRES, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  p.GMRES_m = *restart;
  p.GMRES_GSflag = *gmres_gsflag;
  ddm_run(&p, PARCEL_B_DDM_BOXES_CUBES, n, nnd, (int32_t*)*offset, (double*)*diaA, num_neighbor_ranks,
          neighbor_ranks, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, (double*)*vecb,
          (double*)*vecx, reshistory, niter, iret);
}

void parcel_dcagmres_ddm_gpu_c_(int* icomm, void** vecx, void** vecb, int32_t* n, int* nnd, void** offset,
                                void** diaA, int* num_neighbor_ranks, int* neighbor_ranks, int* margin,
                                int* ndim, int* npe_dim, int* n_grids, int* offset_dim, int* div_direc_th,
                                int* ipreflag, int* addl, int* iflagas, int* niter, double* rtolmax,
                                double* reshistory, int* iovlflag, int* precon_thblock, int* neuman_itr,
                                int* independ_nvec, int* nblock, int* cagmres_sstep, int* cagmres_tstep,
                                int* cagmres_basis, int* cagmres_qrflag, int* iret) {
  (void)icomm;
  parcel_b_input p;
  ddm_params(&p, PARCEL_B_SOLVER_CAGMRES, ipreflag, addl, iflagas, niter, rtolmax, iovlflag, precon_thblock,
             neuman_itr, independ_nvec, nblock);
  p.CAGMRES_sstep = *cagmres_sstep;
  p.CAGMRES_tstep = *cagmres_tstep;
  p.CAGMRES_basis = *cagmres_basis;
  p.CAGMRES_QRflag = *cagmres_qrflag;
  ddm_run(&p, PARCEL_B_DDM_BOXES_CUBES, n, nnd, (int32_t*)*offset, (double*)*diaA, num_neighbor_ranks,
          neighbor_ranks, margin, ndim, npe_dim, n_grids, offset_dim, div_direc_th, (double*)*vecb,
          (double*)*vecx, reshistory, niter, iret);
}

}  // extern "C"
