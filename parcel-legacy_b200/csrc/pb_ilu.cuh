// pb_ilu.cuh -- block-Jacobi ILU(0) / D-ILU preconditioner on the level-major layout.
#pragma once

#include <functional>
#include <vector>

#include "pb_common.cuh"

namespace pb {

// Device matrix view.  Row pointers and columns may be 1-based (the reference's arrays,
// rbase = 1, cbase = istart) or 0-based (internal copies, rbase = cbase = 0).
template <class VT>
struct DevMat {
  int n = 0;
  int64_t nnz = 0;
  const int* rowptr = nullptr;
  const int* col = nullptr;
  const VT* val = nullptr;
  int rbase = 0;
  int cbase = 0;
  // Sliced ELLPACK copy (32-row slices, column-major within a slice) used by the SpMV
  // when present: entry k of row r lives at s_off[r/32] + 32 k + r%32.
  int nslices = 0;
  const int* s_off = nullptr;
  const int* s_w = nullptr;
  const int* s_col = nullptr;
  const VT* s_val = nullptr;
  // Diagonal (DIA) copy used by the SpMV when present (natural layout of a matrix whose
  // entries lie on at most kDiaMaxDiag diagonals): entry of row r on diagonal k (column
  // r + d_off[k], offsets ascending) at d_val[(r - r % 32) nd + 32 k + r % 32] (32-row
  // slices, as the ELLPACK copy), zero where the row has no entry.
  int ndiag = 0;
  const int* d_off = nullptr;
  const VT* d_val = nullptr;
};

template <class VT>
struct SellBuf {
  DBuf off, w, col, val;
  DBuf doff, dval;   // diagonal copy (build_dia)
};

constexpr int kDiaMaxDiag = 16;

// Builds the sliced-ELLPACK copy of the natural CRS matrix A in the row order
// rowAt (device: permuted position -> natural row, -1 = empty row; null = identity) with
// columns mapped through pos (device: natural -> permuted; null = identity).  Slice widths
// and offsets are computed on the device.  Fills M's SELL fields.
template <class VT>
void build_sell(const DevMat<double>& A, int np, const int* rowAt_d, const int* pos_d, SellBuf<VT>& buf,
                DevMat<VT>& M);
// Builds the diagonal copy of the natural CRS matrix A when every entry lies on one of at
// most kDiaMaxDiag diagonals and the copy holds at most 1.5 nnz values; fills M's DIA fields
// and returns the number of diagonals (0: not built).
template <class VT>
int build_dia(const DevMat<double>& A, SellBuf<VT>& buf, DevMat<VT>& M);

// One chunk = up to kIluChunk rows of one wavefront level of one block.  Wider levels are
// split into several chunks (their rows are independent; each chunk is one sweep step).
struct IluChunk {
  int start;         // permuted position of the first row (multiple of 4)
  int w;             // rows
  int wpad;          // rows rounded up to 4
  int KL, KU;        // max strictly-lower / strictly-upper in-block entries of its rows
  int lvl;           // level index within the block
  int off_in_level;  // position of the chunk's first row within its level
  int blk;           // block-Jacobi block
  int64_t offF, offB;   // byte offsets of the packed forward / backward data
  // left uninitialised: the plan writes every field, and a plan of tens of thousands of
  // small blocks holds hundreds of thousands of chunks
  __host__ __device__ IluChunk() {}
};
constexpr int kIluChunk = 512;      // rows per chunk (multiple of 4)
constexpr int kIluHeader = 32;      // bytes of the per-chunk header in the packed data

// Host-side plan: wavefront levels of every block and the permuted, padded layout.
struct IluPlan {
  int n = 0;            // natural rows
  int np = 0;           // permuted length incl. padding
  int nb = 0;           // blocks
  int W = 1;            // ring depth in levels
  int maxWp = 0;        // widest chunk (padded)
  int max_levels = 0;
  int* pos = nullptr;           // natural row -> permuted position (caller's storage, n)
  int* lev = nullptr;           // natural row -> level within its block (caller's storage, n)
  std::vector<IluChunk> chunks;
  std::vector<int> blk_chunk;   // nb + 1
  std::vector<int> blk_lo, blk_hi;   // natural row ranges [lo, hi)
  std::vector<int> lvl_start;   // per block-level (global index) permuted start
  std::vector<int> lvl_end;     // per block-level permuted end (start + width)
  std::vector<int> blk_lvl;     // nb + 1 index into lvl_start
};

// Device-resident preconditioner.
template <class T>
struct IluDev {
  int nb = 0, np = 0, n = 0;
  int W = 1, maxWp = 0;
  bool ring = true;
  bool dilu = false;
  bool grp = false;  // grouped sweep (ring mode, K <= 8, two stages fit); else the general one
  int nc = 256;      // consumer threads of the grouped sweep (128 or 256)
  int rows = 1;      // rows per consumer thread of the grouped sweep (1 or 2)
  int K = 0;         // coupled entries per row in every record
  int ngroups = 0;
  int stage_bytes = 0, nstages = 0, smem_bytes = 0;
  DBuf chunks;      // IluChunk[]
  DBuf tabF, tabB;  // producer descriptors: per group (grouped sweep) or per chunk
  DBuf blk_grp;     // int[nb+1]: first group of each block
  DBuf ginfo, goff; // per group {first chunk, end chunk, sstart, sspan} and record offsets
  DBuf blk_chunk;   // int[nb+1]
  DBuf packF, packB;
  int64_t packF_bytes = 0, packB_bytes = 0;
  DBuf ytmp;        // forward result, np + 1 entries
  DBuf err;         // int error flag
  // Many small blocks (k_ilu_small): one warp per block, per-row records in the iteration
  // layout: K coupled entries (permuted column or -1, value) and a diagonal factor for each
  // sweep, forward (F) and backward (B).
  bool small = false;
  int s_lpb = 32;                           // lanes per block (8, 16 or 32)
  DBuf s_blvl, s_lo, s_hi;                  // block -> first level (nb + 1); level -> [lo, hi)
  DBuf s_cF, s_vF, s_dF, s_cB, s_vB, s_dB;
  // staged variant (k_ilu_small_staged): per block its first iteration-layout position and
  // its stretch rounded up to 4 positions; the largest stretch and level count; the shared
  // memory of one block (0: the stretches are too long, the unstaged sweep runs)
  DBuf s_box;
  int s_span = 0, s_levcap = 0, s_box_bytes = 0;
};

// Sparsity structure of the natural matrix on the host (for the wavefront plan).
struct HostCSR {
  int n = 0;
  int64_t nnz = 0;
  int istart = 1;
  const int* rowptr = nullptr;   // 1-based
  const int* col = nullptr;      // 1-based global
};

// Natural rows [lo, hi) of block-Jacobi block b of nb (0-based).
void ilu_block_rows(int b, int nb, int n, int* lo, int* hi);

// Row ranges of the block-Jacobi blocks: divide_region's equal split of the n rows into nb
// parts (common.f90:125-182), or explicit 0-based row starts, starts[nb] = n (the boxes of a
// stencil-format matrix, laid out one after another).
struct BlockSplit {
  int nb = 1;
  std::vector<int> starts;
  void rows(int b, int n, int* lo, int* hi) const {
    if (starts.empty()) { ilu_block_rows(b, nb, n, lo, hi); return; }
    *lo = starts[b];
    *hi = starts[b + 1];
  }
};
// Threads of the one-CTA-per-block factorisation kernels: the widest level rounded up to a
// warp, at most 256 (a CTA walks its block's levels with a stride of its size, so any size
// gives the same result; small blocks with narrow levels then fit many more CTAs per SM).
inline int ilu_factor_threads(int maxWp) { return std::min(256, std::max(32, (maxWp + 31) & ~31)); }

// rowAt[pos[i]] = i for i < n (entries not hit keep their value).
void scatter_positions(int n, const int* pos, int* rowAt, cudaStream_t st);

// Wavefront plan of the block-Jacobi blocks.  pos_out and lev_out (n entries each) receive
// the permutation and the levels.  block_ready(b), when given, is called before block b's
// rows are read (the structure may still be arriving from the device).
void ilu_build_plan(const HostCSR& A, const BlockSplit& blocks, IluPlan& P, int* pos_out, int* lev_out,
                    const std::function<void(int)>& block_ready = {});

// Factorises (ILU(0)) or computes the D-ILU diagonal on the device and packs the sweep
// data.  ilu_method: 0 ILU(0), 1 ILUD, 2 MLUD (define.f90:40-42).  Returns a status.
template <class T>
int ilu_setup_device(const IluPlan& P, const DevMat<double>& A, int ilu_method,
                     const int* d_pos, const int* d_rowAt, const int* d_lev, IluDev<T>& D);

// s = M^-1 r on permuted vectors (np entries each).  If `accum` is non-null the result
// is added into it instead of being written to s (s may then be null).
template <class T>
void ilu_apply(const IluDev<T>& D, const T* r, T* s, T* accum, const int* gate, cudaStream_t st);

}  // namespace pb
