// pb_ilu.cu -- block-Jacobi ILU(0) and D-ILU on B200.
//
// Reference algorithms (restated, not translated):
//   * blocks: contiguous row ranges from divide_region (src/common.f90:125-182);
//   * ILU(0): IKJ factorisation of each block's in-block submatrix, L unit-diagonal,
//     U with its diagonal (src/matrix.f90:7970-8072, 8249-8392); sweeps
//     solve_LU_crs (matrix.f90:8548-8747);
//   * D-ILU: K = (D+L) D^-1 (D+U) with D matched to the diagonal (ILUD) or the row sum
//     (MLUD) (DILU_DInv_crs, matrix.f90:3482-3648); sweeps solve_ILU_crs
//     (matrix.f90:4987-5163).
// The reference runs each block's sweeps sequentially on one OpenMP thread (CPU) or one
// cuSPARSE csrsv2 solve per process (src/CUDA/src/cusparse.cu:712-787).
//
// B200 design.  Rows of every block are grouped into wavefront levels (row i depends on
// the in-block rows it couples to with a smaller index), and the library stores every
// Krylov vector in a permuted, level-major layout where each level is contiguous and
// starts on a 16-byte boundary.  One CTA sweeps one block.  A producer warp streams each
// level's packed coefficients and its input-vector slice into a ring of shared-memory
// stages with bulk asynchronous copies (cp.async.bulk + mbarrier); the consumer warps
// solve the level's rows from shared memory, keeping the last W levels of the solution in
// a shared-memory ring, so a level step costs shared-memory latency and one named
// barrier.  The arithmetic of every row is the reference's: same operands, same order.
#include <algorithm>
#include <omp.h>
#include <climits>
#include <cmath>
#include <memory>
#include <numeric>

#include "pb_device.cuh"
#include "pb_ilu.cuh"

namespace pb {

namespace {

inline int align4(int x) { return (x + 3) & ~3; }
inline int64_t align16(int64_t x) { return (x + 15) & ~int64_t(15); }

void divide_region(int r, int np, long idown, long iup, long* lo, long* hi) {
  if (iup == idown) { *lo = idown; *hi = iup; return; }
  long region = iup - idown + 1, blk = region / np, over = region % np;
  if (r < over) { *lo = idown + blk * r + r; *hi = *lo + blk; }
  else { *lo = idown + blk * r + over; *hi = *lo + blk - 1; }
}

}  // namespace

void ilu_block_rows(int b, int nb, int n, int* lo, int* hi) {
  long l, h;
  divide_region(b, nb, 1, n, &l, &h);
  *lo = (int)(l - 1);
  *hi = (int)h;
}

__global__ void k_scatter_rowat(int n, const int* __restrict__ pos, int* __restrict__ rowAt) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) rowAt[pos[i]] = i;
}

void scatter_positions(int n, const int* pos, int* rowAt, cudaStream_t st) {
  if (n <= 0) return;
  const int grid = (int)std::min<int64_t>(((int64_t)n + 255) / 256, 8LL * num_sms());
  k_scatter_rowat<<<grid, 256, 0, st>>>(n, pos, rowAt);
  PB_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ host plan
// Levels: row x waits for every in-block row y < x coupled to it in either direction
// (a lower entry of x, or an upper entry (y, x) of y), so one level order serves the
// forward and the backward sweep.  The dependency window W is the largest level gap of
// any coupling + 1; it is found in the same pass: lower couplings compare with rows whose
// level is final, upper couplings (y, x) through the lowest level among x's upper-entry
// sources, known once x is reached.
void ilu_build_plan(const HostCSR& A, const BlockSplit& blocks, IluPlan& P, int* pos_out, int* lev_out,
                    const std::function<void(int)>& block_ready) {
  const int n = A.n;
  const int nb = blocks.nb;
  P.n = n;
  P.nb = nb;
  P.lev = lev_out;
  P.pos = pos_out;
  P.blk_lo.resize(nb);
  P.blk_hi.resize(nb);
  for (int b = 0; b < nb; ++b) blocks.rows(b, n, &P.blk_lo[b], &P.blk_hi[b]);
  std::vector<int> nlev(nb, 0), gap(nb, 0), missing_diag(nb, 0);
  // per-row coupling counts, written for every row by the level pass (no zero fill: first
  // touched by the threads that use them)
  std::unique_ptr<int[]> cL(new int[std::max(n, 1)]), cU(new int[std::max(n, 1)]);
  const int* rp = A.rowptr;
  const int* ci = A.col;
  const int cb = A.istart;
  int* lev = lev_out;
  // one core is left to the caller's other threads: a plan thread that the scheduler
  // pre-empts for a time slice would hold up the whole loop
  const int nthr = std::max(1, omp_get_num_procs() - 1);
  // blocks are handed out in runs: one at a time when there are few (large) blocks, about
  // 32 runs per thread when there are tens of thousands of small ones, so that the
  // per-level counters of neighbouring blocks are mostly written by one thread
  const int grain = std::max(1, nb / (32 * nthr));
#pragma omp parallel num_threads(nthr)
  {
    std::vector<int> lb, lsrc;   // this thread's scratch, reused across its blocks
#pragma omp for schedule(dynamic, grain)
    for (int b = 0; b < nb; ++b) {
      if (block_ready) block_ready(b);
      const int lo = P.blk_lo[b], hi = P.blk_hi[b];
      lb.assign(hi - lo, 0);
      lsrc.assign(hi - lo, INT_MAX);
      int maxlev = 0, g = 0;
      for (int i = lo; i < hi; ++i) {
        // columns are sorted: the lower entries come first, so the row's level is final at
        // its first upper entry and one walk over the row suffices
        int L = lb[i - lo];
        int nl = 0, nu = 0, lmin = lsrc[i - lo];
        bool diag = false, fixed = false, unsorted = false;
        for (int j = rp[i] - 1; j < rp[i + 1] - 1; ++j) {
          const int c = ci[j] - cb;
          if (c < lo || c >= hi) continue;
          if (c < i) {
            unsorted |= fixed;
            L = std::max(L, lev[c] + 1);
            lmin = std::min(lmin, lev[c]);
            ++nl;
          } else if (c == i) {
            diag = true;
          } else {
            fixed = true;
            // an upper entry (i, c) makes c wait for i in the backward sweep order as well
            lb[c - lo] = std::max(lb[c - lo], L + 1);
            lsrc[c - lo] = std::min(lsrc[c - lo], L);
            ++nu;
          }
        }
        if (unsorted)   // a lower entry after an upper one: redo the upper entries with the final level
          for (int j = rp[i] - 1; j < rp[i + 1] - 1; ++j) {
            const int c = ci[j] - cb;
            if (c > i && c < hi) {
              lb[c - lo] = std::max(lb[c - lo], L + 1);
              lsrc[c - lo] = std::min(lsrc[c - lo], L);   // an earlier, smaller L only widens W
            }
          }
        if (!diag) missing_diag[b] = 1;
        lev[i] = L;
        cL[i] = nl; cU[i] = nu;
        maxlev = std::max(maxlev, L);
        if (lmin != INT_MAX) g = std::max(g, L - lmin);
      }
      nlev[b] = maxlev + 1;
      gap[b] = g;
    }
  }
  for (int b = 0; b < nb; ++b)
    if (missing_diag[b]) {
      set_last_error(PARCEL_B_E_ZERO_PIVOT,
                     "block-Jacobi block %d has a row without an in-block diagonal entry", b);
      throw Error{PARCEL_B_E_ZERO_PIVOT, "missing diagonal"};
    }
  // level widths and coupling counts
  P.blk_lvl.assign(nb + 1, 0);
  for (int b = 0; b < nb; ++b) P.blk_lvl[b + 1] = P.blk_lvl[b] + nlev[b];
  const int totlev = P.blk_lvl[nb];
  std::unique_ptr<int[]> width(new int[std::max(totlev, 1)]), kl(new int[std::max(totlev, 1)]),
      ku(new int[std::max(totlev, 1)]);   // zeroed block by block below
  // per block: its span in the permuted layout (every level starts on a multiple of 4, so a
  // block that starts on one spans the sum of its rounded-up widths) and its chunks (a level
  // split at kIluChunk rows)
  std::vector<int64_t> span(nb + 1, 0);
  std::vector<int> nchunk(nb + 1, 0);
#pragma omp parallel for schedule(dynamic, grain) num_threads(nthr)
  for (int b = 0; b < nb; ++b) {   // blocks own disjoint level ranges
    const int l0 = P.blk_lvl[b];
    for (int l = 0; l < nlev[b]; ++l) width[l0 + l] = kl[l0 + l] = ku[l0 + l] = 0;
    for (int i = P.blk_lo[b]; i < P.blk_hi[b]; ++i) {
      const int gl = l0 + lev[i];
      width[gl]++;
      kl[gl] = std::max(kl[gl], cL[i]);
      ku[gl] = std::max(ku[gl], cU[i]);
    }
    int64_t sp = 0;
    int nc = 0;
    for (int l = 0; l < nlev[b]; ++l) {
      sp += align4(width[l0 + l]);
      nc += (width[l0 + l] + kIluChunk - 1) / kIluChunk;
    }
    span[b + 1] = sp;
    nchunk[b + 1] = nc;
  }
  for (int b = 0; b < nb; ++b) {
    span[b + 1] += span[b];
    nchunk[b + 1] += nchunk[b];
  }
  PB_CHECK(span[nb] <= INT_MAX - 3, PARCEL_B_E_ARG, "the permuted layout of %d rows exceeds 2^31 entries", n);
  P.lvl_start.assign(totlev, 0);
  P.lvl_end.assign(totlev, 0);
  P.blk_chunk.assign(nchunk.begin(), nchunk.end());
  P.chunks.resize(nchunk[nb]);
  int maxw = 0;
  // level starts, positions (stable by natural index within a level) and chunks, in block
  // order
#pragma omp parallel for schedule(dynamic, grain) num_threads(nthr) reduction(max : maxw)
  for (int b = 0; b < nb; ++b) {
    const int l0 = P.blk_lvl[b];
    int cursor = (int)span[b];
    int c = P.blk_chunk[b];
    for (int l = 0; l < nlev[b]; ++l) {
      const int gl = l0 + l, w = width[gl];
      P.lvl_start[gl] = cursor;
      P.lvl_end[gl] = cursor + w;
      maxw = std::max(maxw, w);
      for (int o = 0; o < w; o += kIluChunk) {
        IluChunk& C = P.chunks[c++];
        C.start = cursor + o;
        C.w = std::min(kIluChunk, w - o);
        C.wpad = align4(C.w);
        C.KL = kl[gl];
        C.KU = ku[gl];
        C.lvl = l;
        C.off_in_level = o;
        C.blk = b;
        C.offF = 0;
        C.offB = 0;
      }
      cursor = align4(cursor + w);
    }
    for (int l = 0; l < nlev[b]; ++l) width[l0 + l] = 0;   // reused as the fill counters
    for (int i = P.blk_lo[b]; i < P.blk_hi[b]; ++i) {
      const int gl = l0 + lev[i];
      pos_out[i] = P.lvl_start[gl] + width[gl]++;
    }
  }
  // the last level of the last block is not padded at its end
  P.np = nb > 0 ? align4(P.lvl_end[totlev - 1]) : 0;
  P.maxWp = align4(maxw);
  P.max_levels = nb > 0 ? *std::max_element(nlev.begin(), nlev.end()) : 0;
  P.W = (nb > 0 ? *std::max_element(gap.begin(), gap.end()) : 0) + 1;
}


// ------------------------------------------------------------------ factorisation
// In-block column range of natural row i (columns sorted): [first, last) positions.
__device__ __forceinline__ void inblock_range(const int* rp, const int* ci, int rbase, int cbase,
                                              int i, int lo, int hi, int* ja, int* jz, int* jd) {
  int a = rp[i] - rbase, z = rp[i + 1] - rbase;
  int s = z, e = z, d = -1;
  for (int j = a; j < z; ++j) {
    int c = ci[j] - cbase;
    if (c >= lo && s == z) s = j;
    if (c >= hi) { e = j; break; }
    if (c == i) d = j;
  }
  if (s > e) s = e;
  *ja = s; *jz = e; *jd = d;
}

// ILU(0) IKJ factorisation of every block, level by level; one CTA per block.
// ILU_LU_crs (matrix.f90:7970-8072).  Explicit roundings keep the reference's
// two-rounding a - b*c.
//
// A row of at most kFacCap entries is staged in registers: its columns and values in one
// batch of loads, then for each lower in-block entry (increasing column) the pivot row in
// one batch; the eliminations run on the registers in the reference's order and the row
// is written back once.  Longer rows (or pivot rows) take the entry-by-entry path.
constexpr int kFacCap = 8;

__device__ __forceinline__ void ilu0_row_generic(const int* rp, const int* ci, int rbase, int cbase, int i, int lo, int hi,
                                 double* lu) {
  int ia, iz, idg;
  inblock_range(rp, ci, rbase, cbase, i, lo, hi, &ia, &iz, &idg);
  for (int kc = ia; kc < iz; ++kc) {
    int k = ci[kc] - cbase;
    if (k > i - 1) break;
    int ka, kz, kk;
    inblock_range(rp, ci, rbase, cbase, k, lo, hi, &ka, &kz, &kk);
    double lik = __ddiv_rn(lu[kc], lu[kk]);
    lu[kc] = lik;
    for (int jc = kc + 1; jc < iz; ++jc) {
      int j = ci[jc] - cbase;
      for (int kj = kk; kj < kz; ++kj) {
        int cj = ci[kj] - cbase;
        if (cj == j) { lu[jc] = __dsub_rn(lu[jc], __dmul_rn(lik, lu[kj])); break; }
        if (cj > j) break;
      }
    }
  }
}

__global__ void k_ilu0_factor(const IluChunk* __restrict__ ch, const int* __restrict__ blk_chunk,
                              const int* __restrict__ blk_lo, const int* __restrict__ blk_hi,
                              const int* __restrict__ rowAt, const int* __restrict__ rp,
                              const int* __restrict__ ci, int rbase, int cbase, double* lu) {
  const int b = blockIdx.x;
  const int lo = blk_lo[b], hi = blk_hi[b];
  for (int c = blk_chunk[b]; c < blk_chunk[b + 1]; ++c) {
    const IluChunk C = ch[c];
    for (int p = threadIdx.x; p < C.w; p += blockDim.x) {
      const int i = rowAt[C.start + p];
      const int a = rp[i] - rbase, z = rp[i + 1] - rbase;
      if (z - a > kFacCap) {
        ilu0_row_generic(rp, ci, rbase, cbase, i, lo, hi, lu);
        continue;
      }
      int col[kFacCap];
      double val[kFacCap];
#pragma unroll
      for (int e = 0; e < kFacCap; ++e) {
        col[e] = e < z - a ? ci[a + e] - cbase : INT_MAX;
        val[e] = e < z - a ? lu[a + e] : 0.0;
      }
      // pivot rows must fit as well; otherwise the whole row goes the generic way.  Their
      // bounds are kept for the eliminations.
      bool fits = true;
      int pa[kFacCap], pz[kFacCap];
#pragma unroll
      for (int e = 0; e < kFacCap; ++e) {
        const int k = col[e];
        pa[e] = 0;
        pz[e] = 0;
        if (k >= lo && k < i) {
          pa[e] = rp[k] - rbase;
          pz[e] = rp[k + 1] - rbase;
          if (pz[e] - pa[e] > kFacCap) fits = false;
        }
      }
      if (!fits) {
        ilu0_row_generic(rp, ci, rbase, cbase, i, lo, hi, lu);
        continue;
      }
      // e walks the row; the register arrays are only ever indexed by unrolled loops
      for (int e = 0; e < z - a; ++e) {
        int k = INT_MAX, ka = 0, kz = 0;
        double ve = 0.0;
#pragma unroll
        for (int q = 0; q < kFacCap; ++q)
          if (q == e) { k = col[q]; ve = val[q]; ka = pa[q]; kz = pz[q]; }
        if (k < lo || k >= i) continue;   // lower in-block entries only, increasing column
        int kcol[kFacCap];
        double kval[kFacCap];
#pragma unroll
        for (int f = 0; f < kFacCap; ++f) {
          kcol[f] = f < kz - ka ? ci[ka + f] - cbase : INT_MAX;
          kval[f] = f < kz - ka ? lu[ka + f] : 0.0;
        }
        double ukk = 0.0;
#pragma unroll
        for (int f = 0; f < kFacCap; ++f)
          if (kcol[f] == k) ukk = kval[f];
        const double lik = __ddiv_rn(ve, ukk);
        // l_ik replaces a_ik; the in-block entries after it lose l_ik u_kj where row k
        // has column j (> k)
#pragma unroll
        for (int g = 0; g < kFacCap; ++g) {
          if (g == e) val[g] = lik;
          const int j = col[g];
#pragma unroll
          for (int f = 0; f < kFacCap; ++f)
            if (g > e && kcol[f] == j && j > k && j < hi) val[g] = __dsub_rn(val[g], __dmul_rn(lik, kval[f]));
        }
      }
#pragma unroll
      for (int e = 0; e < kFacCap; ++e)
        if (e < z - a) lu[a + e] = val[e];
    }
    __syncthreads();
  }
}

__global__ void k_dilu_diag(const IluChunk* __restrict__ ch, const int* __restrict__ blk_chunk,
                            const int* __restrict__ blk_lo, const int* __restrict__ blk_hi,
                            const int* __restrict__ rowAt, const int* __restrict__ rp,
                            const int* __restrict__ ci, const double* __restrict__ va, int rbase,
                            int cbase, int mlud, double* D, double* Dinv) {
  const int b = blockIdx.x;
  const int lo = blk_lo[b], hi = blk_hi[b];
  for (int c = blk_chunk[b]; c < blk_chunk[b + 1]; ++c) {
    const IluChunk C = ch[c];
    for (int p = threadIdx.x; p < C.w; p += blockDim.x) {
      int k = rowAt[C.start + p];
      int ia, iz, idg;
      inblock_range(rp, ci, rbase, cbase, k, lo, hi, &ia, &iz, &idg);
      double d = va[idg];
      for (int jr = ia; jr < idg; ++jr) {
        int kr = ci[jr] - cbase;
        int ra, rz, rd;
        inblock_range(rp, ci, rbase, cbase, kr, lo, hi, &ra, &rz, &rd);
        double dk = D[kr];
        for (int i = ra; i < rz; ++i) {
          int rc = ci[i] - cbase;
          if (!mlud) {
            if (rc == k) { d = __dsub_rn(d, __ddiv_rn(__dmul_rn(va[jr], va[i]), dk)); break; }
          } else if (kr < rc) {
            d = __dsub_rn(d, __ddiv_rn(__dmul_rn(va[jr], va[i]), dk));
          }
        }
      }
      D[k] = d;
      Dinv[k] = __ddiv_rn(1.0, d);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ packing
// Packed chunk layout (bytes, every section 16-byte aligned):
//   header int[8] = {start, w, wpad, K, lvl, off_in_level, 0, 0}
//   header int[6] = ring offset of the chunk's first row: (lvl % W) * maxWp + off_in_level
//   diag   T[wpad]          forward: 1 (ILU(0)) or D^-1 (D-ILU); backward: 1/U_kk or D^-1
//   val    T[K * wpad]      entry k of row p at k*wpad + p
//   slot   int[K * wpad]    ring slot (or permuted position) of the coupled row, -1 = none
template <class T>
__host__ __device__ inline int64_t chunk_bytes(int wpad, int K) {
  return kIluHeader + (int64_t)wpad * sizeof(T) * (1 + K) + (int64_t)4 * K * wpad;
}

template <class T>
__global__ void k_ilu_pack(const IluChunk* __restrict__ ch, int nchunks,
                           const int* __restrict__ blk_lo, const int* __restrict__ blk_hi,
                           const int* __restrict__ blk_lvl, const int* __restrict__ lvl_start,
                           const int* __restrict__ rowAt, const int* __restrict__ pos,
                           const int* __restrict__ lev, const int* __restrict__ rp,
                           const int* __restrict__ ci, int rbase, int cbase,
                           const double* __restrict__ vL,    // values of L entries
                           const double* __restrict__ vU,    // values of U entries
                           const double* __restrict__ Dinv,  // D-ILU only
                           int dilu, int ring, int W, int maxWp,
                           unsigned char* packF, unsigned char* packB) {
  for (int c = blockIdx.x; c < nchunks; c += gridDim.x) {
    const IluChunk C = ch[c];
    const int lo = blk_lo[C.blk], hi = blk_hi[C.blk];
    unsigned char* f = packF + C.offF;
    unsigned char* g = packB + C.offB;
    if (threadIdx.x == 0) {
      int* hf = (int*)f;
      int* hb = (int*)g;
      hf[0] = C.start; hf[1] = C.w; hf[2] = C.wpad; hf[3] = C.KL; hf[4] = C.lvl;
      hf[5] = C.off_in_level; hf[6] = (C.lvl % W) * maxWp + C.off_in_level; hf[7] = 0;
      hb[0] = C.start; hb[1] = C.w; hb[2] = C.wpad; hb[3] = C.KU; hb[4] = C.lvl;
      hb[5] = C.off_in_level; hb[6] = (C.lvl % W) * maxWp + C.off_in_level; hb[7] = 0;
    }
    T* dF = (T*)(f + kIluHeader);
    T* valF = dF + C.wpad;
    int* slF = (int*)(valF + (size_t)C.KL * C.wpad);
    T* dB = (T*)(g + kIluHeader);
    const int zslot = ring ? W * maxWp : -1;   // ring mode: a slot that always holds 0
    T* valB = dB + C.wpad;
    int* slB = (int*)(valB + (size_t)C.KU * C.wpad);
    for (int p = threadIdx.x; p < C.wpad; p += blockDim.x) {
      if (p >= C.w) {
        dF[p] = (T)0; dB[p] = (T)0;
        for (int k = 0; k < C.KL; ++k) { valF[k * C.wpad + p] = (T)0; slF[k * C.wpad + p] = zslot; }
        for (int k = 0; k < C.KU; ++k) { valB[k * C.wpad + p] = (T)0; slB[k * C.wpad + p] = zslot; }
        continue;
      }
      int i = rowAt[C.start + p];
      int ia, iz, idg;
      inblock_range(rp, ci, rbase, cbase, i, lo, hi, &ia, &iz, &idg);
      auto slot_of = [&](int cnat) -> int {
        int q = pos[cnat];
        if (!ring) return q;
        int l = lev[cnat];
        return (l % W) * maxWp + (q - lvl_start[blk_lvl[C.blk] + l]);
      };
      // forward: strictly lower in-block entries, increasing column
      int k = 0;
      for (int j = ia; j < idg; ++j, ++k) {
        valF[k * C.wpad + p] = (T)vL[j];
        slF[k * C.wpad + p] = slot_of(ci[j] - cbase);
      }
      for (; k < C.KL; ++k) { valF[k * C.wpad + p] = (T)0; slF[k * C.wpad + p] = zslot; }
      dF[p] = dilu ? (T)Dinv[i] : (T)1;
      // backward: strictly upper in-block entries; ILU(0) increasing column
      // (solve_LU_crs), D-ILU decreasing column (solve_ILU_crs runs Ustart down to Uend)
      k = 0;
      if (!dilu) {
        for (int j = idg + 1; j < iz; ++j, ++k) {
          valB[k * C.wpad + p] = (T)vU[j];
          slB[k * C.wpad + p] = slot_of(ci[j] - cbase);
        }
        dB[p] = (T)(1.0 / vU[idg]);   // reciprocal of U_kk: the sweep multiplies
      } else {
        for (int j = iz - 1; j > idg; --j, ++k) {
          valB[k * C.wpad + p] = (T)vU[j];
          slB[k * C.wpad + p] = slot_of(ci[j] - cbase);
        }
        dB[p] = (T)Dinv[i];
      }
      for (; k < C.KU; ++k) { valB[k * C.wpad + p] = (T)0; slB[k * C.wpad + p] = zslot; }
    }
  }
}

// ------------------------------------------------------------------ grouped sweep
// The fast sweep streams GROUPS of consecutive chunks (levels, or 512-row pieces of a
// level) of one block: one bulk copy of the group's packed record plus one of its slice of
// the input vector fills one shared-memory stage, so the consumers wait on a stage
// barrier once per group and, between levels, pass only the level barrier.  The rows of a
// group are contiguous in the permuted layout ([sstart, sstart + sspan)).  Group record:
//   int4 hdr              {nchunks, sstart, sspan, 0}
//   int4 cd[kGrpMax][2]   per chunk in sweep order: {rec, w, ring, gs}, {xin, 0, 0, 0}:
//                         stage byte offsets of the first row's row record and input
//                         value, rows, ring byte offset of the first row, permuted
//                         position of the first row
//   row records           one per position of the span, `stride` bytes apart:
//                           T dg        1/U_kk or D^-1 (backward sweep, forward D-ILU only)
//                           T val[K]    coupled coefficients in the reference's order
//                           u16 slot[K] ring byte offsets of the coupled rows (the ring's
//                                       zero slot for padding)
//                         padded to an odd number of T-sized words, so that the 32 lanes
//                         of a warp reading consecutive records hit distinct banks.
// The stage holds T xin[sspan] (the input slice) after the records, 16-byte aligned.
// Positions without a row (level padding) have zero records.
constexpr int kGrpMax = 15;
constexpr int kGrpHdr = 512;   // 16 + kGrpMax * 32, rounded up

__host__ __device__ constexpr int rec_words(int tsize, bool has_dg, int K) {
  return ((has_dg ? 1 : 0) + K + (2 * K + tsize - 1) / tsize) | 1;
}
__host__ __device__ constexpr int rec_stride(int tsize, bool has_dg, int K) {
  return rec_words(tsize, has_dg, K) * tsize;
}

// Packs the group records of the grouped sweep (layout above): one CTA per group;
// gi[g] = {first chunk, end chunk, sstart, sspan}, goff[g] = byte offsets of the forward
// and backward records.
template <class T>
__global__ void k_ilu_pack_grp(const int4* __restrict__ gi, const int64_t* __restrict__ goff, int ngroups,
                               const IluChunk* __restrict__ ch, const int* __restrict__ blk_lo,
                               const int* __restrict__ blk_hi, const int* __restrict__ blk_lvl,
                               const int* __restrict__ lvl_start, const int* __restrict__ rowAt,
                               const int* __restrict__ pos, const int* __restrict__ lev,
                               const int* __restrict__ rp, const int* __restrict__ ci, int rbase, int cbase,
                               const double* __restrict__ vL, const double* __restrict__ vU,
                               const double* __restrict__ Dinv, int dilu, int W, int maxWp, int K,
                               unsigned char* packF, unsigned char* packB) {
  const int sz = (int)sizeof(T);
  const int zslot = W * maxWp * sz;   // byte offset of the ring's zero slot
  const int strF = rec_stride(sz, dilu != 0, K), strB = rec_stride(sz, true, K);
  for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
    const int4 G = gi[g];
    const int c0 = G.x, c1 = G.y, sstart = G.z, sspan = G.w;
    const int nch = c1 - c0;
    const int blk = ch[c0].blk;
    const int lo = blk_lo[blk], hi = blk_hi[blk];
    unsigned char* f = packF + goff[2 * g];
    unsigned char* bk = packB + goff[2 * g + 1];
    const int xF = kGrpHdr + (int)(((int64_t)sspan * strF + 15) & ~int64_t(15));
    const int xB = kGrpHdr + (int)(((int64_t)sspan * strB + 15) & ~int64_t(15));
    for (int t = threadIdx.x; t < kGrpHdr / 16; t += blockDim.x) {
      int4 hf = make_int4(0, 0, 0, 0), hb = make_int4(0, 0, 0, 0);
      const int j = (t - 1) >> 1, half = (t - 1) & 1;
      if (t == 0) {
        hf = make_int4(nch, sstart, sspan, 0);
        hb = hf;
      } else if (j < nch) {
        const IluChunk& cf = ch[c0 + j];       // forward: increasing level
        const IluChunk& cb = ch[c1 - 1 - j];   // backward: decreasing level
        if (half == 0) {
          hf = make_int4(kGrpHdr + (cf.start - sstart) * strF, cf.w,
                         ((cf.lvl % W) * maxWp + cf.off_in_level) * sz, cf.start);
          hb = make_int4(kGrpHdr + (cb.start - sstart) * strB, cb.w,
                         ((cb.lvl % W) * maxWp + cb.off_in_level) * sz, cb.start);
        } else {
          hf = make_int4(xF + (cf.start - sstart) * sz, 0, 0, 0);
          hb = make_int4(xB + (cb.start - sstart) * sz, 0, 0, 0);
        }
      }
      reinterpret_cast<int4*>(f)[t] = hf;
      reinterpret_cast<int4*>(bk)[t] = hb;
    }
    for (int i = threadIdx.x; i < sspan; i += blockDim.x) {
      unsigned char* rf = f + kGrpHdr + (size_t)i * strF;
      unsigned char* rb = bk + kGrpHdr + (size_t)i * strB;
      for (int o = 0; o < strF; o += 4) *reinterpret_cast<int*>(rf + o) = 0;
      for (int o = 0; o < strB; o += 4) *reinterpret_cast<int*>(rb + o) = 0;
      T* valF = reinterpret_cast<T*>(rf + (dilu ? sz : 0));
      unsigned short* slF = reinterpret_cast<unsigned short*>(rf + (dilu ? sz : 0) + K * sz);
      T* valB = reinterpret_cast<T*>(rb + sz);
      unsigned short* slB = reinterpret_cast<unsigned short*>(rb + sz + K * sz);
      const int nat = rowAt[sstart + i];
      if (nat < 0) {
        for (int k = 0; k < K; ++k) { slF[k] = (unsigned short)zslot; slB[k] = (unsigned short)zslot; }
        continue;
      }
      int ia, iz, idg;
      inblock_range(rp, ci, rbase, cbase, nat, lo, hi, &ia, &iz, &idg);
      auto slot_of = [&](int cnat) -> int {
        const int l = lev[cnat];
        return ((l % W) * maxWp + (pos[cnat] - lvl_start[blk_lvl[blk] + l])) * sz;
      };
      // forward: strictly lower in-block entries, increasing column
      int k = 0;
      for (int j = ia; j < idg; ++j, ++k) {
        valF[k] = (T)vL[j];
        slF[k] = (unsigned short)slot_of(ci[j] - cbase);
      }
      for (; k < K; ++k) slF[k] = (unsigned short)zslot;
      if (dilu) *reinterpret_cast<T*>(rf) = (T)Dinv[nat];
      // backward: strictly upper in-block entries; ILU(0) increasing column
      // (solve_LU_crs), D-ILU decreasing column (solve_ILU_crs runs Ustart down to Uend)
      k = 0;
      if (!dilu) {
        for (int j = idg + 1; j < iz; ++j, ++k) {
          valB[k] = (T)vU[j];
          slB[k] = (unsigned short)slot_of(ci[j] - cbase);
        }
        *reinterpret_cast<T*>(rb) = (T)(1.0 / vU[idg]);   // reciprocal of U_kk: the sweep multiplies
      } else {
        for (int j = iz - 1; j > idg; --j, ++k) {
          valB[k] = (T)vU[j];
          slB[k] = (unsigned short)slot_of(ci[j] - cbase);
        }
        *reinterpret_cast<T*>(rb) = (T)Dinv[nat];
      }
      for (; k < K; ++k) slB[k] = (unsigned short)zslot;
    }
  }
}

// ------------------------------------------------------------------ the sweep kernel
constexpr int kIluProducerWarps = 1;
constexpr int kIluConsumerThreads = 256;
constexpr int kIluThreads = 32 * kIluProducerWarps + kIluConsumerThreads;
constexpr unsigned kWaitLimit = 1u << 20;   // polls of one mbarrier wait before giving up
constexpr int kIluKUnroll = 4;            // coupled entries gathered per step

// What the producer needs per chunk, in the order it streams them:
// {packed offset / 16, first permuted row, packed bytes, vector-slice bytes}.
struct ProdDesc { int off16, start, cbytes, vbytes; };

template <class T>
struct IluSolveArgs {
  const ProdDesc* tabF;   // per chunk, forward order
  const ProdDesc* tabB;   // per chunk, forward order (read backwards)
  const int* blk_chunk;
  const unsigned char* packF;
  const unsigned char* packB;
  const T* r;
  T* y;
  T* s;
  T* accum;
  int W, maxWp, stage_bytes, nstages, ring_elems;
  const int* gate;
  int* err;
};

constexpr int kBarLevel = 1;                      // consumers, once per chunk
constexpr int kBarTurn = 2;                       // consumers -> producer: forward sweep written
constexpr int kBarStage0 = 3;                     // consumers -> producer: stage s free (id 3 + s)
constexpr int kGrpMaxStages = 12;                 // named barrier ids 3..14

// Producer descriptor of one group: {packed offset / 16, record bytes, first permuted
// position, vector-slice bytes}.
struct GrpDesc { int off16, cbytes, start, vbytes; };

template <class T>
struct GrpArgs {
  const GrpDesc* tabF;   // per group, forward order
  const GrpDesc* tabB;   // per group, forward order (the backward sweep walks it backwards)
  const int* blk_grp;    // nb + 1
  const unsigned char* packF;
  const unsigned char* packB;
  const T* r;
  T* y;
  T* s;
  int stage_bytes, nstages, ring_elems;
  const int* gate;
  int* err;
};

// Operands of the R rows (p, p + NC, ...) a consumer thread owns in one chunk, staged in
// registers one chunk ahead: coefficients, the input values, the shared-memory addresses
// of the coupled ring values and of the row's own ring slot, and the output address.
// Every chunk carries exactly KM coupled entries per row (shorter rows point at the ring's
// zero slot), so the loops have compile-time trip counts.
template <class T, int KM, int R>
struct GOps {
  T xin[R], dg[R];
  T val[R][KM];
  uint32_t gaddr[R][KM];
  uint32_t waddr;
  T* gout;
  int w;
};

__device__ __forceinline__ void named_bar_arrive(int id, int nthreads) {
  asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Shared-memory accesses that the compiler keeps in program order ("memory" clobber): the
// ring gathers of a level are issued before the next chunk's operand loads, so they do not
// queue behind them.
__device__ __forceinline__ double lds_ord(uint32_t a, double) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ float lds_ord(uint32_t a, float) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a) : "memory");
  return v;
}
__device__ __forceinline__ void sts(uint32_t a, double v) {
  asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void sts(uint32_t a, float v) {
  asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}


// The K ring byte offsets of a row record, read as whole T-sized words.
template <class T, int KM>
__device__ __forceinline__ void load_slots(const unsigned char* sp, uint32_t ring_s, uint32_t (&ga)[KM]) {
  if constexpr (sizeof(T) == 8) {
    const unsigned long long* w = reinterpret_cast<const unsigned long long*>(sp);
#pragma unroll
    for (int k0 = 0; k0 < KM; k0 += 4) {
      const unsigned long long v = w[k0 / 4];
#pragma unroll
      for (int k = k0; k < KM && k < k0 + 4; ++k) ga[k] = ring_s + (uint32_t)((v >> (16 * (k - k0))) & 0xffffu);
    }
  } else {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(sp);
#pragma unroll
    for (int k0 = 0; k0 < KM; k0 += 2) {
      const uint32_t v = w[k0 / 2];
      ga[k0] = ring_s + (v & 0xffffu);
      if (k0 + 1 < KM) ga[k0 + 1] = ring_s + (v >> 16);
    }
  }
}

template <class T, bool HAS_DG, int KM, int R, int NC>
__device__ __forceinline__ void gload(GOps<T, KM, R>& o, const unsigned char* sp, int j, int p, uint32_t ring_s,
                                      T* vout) {
  constexpr int STR = rec_stride((int)sizeof(T), HAS_DG, KM);
  constexpr int VOFF = HAS_DG ? (int)sizeof(T) : 0;
  constexpr int SOFF = VOFF + KM * (int)sizeof(T);
  const int4 c0 = reinterpret_cast<const int4*>(sp)[1 + 2 * j];
  const int xoff = reinterpret_cast<const int*>(sp)[4 * (2 + 2 * j)];
  o.w = c0.y;
  o.waddr = ring_s + (uint32_t)c0.z + (uint32_t)(p * (int)sizeof(T));
  o.gout = vout + c0.w + p;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int q = p + r * NC;
    if (q < o.w) {
      const unsigned char* rec = sp + c0.x + q * STR;
      o.xin[r] = *reinterpret_cast<const T*>(sp + xoff + q * (int)sizeof(T));
      o.dg[r] = HAS_DG ? *reinterpret_cast<const T*>(rec) : T(1);
#pragma unroll
      for (int k = 0; k < KM; ++k) o.val[r][k] = reinterpret_cast<const T*>(rec + VOFF)[k];
      load_slots<T, KM>(rec + SOFF, ring_s, o.gaddr[r]);
    }
  }
}

template <class T, int KM, int R, int NC>
__device__ __forceinline__ void ggather(const GOps<T, KM, R>& c, int p, T (&dv)[R][KM]) {
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (p + r * NC < c.w) {
#pragma unroll
      for (int k = 0; k < KM; ++k) dv[r][k] = lds_ord(c.gaddr[r][k], T(0));
    }
}

template <class T, bool DILU, bool FWD, int KM, int R, int NC>
__device__ __forceinline__ void gsolve(const GOps<T, KM, R>& c, const T (&dv)[R][KM], int p) {
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (p + r * NC >= c.w) continue;
    T acc = (FWD || !DILU) ? c.xin[r] : T(0);
#pragma unroll
    for (int k = 0; k < KM; ++k) {
      if (FWD) acc = acc - c.val[r][k] * dv[r][k];
      else if (DILU) acc = acc + dv[r][k] * c.val[r][k];
      else acc = acc - dv[r][k] * c.val[r][k];
    }
    T out;
    if (FWD) out = DILU ? c.dg[r] * acc : acc;
    else if (DILU) out = c.xin[r] - c.dg[r] * acc;
    else out = acc * c.dg[r];
    sts(c.waddr + (uint32_t)(r * NC * (int)sizeof(T)), out);
    c.gout[r * NC] = out;
  }
}

// Consumer side of one sweep over groups [g0, g0 + ng) of the sequence (NG groups over both
// sweeps).  Per chunk: gather the coupled values from the ring, load the next chunk's
// operands, finish the rows, and pass the level barrier.  A stage that never landed sets
// the abort flag; every consumer reads it after the barrier that follows a stage wait, so
// all return together (`arrived` tells how far each released stages).
template <class T, bool DILU, bool FWD, int KM, int R, int NC>
__device__ __forceinline__ void gsweep(const GrpArgs<T>& a, uint64_t* full, volatile int* sflags,
                                       unsigned char* stages, uint32_t ring_s, int g0, int ng, int NG, int p,
                                       T* vout, int* arrived) {
  constexpr bool HAS_DG = DILU || !FWD;
  constexpr int NT = NC + 32;
  const int NST = a.nstages;
  if (ng <= 0) return;
  int g = g0, st = g0 % NST, ph = (g0 / NST) & 1, j = 0, nch = 0;
  // Loads the chunk at the cursor into o (waiting for its group's stage when the cursor
  // has just entered the group), then advances the cursor.  Returns 1 when loaded, 0 at
  // the end of the sweep (the same for every thread), -1 when the stage did not land.
  bool entered = false;   // the last next() waited for a stage (the same for every thread)
  auto next = [&](GOps<T, KM, R>& o) -> int {
    entered = false;
    if (g >= g0 + ng) return 0;
    const unsigned char* sp = stages + (size_t)st * a.stage_bytes;
    if (j == 0) {
      entered = true;
      // warp-uniform outcome, so the aligned barrier instructions below never diverge
      if (!__all_sync(kFull, mbar_wait(&full[st], ph, kWaitLimit))) {
        atomicExch(a.err, 3);
        sflags[0] = 1;
        return -1;
      }
      nch = reinterpret_cast<const int*>(sp)[0];
    }
    gload<T, HAS_DG, KM, R, NC>(o, sp, j, p, ring_s, vout);
    if (++j == nch) {
      // every operand of the group is in this thread's registers: release the stage
      if (g + NST < NG) named_bar_arrive(kBarStage0 + st, NT);
      *arrived = g + 1;
      j = 0;
      ++g;
      if (++st == NST) { st = 0; ph ^= 1; }
    }
    return 1;
  };
  // level barrier; after a stage wait every consumer also reads the abort flag, which a
  // consumer whose wait failed has set before the barrier
  auto level_barrier = [&]() -> bool {
    named_bar_sync(kBarLevel, NC);
    return !(entered && sflags[0]);
  };
  GOps<T, KM, R> A, B;
  T dv[R][KM];
  int sA = next(A), sB = 0;
  if (!level_barrier()) return;
  while (sA > 0) {
    ggather<T, KM, R, NC>(A, p, dv);
    sB = next(B);
    gsolve<T, DILU, FWD, KM, R, NC>(A, dv, p);
    if (!level_barrier() || sB == 0) return;
    ggather<T, KM, R, NC>(B, p, dv);
    sA = next(A);
    gsolve<T, DILU, FWD, KM, R, NC>(B, dv, p);
    if (!level_barrier()) return;
  }
}

template <class T, bool DILU, int KM, int R, int NC>
__global__ void __launch_bounds__(NC + 32, 1) k_ilu_sweep_grp(GrpArgs<T> a) {
  if (gated(a.gate)) return;
  constexpr int NT = NC + 32;
  extern __shared__ __align__(128) unsigned char smem[];
  const int NST = a.nstages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  volatile int* sflags = reinterpret_cast<volatile int*>(full + kGrpMaxStages);
  T* ring = reinterpret_cast<T*>(smem + 128);
  unsigned char* stages =
      reinterpret_cast<unsigned char*>(ring) + (((size_t)a.ring_elems * sizeof(T) + 127) & ~size_t(127));
  const int b = blockIdx.x;
  const int c0 = a.blk_grp[b], c1 = a.blk_grp[b + 1];
  const int nGF = c1 - c0, NG = 2 * nGF;
  if (threadIdx.x == 0) {
    for (int i = 0; i < NST; ++i) mbar_init(&full[i], 1);
    sflags[0] = 0;
    mbar_fence_init();
  }
  for (int i = threadIdx.x; i < a.ring_elems; i += blockDim.x) ring[i] = T(0);
  __syncthreads();
  if (threadIdx.x >= NC) {
    // Producer warp: lane 0 fills stage g % NST with group g once the consumers have
    // released the stage (named barrier kBarStage0 + stage: a hardware wait, no polling).
    // A backward group's slice of y can only be copied once the forward sweep has
    // written it (barrier kBarTurn), so before that only its record is copied.
    const bool lead = threadIdx.x == NC;
    int issued = 0;     // groups whose copies were issued
    bool turned = false;
    auto desc = [&](int g) -> GrpDesc { return g < nGF ? a.tabF[c0 + g] : a.tabB[c1 - 1 - (g - nGF)]; };
    auto turn = [&]() {
      named_bar_sync(kBarTurn, NT);
      turned = true;
      if (lead)
        for (int g = nGF; g < issued; ++g) {
          const GrpDesc d = desc(g);
          bulk_g2s(stages + (size_t)(g % NST) * a.stage_bytes + d.cbytes, a.y + d.start, (unsigned)d.vbytes,
                   &full[g % NST]);
        }
    };
    for (int g = 0; g < NG; ++g) {
      if (g == nGF + NST && !turned) turn();
      if (g >= NST) named_bar_sync(kBarStage0 + g % NST, NT);
      if (sflags[0]) continue;   // aborted: keep the barrier sequence, issue nothing
      if (lead) {
        const GrpDesc d = desc(g);
        const int st = g % NST;
        unsigned char* dst = stages + (size_t)st * a.stage_bytes;
        const bool fwd = g < nGF;
        mbar_arrive_expect_tx(&full[st], (unsigned)(d.cbytes + d.vbytes));
        bulk_g2s(dst, (fwd ? a.packF : a.packB) + (size_t)d.off16 * 16, (unsigned)d.cbytes, &full[st]);
        if (fwd) bulk_g2s(dst + d.cbytes, a.r + d.start, (unsigned)d.vbytes, &full[st]);
        else if (turned) bulk_g2s(dst + d.cbytes, a.y + d.start, (unsigned)d.vbytes, &full[st]);
      }
      issued = g + 1;
    }
    if (!turned) turn();
    // wait (bounded) for the last copy into every stage, so that no bulk copy is still
    // writing into this CTA's shared memory when it exits
    if (lead)
      for (int g = max(0, issued - NST); g < issued; ++g) mbar_wait(&full[g % NST], (g / NST) & 1, kWaitLimit);
    return;
  }
  const int p = threadIdx.x;
  const uint32_t ring_s = smem_u32(ring);
  int arrived = 0;   // groups (sequence index) whose stage this thread has released
  gsweep<T, DILU, true, KM, R, NC>(a, full, sflags, stages, ring_s, 0, nGF, NG, p, a.y, &arrived);
  // forward result written: make it visible to the producer's bulk copies
  fence_proxy_async_global();
  if (sflags[0]) {
    // aborted: complete the producer's barrier sequence (blocking syncs, in its order)
    for (int g = arrived; g < nGF; ++g)
      if (g + NST < NG) named_bar_sync(kBarStage0 + g % NST, NT);
    arrived = max(arrived, nGF);
    named_bar_sync(kBarTurn, NT);
  } else {
    named_bar_arrive(kBarTurn, NT);
    gsweep<T, DILU, false, KM, R, NC>(a, full, sflags, stages, ring_s, nGF, nGF, NG, p, a.s, &arrived);
  }
  if (sflags[0])
    for (int g = arrived; g < NG; ++g)
      if (g + NST < NG) named_bar_sync(kBarStage0 + g % NST, NT);
}

template <class T, bool DILU, bool RING>
__global__ void __launch_bounds__(kIluThreads, 1) k_ilu_solve(IluSolveArgs<T> a) {
  if (gated(a.gate)) return;
  extern __shared__ __align__(128) unsigned char smem[];
  const int NST = a.nstages;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem);
  uint64_t* empty = full + NST;
  volatile int* sflags = reinterpret_cast<volatile int*>(empty + NST);   // [0] abort, [1] consumed
  T* ring = reinterpret_cast<T*>(smem + ((16 * NST + 16 + 127) & ~127));
  unsigned char* stages =
      reinterpret_cast<unsigned char*>(ring) + (((size_t)a.ring_elems * sizeof(T) + 127) & ~size_t(127));

  const int b = blockIdx.x;
  const int c0 = a.blk_chunk[b], c1 = a.blk_chunk[b + 1];
  const int nc = c1 - c0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const bool producer = warp < kIluProducerWarps;
  const int ctid = threadIdx.x - 32 * kIluProducerWarps;
  int issued = 0;   // producer lane 0: copies issued so far (over both phases)

  if (threadIdx.x == 0) {
    for (int i = 0; i < NST; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
    sflags[0] = 0;
    sflags[1] = 0;
    mbar_fence_init();
  }
  if (RING) {
    for (int i = threadIdx.x; i < a.ring_elems; i += blockDim.x) ring[i] = T(0);
  }
  __syncthreads();

  for (int phase = 0; phase < 2; ++phase) {
    const bool fwd = phase == 0;
    const unsigned char* pack = fwd ? a.packF : a.packB;
    const T* vin = fwd ? a.r : a.y;
    T* vout = fwd ? a.y : a.s;
    const int gbase = phase * nc;
    if (producer) {
      // The whole warp walks the chunk list: 32 descriptors per coalesced load, prefetched
      // one batch ahead and broadcast with shuffles; lane 0 issues the bulk copies.
      const ProdDesc* tab = fwd ? a.tabF : a.tabB;
      auto fetch = [&](int i) -> ProdDesc {
        if (i >= nc) return ProdDesc{0, 0, 0, 0};
        return tab[fwd ? c0 + i : c1 - 1 - i];
      };
      ProdDesc cur = fetch(lane);
      int pst = gbase % NST, puse = gbase / NST;   // stage and reuse count of chunk gbase
      for (int i0 = 0; i0 < nc; i0 += 32) {
        ProdDesc nxt = fetch(i0 + 32 + lane);
        const int kmax = min(32, nc - i0);
        bool stop = false;
        for (int k = 0; k < kmax; ++k) {
          ProdDesc d;
          d.off16 = __shfl_sync(kFull, cur.off16, k);
          d.start = __shfl_sync(kFull, cur.start, k);
          d.cbytes = __shfl_sync(kFull, cur.cbytes, k);
          d.vbytes = __shfl_sync(kFull, cur.vbytes, k);
          if (lane == 0) {
            const int st = pst, use = puse;
            if (++pst == NST) { pst = 0; ++puse; }
            if (sflags[0]) {
              stop = true;
            } else if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1, kWaitLimit)) {
              atomicExch(a.err, 2);
              sflags[0] = 1;
              stop = true;
            } else {
              unsigned char* dst = stages + (size_t)st * a.stage_bytes;
              mbar_arrive_expect_tx(&full[st], (unsigned)(d.cbytes + d.vbytes));
              bulk_g2s(dst, pack + (size_t)d.off16 * 16, (unsigned)d.cbytes, &full[st]);
              bulk_g2s(dst + d.cbytes, vin + d.start, (unsigned)d.vbytes, &full[st]);
              ++issued;
            }
          }
          stop = __shfl_sync(kFull, stop, 0);
          if (stop) break;
        }
        if (stop) break;
        cur = nxt;
      }
    } else {
      for (int i = 0; i < nc; ++i) {
        const int g = gbase + i;
        const int st = g % NST;
        const bool ok = mbar_wait(&full[st], (g / NST) & 1, kWaitLimit);
        if (!ok) {
          atomicExch(a.err, 3);
          sflags[0] = 1;
        } else {
          const unsigned char* sp = stages + (size_t)st * a.stage_bytes;
          const int* hdr = reinterpret_cast<const int*>(sp);
          const int start = hdr[0], w = hdr[1], wpad = hdr[2], K = hdr[3], lvl = hdr[4], off = hdr[5];
          const T* dg = reinterpret_cast<const T*>(sp + kIluHeader);
          const T* val = dg + wpad;
          const int* slot = reinterpret_cast<const int*>(val + (size_t)K * wpad);
          const T* xin = reinterpret_cast<const T*>(sp + chunk_bytes<T>(wpad, K));
          const T* dep = RING ? ring : vout;
          T* rslot = ring + (size_t)(lvl % a.W) * a.maxWp + off;
          for (int p = ctid; p < w; p += kIluConsumerThreads) {
            T out;
            // Gather the K coupled values first (independent loads), then accumulate in
            // the reference's order.
            T dv[kIluKUnroll], av[kIluKUnroll];
            T acc = (fwd || !DILU) ? xin[p] : T(0);
            for (int k0 = 0; k0 < K; k0 += kIluKUnroll) {
#pragma unroll
              for (int u = 0; u < kIluKUnroll; ++u) {
                const int k = k0 + u;
                dv[u] = T(0);
                av[u] = T(0);
                if (k < K) {
                  const int sl = slot[k * wpad + p];
                  av[u] = val[k * wpad + p];
                  if (RING || sl >= 0) dv[u] = dep[sl];
                }
              }
#pragma unroll
              for (int u = 0; u < kIluKUnroll; ++u) {
                if (k0 + u < K) {
                  if (fwd) acc = acc - av[u] * dv[u];
                  else if (DILU) acc = acc + dv[u] * av[u];
                  else acc = acc - dv[u] * av[u];
                }
              }
            }
            if (fwd) out = DILU ? dg[p] * acc : acc;
            else if (DILU) out = xin[p] - dg[p] * acc;
            else out = acc * dg[p];
            if (RING) rslot[p] = out;
            vout[start + p] = out;
            if (!fwd && a.accum) a.accum[start + p] += out;
          }
        }
        named_bar_sync(1, kIluConsumerThreads);
        if (ctid == 0) {
          if (ok) mbar_arrive(&empty[st]);
          sflags[1] = g + 1;
        }
        if (sflags[0]) break;   // uniform: read after the barrier
      }
      if (fwd) fence_proxy_async_global();
    }
    __syncthreads();
    if (sflags[0]) break;
  }
  // After an abort, wait (bounded) for copies that were issued but never consumed so no
  // bulk copy is still writing into this CTA's shared memory when it exits.
  if (sflags[0] && threadIdx.x == 0) {
    for (int g = sflags[1]; g < issued; ++g) mbar_wait(&full[g % NST], (g / NST) & 1, kWaitLimit);
  }
}

// ------------------------------------------------------------------ many small blocks
// A block of a few dozen rows (the 4^3 boxes of a stencil-format matrix: 64 rows on 10
// levels) gives the grouped sweep's one CTA per block too little work for its set-up and
// its 20 dependent level steps; with tens of thousands of blocks the CTAs then run one after
// another.  Here one warp sweeps one block: the rows of a level on the lanes (the levels are
// contiguous in the iteration layout), __syncwarp between levels (it orders the warp's global
// writes before the next level's reads).  The records sit in the iteration layout, K entries
// per row: forward the strictly lower in-block couplings in increasing column, backward the
// strictly upper ones (ILU(0) increasing, D-ILU decreasing column), so each row sums in the
// order of the grouped sweep, with the same expressions.
constexpr int kSmallMaxRows = 1024;   // largest block the warp sweep takes
constexpr int kSmallThreads = 256;

template <class T>
__global__ void k_ilu_small_pack(int n, int nb, const int* __restrict__ blk_lo, const int* __restrict__ blk_hi,
                                 const int* __restrict__ pos, const int* __restrict__ rp, const int* __restrict__ ci,
                                 int rbase, int cbase, const double* __restrict__ vL, const double* __restrict__ vU,
                                 const double* __restrict__ Dinv, int dilu, int K, int* __restrict__ cF,
                                 T* __restrict__ vF, T* __restrict__ dF, int* __restrict__ cB, T* __restrict__ vB,
                                 T* __restrict__ dB) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    int a = 0, z = nb - 1;   // block of row i: the last b with blk_lo[b] <= i
    while (a < z) {
      const int mid = (a + z + 1) >> 1;
      if (blk_lo[mid] <= i) a = mid; else z = mid - 1;
    }
    int ia, iz, idg;
    inblock_range(rp, ci, rbase, cbase, i, blk_lo[a], blk_hi[a], &ia, &iz, &idg);
    const int64_t p = pos[i];
    int k = 0;
    for (int j = ia; j < idg; ++j, ++k) {
      cF[p * K + k] = pos[ci[j] - cbase];
      vF[p * K + k] = (T)vL[j];
    }
    for (; k < K; ++k) { cF[p * K + k] = -1; vF[p * K + k] = T(0); }
    dF[p] = dilu ? (T)Dinv[i] : T(1);
    k = 0;
    if (!dilu) {
      for (int j = idg + 1; j < iz; ++j, ++k) {
        cB[p * K + k] = pos[ci[j] - cbase];
        vB[p * K + k] = (T)vU[j];
      }
      dB[p] = (T)(1.0 / vU[idg]);
    } else {
      for (int j = iz - 1; j > idg; --j, ++k) {
        cB[p * K + k] = pos[ci[j] - cbase];
        vB[p * K + k] = (T)vU[j];
      }
      dB[p] = (T)Dinv[i];
    }
    for (; k < K; ++k) { cB[p * K + k] = -1; vB[p * K + k] = T(0); }
  }
}

// The columns of one row's record (what its gathers wait for), loaded a level ahead.
template <int K>
struct SmallCols {
  int p;        // permuted row, -1: none
  int c[K];
};

template <int K>
__device__ __forceinline__ void small_cols(SmallCols<K>& o, int p, const int* __restrict__ cc) {
  o.p = p;
  if (p < 0) return;
#pragma unroll
  for (int k = 0; k < K; ++k) o.c[k] = cc[(int64_t)p * K + k];
}

// Row p of one sweep: its values, its input x[p] (r forward, y backward) and its diagonal
// factor load beside the gathers of the coupled values, so the row costs one round trip.
template <class T, bool DILU, bool FWD, int K>
__device__ __forceinline__ void small_row(const SmallCols<K>& o, const T* __restrict__ vv, const T* __restrict__ dd,
                                          const T* x, const T* g, T* out) {
  const int p = o.p;
  T v[K], gv[K];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    v[k] = vv[(int64_t)p * K + k];
    gv[k] = o.c[k] >= 0 ? g[o.c[k]] : T(0);
  }
  const T xp = x[p], dp_ = dd[p];
  T acc = (FWD || !DILU) ? xp : T(0);
#pragma unroll
  for (int k = 0; k < K; ++k)
    if (o.c[k] >= 0) {
      if (FWD) acc = acc - v[k] * gv[k];
      else if (DILU) acc = acc + gv[k] * v[k];
      else acc = acc - gv[k] * v[k];
    }
  if (FWD) out[p] = DILU ? dp_ * acc : acc;
  else out[p] = DILU ? xp - dp_ * acc : acc * dp_;
}

// LPB lanes per block, 32 / LPB blocks per warp; y and s are written and re-read across
// levels (no __restrict__ on them).  Each lane loads its next level's columns before it
// works on the current level, so a level costs one dependent round trip.
template <class T, bool DILU, int K, int LPB>
__global__ void __launch_bounds__(kSmallThreads, K <= 3 ? 4 : (K <= 4 ? 3 : 2))
k_ilu_small(int nb, const int* __restrict__ blvl, const int* __restrict__ lo, const int* __restrict__ hi,
            const int* __restrict__ cF, const T* __restrict__ vF, const T* __restrict__ dF,
            const int* __restrict__ cB, const T* __restrict__ vB, const T* __restrict__ dB,
            const T* __restrict__ r, T* y, T* s, const int* gate) {
  if (gated(gate)) return;
  constexpr int BPW = 32 / LPB;
  const int lane = threadIdx.x & 31, sub = lane / LPB, li = lane % LPB;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  const int ngroups = (nb + BPW - 1) / BPW;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < ngroups; w += nwarps) {
    const int b = w * BPW + sub;
    const int l0 = b < nb ? blvl[b] : 0, l1 = b < nb ? blvl[b + 1] : 0;
    const int nlev = l1 - l0;
    int maxlev = nlev;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxlev = max(maxlev, __shfl_xor_sync(0xffffffffu, maxlev, o));
    auto first_row = [&](int t, bool fwd) -> int {   // this lane's first row of step t, or -1
      if (t >= nlev) return -1;
      const int l = fwd ? l0 + t : l1 - 1 - t;
      const int p = lo[l] + li;
      return p < hi[l] ? p : -1;
    };
    SmallCols<K> cur, nxt;
    // forward: y = D^-1 (r - L y) (D-ILU) or r - L y (ILU(0), unit L)
    small_cols<K>(cur, first_row(0, true), cF);
    for (int t = 0; t < maxlev; ++t) {
      small_cols<K>(nxt, first_row(t + 1, true), cF);
      if (cur.p >= 0) {
        small_row<T, DILU, true, K>(cur, vF, dF, r, y, y);
        const int e = hi[l0 + t];
        for (int p = cur.p + LPB; p < e; p += LPB) {   // levels wider than LPB
          SmallCols<K> o;
          small_cols<K>(o, p, cF);
          small_row<T, DILU, true, K>(o, vF, dF, r, y, y);
        }
      }
      __syncwarp();
      cur = nxt;
    }
    // backward from the forward result y
    small_cols<K>(cur, first_row(0, false), cB);
    for (int t = 0; t < maxlev; ++t) {
      small_cols<K>(nxt, first_row(t + 1, false), cB);
      if (cur.p >= 0) {
        small_row<T, DILU, false, K>(cur, vB, dB, y, s, s);
        const int e = hi[l1 - 1 - t];
        for (int p = cur.p + LPB; p < e; p += LPB) {
          SmallCols<K> o;
          small_cols<K>(o, p, cB);
          small_row<T, DILU, false, K>(o, vB, dB, y, s, s);
        }
      }
      __syncwarp();
      cur = nxt;
    }
  }
}

// The same sweep with a block's data staged in shared memory.  A block's rows occupy one
// stretch [P0, P0 + S) of the iteration layout (its levels one after another, each starting
// on a multiple of 4), so the block's lanes copy the stretch's right-hand side, records and
// diagonal factors into the block's own area of shared memory with 16-byte asynchronous
// copies, all in flight at once.  Both sweeps run on shared memory, the solution overwriting
// the right-hand side in place (a level reads only rows of other levels, which are final),
// and each row of s is stored as it is finished.  The backward records are copied over the
// forward ones once the forward sweep is done: a smaller area per block lets more blocks be
// in flight on an SM, which is what the sweep waits on.  Same records, same expressions, same
// order as k_ilu_small.
constexpr int kStageWarps = 4;
constexpr int kStageBoxBytes = 12 * 1024;

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The lanes of a group copy `bytes` (a multiple of 16; both addresses 16-byte aligned).
__device__ __forceinline__ void group_stage(void* dst, const void* src, int bytes, int li, int lanes) {
  char* d = static_cast<char*>(dst);
  const char* g = static_cast<const char*>(src);
  for (int o = li * 16; o < bytes; o += lanes * 16) cp_async16(d + o, g + o);
}

// LPB lanes per block, 32 / LPB blocks per warp (as k_ilu_small), each block with its own
// area of box_bytes; blockDim.x / 32 warps per CTA.
template <class T, bool DILU, int K, int LPB>
__global__ void __launch_bounds__(kStageWarps * 32)
k_ilu_small_staged(int nb, const int2* __restrict__ box, const int* __restrict__ blvl, const int* __restrict__ lo,
                   const int* __restrict__ hi, const int* __restrict__ cF, const T* __restrict__ vF,
                   const T* __restrict__ dF, const int* __restrict__ cB, const T* __restrict__ vB,
                   const T* __restrict__ dB, const T* __restrict__ r, T* __restrict__ s, const int* gate, int span,
                   int levcap, int box_bytes) {
  if (gated(gate)) return;
  constexpr int BPW = 32 / LPB;
  extern __shared__ __align__(16) unsigned char stage_smem[];
  const int lane = threadIdx.x & 31, sub = lane / LPB, li = lane % LPB;
  const int wib = threadIdx.x >> 5, wpc = blockDim.x >> 5;
  // this block's area: T arrays first (each a multiple of 16 bytes, span being a multiple of
  // 4), then the int arrays; V and Cc hold the forward records, then the backward ones
  T* X = reinterpret_cast<T*>(stage_smem + ((size_t)wib * BPW + sub) * box_bytes);
  T* Fd = X + span;
  T* Bd = DILU ? Fd : Fd + span;   // D-ILU: both sweeps scale by the same D^-1
  T* V = Fd + span + (DILU ? 0 : span);   // after Fd (D-ILU) or after Bd (ILU(0))
  int* Cc = reinterpret_cast<int*>(V + (size_t)span * K);
  int* Lo = Cc + (size_t)span * K;
  int* Hi = Lo + levcap;
  const int nwarps = gridDim.x * wpc;
  const int ngroups = (nb + BPW - 1) / BPW;
  for (int w = blockIdx.x * wpc + wib; w < ngroups; w += nwarps) {
    const int b = w * BPW + sub;
    int P0 = 0, S = 0, l0 = 0, nlev = 0;
    if (b < nb) {
      const int2 bx = box[b];   // stretch: first position, length (host-checked: <= span)
      P0 = bx.x;
      S = bx.y;
      l0 = blvl[b];
      nlev = blvl[b + 1] - l0;  // host-checked: <= levcap
    }
    int maxlev = nlev;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxlev = max(maxlev, __shfl_xor_sync(0xffffffffu, maxlev, o));
    if (b < nb) {
      group_stage(X, r + P0, S * (int)sizeof(T), li, LPB);
      group_stage(V, vF + (int64_t)P0 * K, S * K * (int)sizeof(T), li, LPB);
      group_stage(Fd, dF + P0, S * (int)sizeof(T), li, LPB);
      group_stage(Cc, cF + (int64_t)P0 * K, S * K * 4, li, LPB);
      if (!DILU) group_stage(Bd, dB + P0, S * (int)sizeof(T), li, LPB);
      for (int t = li; t < nlev; t += LPB) {
        Lo[t] = lo[l0 + t] - P0;
        Hi[t] = hi[l0 + t] - P0;
      }
    }
    cp_async_commit();
    cp_async_wait<0>();   // this lane's copies
    __syncwarp();         // and everyone's
    // forward: y = D^-1 (r - L y) (D-ILU) or r - L y (ILU(0), unit L)
    for (int t = 0; t < maxlev; ++t) {
      if (t < nlev) {
        const int e = Hi[t];
        for (int q = Lo[t] + li; q < e; q += LPB) {
          T acc = X[q];
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const int c = Cc[q * K + k] - P0;   // -1 (no entry) falls outside [0, S)
            if ((unsigned)c < (unsigned)S) acc = acc - V[q * K + k] * X[c];
          }
          X[q] = DILU ? Fd[q] * acc : acc;
        }
      }
      __syncwarp();
    }
    // the forward records are no longer read (the barrier above): the backward ones replace them
    if (b < nb) {
      group_stage(V, vB + (int64_t)P0 * K, S * K * (int)sizeof(T), li, LPB);
      group_stage(Cc, cB + (int64_t)P0 * K, S * K * 4, li, LPB);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncwarp();
    // backward from the forward result
    for (int t = 0; t < maxlev; ++t) {
      if (t < nlev) {
        const int tl = nlev - 1 - t;
        const int e = Hi[tl];
        for (int q = Lo[tl] + li; q < e; q += LPB) {
          const T xp = X[q], d = Bd[q];
          T acc = DILU ? T(0) : xp;
#pragma unroll
          for (int k = 0; k < K; ++k) {
            const int c = Cc[q * K + k] - P0;
            if ((unsigned)c < (unsigned)S) {
              if (DILU) acc = acc + X[c] * V[q * K + k];
              else acc = acc - X[c] * V[q * K + k];
            }
          }
          const T o = DILU ? xp - d * acc : acc * d;
          X[q] = o;
          s[P0 + q] = o;
        }
      }
      __syncwarp();
    }
  }
}

// ------------------------------------------------------------------ host side
template <class T>
int ilu_setup_device(const IluPlan& P, const DevMat<double>& A, int ilu_method,
                     const int* d_pos, const int* d_rowAt, const int* d_lev, IluDev<T>& D) {
  cudaStream_t st = stream();
  D.nb = P.nb; D.np = P.np; D.n = P.n;
  D.dilu = ilu_method != 0;
  D.W = P.W;
  D.maxWp = std::max(4, P.maxWp);
  // every chunk carries the same number of coupled entries per row (the matrix-wide
  // maximum, rounded up to a supported count)
  std::vector<IluChunk> ch = P.chunks;
  int kmax = 0, maxw = 0;
  for (const auto& c : ch) { kmax = std::max(kmax, std::max(c.KL, c.KU)); maxw = std::max(maxw, c.w); }
  int kuni = kmax;
  for (int c : {1, 2, 3, 4, 6, 8})
    if (kmax <= c) { kuni = c; break; }
  for (auto& c : ch) { c.KL = kuni; c.KU = kuni; }
  D.K = kuni;
  // shared memory budget: barriers + ring + stages
  int dev_smem = 0;
  PB_CUDA(cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx().device));
  const int budget = std::min(dev_smem, 220 * 1024);
  int64_t ring_bytes = ((int64_t)D.W * D.maxWp + 1) * sizeof(T);
  D.ring = ring_bytes <= 64 * 1024;
  int64_t ring_alloc = D.ring ? ((ring_bytes + 127) & ~int64_t(127)) : 0;
  // consumer threads and rows per thread of the grouped sweep
  // (one row per thread: a second row slot costs every level its predicated instructions,
  // although few levels are wider than 256 rows)
  if (maxw <= 128) { D.nc = 128; D.rows = 1; }
  else if (maxw <= 256) { D.nc = 256; D.rows = 1; }
  else if (maxw <= 384) { D.nc = 384; D.rows = 1; }
  else { D.nc = 512; D.rows = 1; }   // chunks have at most kIluChunk = 512 rows
  D.grp = D.ring && D.rows > 0 && kuni <= 8;
  if (D.grp) {
    // Groups of consecutive chunks of one block, each at most kGrpMax chunks and about a
    // quarter of the stage budget (a chunk larger than that forms a group of its own).
    const int64_t sz = sizeof(T);
    const int64_t strF = rec_stride((int)sz, D.dilu, kuni), strB = rec_stride((int)sz, true, kuni);
    auto grp_bytes = [&](int64_t span) {   // backward record (the larger) + vector slice
      return kGrpHdr + ((span * strB + 15) & ~int64_t(15)) + span * sz;
    };
        const int64_t target = (budget - 128 - ring_alloc) / 4;
    std::vector<int4> gi;
    std::vector<int> blk_grp(P.nb + 1, 0);
    int64_t max_stage = 0;
    for (int b = 0; b < P.nb; ++b) {
      blk_grp[b] = (int)gi.size();
      int c = P.blk_chunk[b];
      while (c < P.blk_chunk[b + 1]) {
        const int sstart = ch[c].start;
        int e = c + 1;
        auto span_to = [&](int ce) { return (int64_t)align4(ch[ce - 1].start + ch[ce - 1].w) - sstart; };
        while (e < P.blk_chunk[b + 1] && e - c < kGrpMax && grp_bytes(span_to(e + 1)) <= target) ++e;
        const int64_t span = span_to(e);
        gi.push_back(make_int4(c, e, sstart, (int)span));
        max_stage = std::max(max_stage, grp_bytes(span));
        c = e;
      }
    }
    blk_grp[P.nb] = (int)gi.size();
    const int ng = (int)gi.size();
    std::vector<int64_t> goff(2 * (size_t)std::max(ng, 1), 0);
    std::vector<GrpDesc> tf(ng), tb(ng);
    int64_t oF = 0, oB = 0;
    for (int g = 0; g < ng; ++g) {
      const int64_t span = gi[g].w;
      const int64_t cbF = kGrpHdr + ((span * strF + 15) & ~int64_t(15));
      const int64_t cbB = kGrpHdr + ((span * strB + 15) & ~int64_t(15));
      goff[2 * g] = oF;
      goff[2 * g + 1] = oB;
      PB_CHECK(oF / 16 < INT32_MAX && oB / 16 < INT32_MAX, PARCEL_B_E_UNSUPPORTED,
               "packed preconditioner larger than 32 GiB");
      tf[g] = GrpDesc{(int)(oF / 16), (int)cbF, gi[g].z, (int)(span * sz)};
      tb[g] = GrpDesc{(int)(oB / 16), (int)cbB, gi[g].z, (int)(span * sz)};
      oF += align16(cbF);
      oB += align16(cbB);
    }
    D.packF_bytes = std::max<int64_t>(oF, 16);
    D.packB_bytes = std::max<int64_t>(oB, 16);
    D.stage_bytes = (int)((max_stage + 127) & ~int64_t(127));
    const int64_t room = budget - 128 - ring_alloc;
    D.nstages = (int)std::min<int64_t>(kGrpMaxStages, room / D.stage_bytes);
    PB_CHECK(D.nstages >= 2, PARCEL_B_E_UNSUPPORTED,
             "block-Jacobi level too wide for shared memory (stage %d bytes)", D.stage_bytes);
    D.smem_bytes = (int)(128 + ring_alloc + (int64_t)D.nstages * D.stage_bytes);
    D.ngroups = ng;
    D.tabF.alloc(sizeof(GrpDesc) * std::max(ng, 1));
    D.tabB.alloc(sizeof(GrpDesc) * std::max(ng, 1));
    h2d(D.tabF.p, tf.data(), sizeof(GrpDesc) * ng);
    h2d(D.tabB.p, tb.data(), sizeof(GrpDesc) * ng);
    D.blk_grp.alloc(sizeof(int) * (P.nb + 1));
    h2d(D.blk_grp.p, blk_grp.data(), sizeof(int) * (P.nb + 1));
    D.ginfo.alloc(sizeof(int4) * std::max(ng, 1));
    h2d(D.ginfo.p, gi.data(), sizeof(int4) * ng);
    D.goff.alloc(sizeof(int64_t) * goff.size());
    h2d(D.goff.p, goff.data(), sizeof(int64_t) * goff.size());
  } else {
    // per-chunk records for the general sweep
    int64_t oF = 0, oB = 0;
    int64_t max_stage = 0;
    for (auto& c : ch) {
      c.offF = oF; c.offB = oB;
      int64_t bf = chunk_bytes<T>(c.wpad, c.KL), bb = chunk_bytes<T>(c.wpad, c.KU);
      oF += align16(bf); oB += align16(bb);
      max_stage = std::max(max_stage, std::max(bf, bb) + (int64_t)c.wpad * (int64_t)sizeof(T));
    }
    D.packF_bytes = std::max<int64_t>(oF, 16);
    D.packB_bytes = std::max<int64_t>(oB, 16);
    D.stage_bytes = (int)((max_stage + 127) & ~int64_t(127));
    int nst = 16;
    auto need = [&](int k) { return (int64_t)((16 * k + 16 + 127) & ~127) + ring_alloc + (int64_t)k * D.stage_bytes; };
    while (nst > 2 && need(nst) > budget) --nst;
    PB_CHECK(need(nst) <= budget, PARCEL_B_E_UNSUPPORTED,
             "block-Jacobi level too wide for shared memory (stage %d bytes)", D.stage_bytes);
    D.nstages = nst;
    D.smem_bytes = (int)need(nst);
    std::vector<ProdDesc> tf(ch.size()), tb(ch.size());
    for (size_t i = 0; i < ch.size(); ++i) {
      const IluChunk& c = ch[i];
      PB_CHECK(c.offF / 16 < INT32_MAX && c.offB / 16 < INT32_MAX, PARCEL_B_E_UNSUPPORTED,
               "packed preconditioner larger than 32 GiB");
      tf[i] = ProdDesc{(int)(c.offF / 16), c.start, (int)chunk_bytes<T>(c.wpad, c.KL),
                       (int)(c.wpad * sizeof(T))};
      tb[i] = ProdDesc{(int)(c.offB / 16), c.start, (int)chunk_bytes<T>(c.wpad, c.KU),
                       (int)(c.wpad * sizeof(T))};
    }
    D.tabF.alloc(sizeof(ProdDesc) * std::max<size_t>(ch.size(), 1));
    D.tabB.alloc(sizeof(ProdDesc) * std::max<size_t>(ch.size(), 1));
    h2d(D.tabF.p, tf.data(), sizeof(ProdDesc) * ch.size());
    h2d(D.tabB.p, tb.data(), sizeof(ProdDesc) * ch.size());
  }
  D.chunks.alloc(sizeof(IluChunk) * std::max<size_t>(ch.size(), 1));
  h2d(D.chunks.p, ch.data(), sizeof(IluChunk) * ch.size());
  D.blk_chunk.alloc(sizeof(int) * (P.nb + 1));
  h2d(D.blk_chunk.p, P.blk_chunk.data(), sizeof(int) * (P.nb + 1));
  DBuf blo(sizeof(int) * P.nb), bhi(sizeof(int) * P.nb);
  h2d(blo.p, P.blk_lo.data(), sizeof(int) * P.nb);
  h2d(bhi.p, P.blk_hi.data(), sizeof(int) * P.nb);
  DBuf blvl(sizeof(int) * (P.nb + 1)), lst(sizeof(int) * std::max<size_t>(P.lvl_start.size(), 1));
  h2d(blvl.p, P.blk_lvl.data(), sizeof(int) * (P.nb + 1));
  h2d(lst.p, P.lvl_start.data(), sizeof(int) * P.lvl_start.size());

  trace_mark("ilu: tables to device");
  // factorisation in natural CSR order
  const int64_t nnz = A.nnz;
  DBuf lu, Dd, Di;
  const double* vL = A.val;
  const double* vU = A.val;
  if (!D.dilu) {
    lu.alloc(sizeof(double) * nnz);
    d2d(lu.p, A.val, sizeof(double) * nnz);
    k_ilu0_factor<<<P.nb, ilu_factor_threads(P.maxWp), 0, st>>>(dp<IluChunk>(D.chunks), dp<int>(D.blk_chunk), dp<int>(blo),
                                        dp<int>(bhi), d_rowAt, A.rowptr, A.col, A.rbase, A.cbase,
                                        dp<double>(lu));
    PB_CUDA(cudaGetLastError());
    vL = dp<double>(lu);
    vU = dp<double>(lu);
  } else {
    Dd.alloc(sizeof(double) * P.n);
    Di.alloc(sizeof(double) * P.n);
    k_dilu_diag<<<P.nb, ilu_factor_threads(P.maxWp), 0, st>>>(dp<IluChunk>(D.chunks), dp<int>(D.blk_chunk), dp<int>(blo),
                                      dp<int>(bhi), d_rowAt, A.rowptr, A.col, A.val, A.rbase, A.cbase,
                                      ilu_method == 2 ? 1 : 0, dp<double>(Dd), dp<double>(Di));
    PB_CUDA(cudaGetLastError());
  }
  trace_mark("ilu: factor");
  D.packF.alloc(D.packF_bytes);
  D.packB.alloc(D.packB_bytes);
  if (D.grp) {
    k_ilu_pack_grp<T><<<std::max(1, std::min(D.ngroups, 65535)), 256, 0, st>>>(
        dp<int4>(D.ginfo), dp<int64_t>(D.goff), D.ngroups, dp<IluChunk>(D.chunks), dp<int>(blo), dp<int>(bhi),
        dp<int>(blvl), dp<int>(lst), d_rowAt, d_pos, d_lev, A.rowptr, A.col, A.rbase, A.cbase, vL, vU,
        D.dilu ? dp<double>(Di) : nullptr, D.dilu ? 1 : 0, D.W, D.maxWp, D.K, dp<unsigned char>(D.packF),
        dp<unsigned char>(D.packB));
  } else {
    k_ilu_pack<T><<<std::min<int>((int)ch.size(), 65535) > 0 ? std::min<int>((int)ch.size(), 65535) : 1,
                    128, 0, st>>>(
        dp<IluChunk>(D.chunks), (int)ch.size(), dp<int>(blo), dp<int>(bhi), dp<int>(blvl),
        dp<int>(lst), d_rowAt, d_pos, d_lev, A.rowptr, A.col, A.rbase, A.cbase, vL, vU,
        D.dilu ? dp<double>(Di) : nullptr, D.dilu ? 1 : 0, D.ring ? 1 : 0, D.W, D.maxWp,
        dp<unsigned char>(D.packF), dp<unsigned char>(D.packB));
  }
  PB_CUDA(cudaGetLastError());
  // many small blocks: the warp-per-block records as well (the packed ones serve the
  // accumulating apply)
  int max_rows = 0;
  for (int b = 0; b < P.nb; ++b) max_rows = std::max(max_rows, P.blk_hi[b] - P.blk_lo[b]);
  D.small = max_rows <= kSmallMaxRows && P.nb >= 8 * num_sms() && D.K <= 8;
  if (D.small) {
    // lanes per block: the widest level, rounded up to 8, 16 or 32 (wider levels take
    // several rows per lane)
    D.s_lpb = maxw <= 8 ? 8 : (maxw <= 16 ? 16 : 32);
    const size_t rk = (size_t)P.np * D.K;
    D.s_cF.alloc(sizeof(int) * rk); D.s_vF.alloc(sizeof(T) * rk); D.s_dF.alloc(sizeof(T) * P.np);
    D.s_cB.alloc(sizeof(int) * rk); D.s_vB.alloc(sizeof(T) * rk); D.s_dB.alloc(sizeof(T) * P.np);
    const int totlev = (int)P.lvl_start.size();
    D.s_blvl.alloc(sizeof(int) * (P.nb + 1));
    D.s_lo.alloc(sizeof(int) * std::max(totlev, 1));
    D.s_hi.alloc(sizeof(int) * std::max(totlev, 1));
    h2d(D.s_blvl.p, P.blk_lvl.data(), sizeof(int) * (P.nb + 1));
    h2d(D.s_lo.p, P.lvl_start.data(), sizeof(int) * totlev);
    h2d(D.s_hi.p, P.lvl_end.data(), sizeof(int) * totlev);
    const int g = (int)std::min<int64_t>(((int64_t)P.n + 255) / 256, 8LL * num_sms());
    k_ilu_small_pack<T><<<std::max(g, 1), 256, 0, st>>>(
        P.n, P.nb, dp<int>(blo), dp<int>(bhi), d_pos, A.rowptr, A.col, A.rbase, A.cbase, vL, vU,
        D.dilu ? dp<double>(Di) : nullptr, D.dilu ? 1 : 0, D.K, dp<int>(D.s_cF), dp<T>(D.s_vF), dp<T>(D.s_dF),
        dp<int>(D.s_cB), dp<T>(D.s_vB), dp<T>(D.s_dB));
    PB_CUDA(cudaGetLastError());
    // the staged variant: each block's stretch of the iteration layout, from its first level's
    // start to its last level's end rounded up to 4 (the next block, or the end of the
    // padded layout, starts there)
    std::vector<int2> bxs(P.nb);
    int span = 0;
    for (int b = 0; b < P.nb; ++b) {
      const int p0 = P.lvl_start[P.blk_lvl[b]], p1 = align4(P.lvl_end[P.blk_lvl[b + 1] - 1]);
      bxs[b] = make_int2(p0, p1 - p0);
      span = std::max(span, p1 - p0);
    }
    const int levcap = align4(std::max(P.max_levels, 1));
    const int64_t tb = (int64_t)span * (2 + D.K + (D.dilu ? 0 : 1)) * (int64_t)sizeof(T) +
                       (int64_t)span * D.K * 4 + 2LL * levcap * 4;
    D.s_box_bytes = 0;
    if (tb <= kStageBoxBytes) {   // a warp's blocks (at most 4) within the default 48 KB of a CTA
      D.s_span = span;
      D.s_levcap = levcap;
      D.s_box_bytes = (int)tb;
      D.s_box.alloc(sizeof(int2) * P.nb);
      h2d(D.s_box.p, bxs.data(), sizeof(int2) * P.nb);
    }
  }
  D.ytmp.alloc(sizeof(T) * (P.np + 4));
  PB_CUDA(cudaMemsetAsync(D.ytmp.p, 0, sizeof(T) * (P.np + 4), st));
  D.err.alloc(sizeof(int));
  PB_CUDA(cudaMemsetAsync(D.err.p, 0, sizeof(int), st));
  // temporaries (lu, Dd, Di, blo, ...) are freed when this function returns: make sure
  // the kernels that read them have finished.
  sync();
  return 0;
}

template <class T, bool DILU, bool RING>
static void launch_ilu(const IluDev<T>& D, const IluSolveArgs<T>& a, cudaStream_t st) {
  auto kern = k_ilu_solve<T, DILU, RING>;
  static int configured = 0;
  if (configured < D.smem_bytes) {
    PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    configured = 227 * 1024;
  }
  kern<<<D.nb, kIluThreads, D.smem_bytes, st>>>(a);
}

template <class T, bool DILU, int KM, int R, int NC>
static void launch_grp(const IluDev<T>& D, const GrpArgs<T>& a, cudaStream_t st) {
  auto kern = k_ilu_sweep_grp<T, DILU, KM, R, NC>;
  static bool configured = false;
  if (!configured) {
    PB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
    configured = true;
  }
  kern<<<D.nb, NC + 32, D.smem_bytes, st>>>(a);
}

template <class T, bool DILU, int K, int LPB>
static void launch_small_lpb(const IluDev<T>& D, const T* r, T* s, const int* gate, cudaStream_t st) {
  const int64_t warps = ((int64_t)D.nb + 32 / LPB - 1) / (32 / LPB);
  const int grid = (int)std::min<int64_t>((warps * 32 + kSmallThreads - 1) / kSmallThreads, 16LL * num_sms());
  k_ilu_small<T, DILU, K, LPB><<<grid, kSmallThreads, 0, st>>>(
      D.nb, dp<int>(D.s_blvl), dp<int>(D.s_lo), dp<int>(D.s_hi), dp<int>(D.s_cF), dp<T>(D.s_vF), dp<T>(D.s_dF),
      dp<int>(D.s_cB), dp<T>(D.s_vB), dp<T>(D.s_dB), r, dp<T>(D.ytmp), s, gate);
}

template <class T, bool DILU, int K, int LPB>
static void launch_staged(const IluDev<T>& D, const T* r, T* s, const int* gate, cudaStream_t st) {
  constexpr int BPW = 32 / LPB;
  const int warp_bytes = BPW * D.s_box_bytes;
  const int wpc = std::max(1, std::min(kStageWarps, 48 * 1024 / warp_bytes));
  const int64_t groups = ((int64_t)D.nb + BPW - 1) / BPW;
  const int grid = (int)std::min<int64_t>((groups + wpc - 1) / wpc, 32LL * num_sms());
  k_ilu_small_staged<T, DILU, K, LPB><<<grid, wpc * 32, (size_t)wpc * warp_bytes, st>>>(
      D.nb, dp<int2>(D.s_box), dp<int>(D.s_blvl), dp<int>(D.s_lo), dp<int>(D.s_hi), dp<int>(D.s_cF),
      dp<T>(D.s_vF), dp<T>(D.s_dF), dp<int>(D.s_cB), dp<T>(D.s_vB), dp<T>(D.s_dB), r, s, gate, D.s_span,
      D.s_levcap, D.s_box_bytes);
}

template <class T, bool DILU, int K>
static void launch_small(const IluDev<T>& D, const T* r, T* s, const int* gate, cudaStream_t st) {
  if (D.s_box_bytes > 0 && (reinterpret_cast<uintptr_t>(r) & 15) == 0) {
    if (D.s_lpb == 8) launch_staged<T, DILU, K, 8>(D, r, s, gate, st);
    else if (D.s_lpb == 16) launch_staged<T, DILU, K, 16>(D, r, s, gate, st);
    else launch_staged<T, DILU, K, 32>(D, r, s, gate, st);
    return;
  }
  if (D.s_lpb == 8) launch_small_lpb<T, DILU, K, 8>(D, r, s, gate, st);
  else if (D.s_lpb == 16) launch_small_lpb<T, DILU, K, 16>(D, r, s, gate, st);
  else launch_small_lpb<T, DILU, K, 32>(D, r, s, gate, st);
}

template <class T>
void ilu_apply(const IluDev<T>& D, const T* r, T* s, T* accum, const int* gate, cudaStream_t st) {
  if (D.small && !accum) {
#define SMALL(K_)                                                                                  \
  case K_:                                                                                         \
    if (D.dilu) launch_small<T, true, K_>(D, r, s, gate, st); else launch_small<T, false, K_>(D, r, s, gate, st); \
    break;
    switch (D.K) {
      SMALL(1) SMALL(2) SMALL(3) SMALL(4) SMALL(6) SMALL(8)
      default: PB_CHECK(false, PARCEL_B_E_ARG, "unsupported coupling count %d", D.K);
    }
#undef SMALL
    PB_CUDA(cudaGetLastError());
    return;
  }
  if (D.grp && !accum) {
    GrpArgs<T> g;
    g.tabF = dp<GrpDesc>(D.tabF);
    g.tabB = dp<GrpDesc>(D.tabB);
    g.blk_grp = dp<int>(D.blk_grp);
    g.packF = dp<unsigned char>(D.packF);
    g.packB = dp<unsigned char>(D.packB);
    g.r = r;
    g.y = dp<T>(D.ytmp);
    g.s = s;
    g.stage_bytes = D.stage_bytes;
    g.nstages = D.nstages;
    g.ring_elems = D.W * D.maxWp + 1;
    g.gate = gate;
    g.err = dp<int>(D.err);
#define GRP_R(KM_, R_, NC_)                                                                        \
  if (D.dilu) launch_grp<T, true, KM_, R_, NC_>(D, g, st); else launch_grp<T, false, KM_, R_, NC_>(D, g, st);
#define GRP(KM_)                                                                                   \
  case KM_:                                                                                        \
    if (D.nc == 128) { GRP_R(KM_, 1, 128) }                                                        \
    else if (D.nc == 256) { GRP_R(KM_, 1, 256) }                                                   \
    else if (D.nc == 384) { GRP_R(KM_, 1, 384) } else { GRP_R(KM_, 1, 512) }                       \
    break;
    switch (D.K) {
      GRP(1) GRP(2) GRP(3) GRP(4) GRP(6) GRP(8)
      default: PB_CHECK(false, PARCEL_B_E_ARG, "unsupported coupling count %d", D.K);
    }
#undef GRP
#undef GRP_R
    PB_CUDA(cudaGetLastError());
    return;
  }
  PB_CHECK(!D.grp, PARCEL_B_E_UNSUPPORTED, "accumulating block-Jacobi apply needs the general sweep");
  IluSolveArgs<T> a;
  a.tabF = dp<ProdDesc>(D.tabF);
  a.tabB = dp<ProdDesc>(D.tabB);
  a.blk_chunk = dp<int>(D.blk_chunk);
  a.packF = dp<unsigned char>(D.packF);
  a.packB = dp<unsigned char>(D.packB);
  a.r = r;
  a.y = dp<T>(D.ytmp);
  a.s = s;
  a.accum = accum;
  a.W = D.W;
  a.maxWp = D.maxWp;
  a.stage_bytes = D.stage_bytes;
  a.nstages = D.nstages;
  a.ring_elems = D.ring ? D.W * D.maxWp + 1 : 0;
  a.gate = gate;
  a.err = dp<int>(D.err);
  if (D.dilu) {
    if (D.ring) launch_ilu<T, true, true>(D, a, st); else launch_ilu<T, true, false>(D, a, st);
  } else {
    if (D.ring) launch_ilu<T, false, true>(D, a, st); else launch_ilu<T, false, false>(D, a, st);
  }
  PB_CUDA(cudaGetLastError());
}

template int ilu_setup_device<double>(const IluPlan&, const DevMat<double>&, int, const int*,
                                      const int*, const int*, IluDev<double>&);
template int ilu_setup_device<float>(const IluPlan&, const DevMat<double>&, int, const int*,
                                     const int*, const int*, IluDev<float>&);
template void ilu_apply<double>(const IluDev<double>&, const double*, double*, double*,
                                const int*, cudaStream_t);
template void ilu_apply<float>(const IluDev<float>&, const float*, float*, float*, const int*,
                               cudaStream_t);

}  // namespace pb
