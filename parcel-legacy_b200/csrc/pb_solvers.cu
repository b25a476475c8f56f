// pb_solvers.cu -- PCG, BiCGStab and GMRES(m) drivers on B200.
//
// Reference loops (restated): KSP_pCG (src/pcg.f90:224-892), KSP_pBiCG
// (src/pbicg.f90:280-698), KSP_pGMRES (src/pgmres.f90:62-525) with GivensRotations and
// update_xVec (src/pcagmres.f90:190-242, 1136-1236).
//
// The reference's GPU path synchronises the device and moves a scalar across PCIe for
// every dot product and axpy (src/CUDA/src/cu_common.cu:412-446,
// src/parcel_vec.f90:466-470).  Here every scalar stays on the device (KState) and the
// solver logic runs in the epilogue of the reduction that produces it, so an iteration
// is a fixed sequence of kernel launches.  Each kernel first reads a device flag and
// returns at once after the reference loop has exited, which lets a whole restart cycle
// (GMRES) or a chunk of iterations (CG, BiCGStab) be captured once into a CUDA graph and
// replayed; the host looks at the flag once per replay.
#include <algorithm>
#include <chrono>
#include <type_traits>

#include "pb_mgs.cuh"

#include <atomic>
#include <functional>
#include "pb_solvers.cuh"

namespace pb {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------------ options
namespace {
thread_local const std::vector<int>* t_block_starts = nullptr;
}  // namespace

ScopedBlockStarts::ScopedBlockStarts(const std::vector<int>* starts) { t_block_starts = starts; }
ScopedBlockStarts::~ScopedBlockStarts() { t_block_starts = nullptr; }

BlockSplit block_split(const Options& o, int n) {
  BlockSplit bs;
  if (o.block_starts.empty()) {
    bs.nb = std::max(1, std::min(o.nblocks, n));
    return bs;
  }
  const auto& s = o.block_starts;
  PB_CHECK(s.size() >= 2 && s.front() == 0 && s.back() == n, PARCEL_B_E_ARG,
           "explicit blocks must start at row 0 and end at n = %d", n);
  for (size_t b = 0; b + 1 < s.size(); ++b)
    PB_CHECK(s[b + 1] > s[b], PARCEL_B_E_ARG, "explicit block %d is empty", (int)b);
  bs.nb = (int)s.size() - 1;
  bs.starts = s;
  return bs;
}

Options resolve_options(const parcel_b_input* p) {
  Options o;
  if (t_block_starts) o.block_starts = *t_block_starts;
  if (!p) return o;
  if (p->solver > 0) o.solver = p->solver;
  if (p->ipreflag >= 0) o.precon = p->ipreflag;
  if (o.precon == PARCEL_B_PRECON_ADDITIVESCHWARZ) o.precon = PARCEL_B_PRECON_BLOCKJACOBI;
  if (p->ILU_method >= 0) o.ilu_method = p->ILU_method;
  if (p->precon_thblock > 0) o.nblocks = p->precon_thblock;
  if (p->GMRES_m > 0) o.m = p->GMRES_m;
  if (p->GMRES_GSflag > 0) o.gs = p->GMRES_GSflag;
  if (p->itrmax > 0) o.itrmax = p->itrmax;
  if (p->rtolmax != -1.0) o.rtol = p->rtolmax;
  if (p->abstolmax > 0.0) o.abstol = p->abstolmax;
  if (p->CAGMRES_sstep > 0) o.sstep = p->CAGMRES_sstep;
  if (p->CAGMRES_tstep > 0) o.tstep = p->CAGMRES_tstep;
  if (p->CAGMRES_basis >= 0) o.basis = p->CAGMRES_basis;
  if (p->CAGMRES_QRflag > 0) o.qrflag = p->CAGMRES_QRflag;
  if (p->inner_precision > 0) o.inner = p->inner_precision;
  if (p->residual_dd > 0) o.residual_dd = 1;
  if (p->inner_rtol > 0.0) o.inner_rtol = p->inner_rtol;
  if (p->max_refine > 0) o.max_refine = p->max_refine;
  if (p->independ_nvec > 0) o.independ_nvec = p->independ_nvec;
  if (p->reserved[0] == 1) o.use_graphs = false;
  if (p->reserved[1] == 1) o.fused_mgs = false;
  return o;
}

// ------------------------------------------------------------------ workspace
void Workspace::init() {
  part.alloc(sizeof(double) * (size_t)red_blocks() * kMaxRed);
  ticket.alloc(sizeof(unsigned) * 4);
  state.alloc(sizeof(KState));
  PB_CUDA(cudaMemsetAsync(ticket.p, 0, sizeof(unsigned) * 4, stream()));
  PB_CUDA(cudaMemsetAsync(state.p, 0, sizeof(KState), stream()));
}

Red Workspace::red(int epi) const {
  Red r;
  r.part = dp<double>(part);
  r.ticket = dp<unsigned>(ticket);
  r.epi = epi;
  r.ea.st = st();
  return r;
}

// ------------------------------------------------------------------ preconditioner
template <class T>
__global__ void k_pj_dinv(int n, const int* __restrict__ rp, const int* __restrict__ ci,
                          const double* __restrict__ va, int rbase, int cbase, T* __restrict__ dinv) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double d = 0.0;
    for (int j = rp[i] - rbase; j < rp[i + 1] - rbase; ++j)
      if (ci[j] - cbase == i) d = va[j];
    if (d == 0.0) d = 1.0e-300;   // get_DInv_crs (matrix.f90:3104-3144)
    dinv[i] = (T)(1.0 / d);
  }
}

template <class T>
void Precon<T>::apply(int64_t np, const T* r, T* s, const int* gate, cudaStream_t st) const {
  switch (kind) {
    case PARCEL_B_PRECON_NONE:
      lincomb<T>(np, s, r, cimm(1.0), nullptr, cimm(0.0), nullptr, cimm(0.0), gate, st);
      break;
    case PARCEL_B_PRECON_POINTJACOBI:
      scale<T>(np, s, dp<T>(dinv), r, gate, st);
      break;
    case PARCEL_B_PRECON_BLOCKJACOBI:
      // the sweeps may read r over the whole padded iteration layout
      PB_CHECK(np >= ilu.np, PARCEL_B_E_ARG, "vector of %lld entries, the iteration layout has %d", (long long)np,
               ilu.np);
      ilu_apply<T>(ilu, r, s, nullptr, gate, st);
      break;
  }
}

// ------------------------------------------------------------------ system setup
template <class T>
void build_system(const Options& o, const parcel_b_crs& A, bool dev, System<T>& S) {
  cudaStream_t st = stream();
  trace_mark(nullptr);
  S.n = A.n;
  S.nnz = A.nnz;
  const int* rp = A.rowptr;
  const int* ci = A.col;
  const double* va = A.val;
  if (!dev) {
    S.up_rowptr.alloc(sizeof(int) * (A.n + 1));
    S.up_col.alloc(sizeof(int) * std::max<int64_t>(A.nnz, 1));
    S.up_val.alloc(sizeof(double) * std::max<int64_t>(A.nnz, 1));
    h2d(S.up_rowptr.p, A.rowptr, sizeof(int) * (A.n + 1));
    h2d(S.up_col.p, A.col, sizeof(int) * A.nnz);
    h2d(S.up_val.p, A.val, sizeof(double) * A.nnz);
    rp = dp<int>(S.up_rowptr);
    ci = dp<int>(S.up_col);
    va = dp<double>(S.up_val);
  }
  S.Anat.n = A.n;
  S.Anat.nnz = A.nnz;
  S.Anat.rowptr = rp;
  S.Anat.col = ci;
  S.Anat.val = va;
  S.Anat.rbase = 1;
  S.Anat.cbase = A.istart;
  S.M.kind = o.precon;

  if (o.precon == PARCEL_B_PRECON_BLOCKJACOBI) {
    // The wavefront analysis runs on the host.  A device-resident structure comes back
    // through page-locked staging: the row pointers first, then the column indices in
    // block-aligned pieces, each with an event, so that the plan of the first blocks
    // overlaps the copy of the others.  The plan writes the permutation and the levels
    // into the same staging area, from where they go back to the device.
    const BlockSplit bs = block_split(o, A.n);
    const int nb = bs.nb;
    const size_t n1 = (size_t)A.n + 1, nz = (size_t)A.nnz;
    int* pin = static_cast<int*>(pinned_staging(sizeof(int) * ((dev ? n1 + nz : 0) + 2 * (size_t)A.n)));
    int* hpos = pin + (dev ? n1 + nz : 0);
    int* hlev = hpos + A.n;
    const int* hrpp = A.rowptr;
    const int* hcip = A.col;
    constexpr int kPieces = 4;
    cudaEvent_t ev[kPieces] = {};
    std::vector<int> piece_of(nb, 0);
    std::atomic<int> copy_failed{0};
    std::atomic<int> piece_done[kPieces];
    for (auto& d : piece_done) d.store(0);
    std::function<void(int)> ready;
    auto destroy_events = [&] {
      for (auto& e : ev)
        if (e) { cudaEventDestroy(e); e = nullptr; }
    };
    if (dev) {
      d2h(pin, A.rowptr, sizeof(int) * n1);   // synchronous: the row pointers size the pieces
      hrpp = pin;
      hcip = pin + n1;
      for (int k = 0; k < kPieces; ++k) {
        const int b0 = (int)((int64_t)nb * k / kPieces), b1 = (int)((int64_t)nb * (k + 1) / kPieces);
        for (int b = b0; b < b1; ++b) piece_of[b] = k;
        cudaError_t e = cudaEventCreateWithFlags(&ev[k], cudaEventDisableTiming);
        if (e == cudaSuccess && b1 > b0) {
          int lo0, hi0, lo1, hi1;
          bs.rows(b0, A.n, &lo0, &hi0);
          bs.rows(b1 - 1, A.n, &lo1, &hi1);
          const size_t j0 = (size_t)(hrpp[lo0] - 1), j1 = (size_t)(hrpp[hi1] - 1);   // 1-based
          if (j1 > j0) e = cudaMemcpyAsync(pin + n1 + j0, A.col + j0, sizeof(int) * (j1 - j0), cudaMemcpyDeviceToHost, st);
        }
        if (e == cudaSuccess) e = cudaEventRecord(ev[k], st);
        if (e != cudaSuccess) {
          destroy_events();
          PB_CUDA(e);
        }
      }
      // called from the plan's parallel loop: no exception may leave it.  A piece is waited
      // for once (with tens of thousands of blocks a wait per block costs more than the plan).
      ready = [&](int b) {
        const int k = piece_of[b];
        if (piece_done[k].load(std::memory_order_acquire)) return;
        if (cudaEventSynchronize(ev[k]) != cudaSuccess) copy_failed = 1;
        piece_done[k].store(1, std::memory_order_release);
      };
    }
    HostCSR H;
    H.n = A.n; H.nnz = A.nnz; H.istart = A.istart; H.rowptr = hrpp; H.col = hcip;
    IluPlan P;
    trace_mark("setup: row pointers to host");
    try {
      ilu_build_plan(H, bs, P, hpos, hlev, ready);
    } catch (...) {
      destroy_events();
      throw;
    }
    destroy_events();
    PB_CHECK(!copy_failed, PARCEL_B_E_CUDA, "copy of the sparsity structure to the host failed");
    trace_mark("setup: wavefront plan (host)");
    S.np = P.np;
    S.permuted = true;
    S.ilu_levels_max = P.max_levels;
    S.ilu_nblocks = P.nb;
    S.pos.alloc(sizeof(int) * A.n);
    S.lev.alloc(sizeof(int) * A.n);
    S.rowAt.alloc(sizeof(int) * P.np);
    h2d(S.pos.p, hpos, sizeof(int) * A.n);
    h2d(S.lev.p, hlev, sizeof(int) * A.n);
    PB_CUDA(cudaMemsetAsync(S.rowAt.p, 0xFF, sizeof(int) * P.np, st));   // padding: -1
    scatter_positions(A.n, dp<int>(S.pos), dp<int>(S.rowAt), st);
    trace_mark("setup: layout maps to device");
    S.A = DevMat<T>{};
    S.A.nnz = A.nnz;
    build_sell<T>(S.Anat, P.np, dp<int>(S.rowAt), dp<int>(S.pos), S.Asell, S.A);
    trace_mark("setup: sliced ELLPACK");
    ilu_setup_device<T>(P, S.Anat, o.ilu_method, dp<int>(S.pos), dp<int>(S.rowAt),
                        dp<int>(S.lev), S.M.ilu);
    trace_mark("setup: ILU factor + pack");
  } else {
    S.np = A.n;
    S.permuted = false;
    if constexpr (std::is_same<T, double>::value) {
      S.A = S.Anat;
    } else {
      S.Aval_T.alloc(sizeof(T) * std::max<int64_t>(A.nnz, 1));
      convert<T, double>(A.nnz, dp<T>(S.Aval_T), va, st);
      S.A.n = A.n; S.A.nnz = A.nnz; S.A.rowptr = rp; S.A.col = ci;
      S.A.val = dp<T>(S.Aval_T); S.A.rbase = 1; S.A.cbase = A.istart;
    }
    {
      DevMat<T> M = S.A;
      build_sell<T>(S.Anat, A.n, nullptr, nullptr, S.Asell, M);
      S.spmv_diagonals = build_dia<T>(S.Anat, S.Asell, M);
      S.A = M;
    }
    if (o.precon == PARCEL_B_PRECON_POINTJACOBI) {
      S.M.dinv.alloc(sizeof(T) * A.n);
      k_pj_dinv<T><<<8 * num_sms(), 256, 0, st>>>(A.n, rp, ci, va, 1, A.istart, dp<T>(S.M.dinv));
      PB_CUDA(cudaGetLastError());
    }
  }
}

// ------------------------------------------------------------------ graph replay
struct GraphRunner {
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
  GraphRunner() = default;
  GraphRunner(const GraphRunner&) = delete;
  ~GraphRunner() { if (exec) cudaGraphExecDestroy(exec); }
  template <class F>
  void launch(F&& f, bool use_graph, cudaStream_t st) {
    if (!use_graph) { f(); return; }
    if (!exec) {
      trace_mark(nullptr);
      cudaGraph_t g = nullptr;
      PB_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      try {
        f();
      } catch (...) {
        cudaGraph_t g2 = nullptr;
        cudaStreamEndCapture(st, &g2);
        if (g2) cudaGraphDestroy(g2);
        throw;
      }
      PB_CUDA(cudaStreamEndCapture(st, &g));
      PB_CUDA(cudaGraphInstantiate(&exec, g, 0));
      cudaGraphDestroy(g);
      trace_mark("graph: capture + instantiate");
    }
    PB_CUDA(cudaGraphLaunch(exec, st));
    trace_mark("graph: replay");
  }
};

static int read_done(const KState* st, cudaStream_t s) {
  static int* pinned = nullptr;
  if (!pinned) PB_CUDA(cudaMallocHost(&pinned, sizeof(int)));
  PB_CUDA(cudaMemcpyAsync(pinned, &st->done, sizeof(int), cudaMemcpyDeviceToHost, s));
  PB_CUDA(cudaStreamSynchronize(s));
  return *pinned;
}

static KState read_state(const KState* st) {
  KState h;
  d2h(&h, st, sizeof(KState));
  return h;
}

static void init_state(Workspace& W, int itr0) {
  KState h;
  memset(&h, 0, sizeof(h));
  h.itr = itr0;
  h.last_inner = 1;
  h2d(W.state.p, &h, sizeof(KState));
}

// ------------------------------------------------------------------ PCG
template <class T>
static SolveOut run_pcg(const Options& o, const System<T>& S, const T* b, T* x, double* hist,
                        Workspace& W) {
  cudaStream_t st = stream();
  const int64_t np = S.np;
  DBuf r(sizeof(T) * np), p(sizeof(T) * np), q(sizeof(T) * np), s(sizeof(T) * np);
  T* R = dp<T>(r); T* P = dp<T>(p); T* Q = dp<T>(q); T* Sv = dp<T>(s);
  KState* K = W.st();
  init_state(W, 1);
  const int* gdone = &K->done;
  auto red = [&](int epi) {
    Red rr = W.red(epi);
    rr.ea.hist = hist; rr.ea.itrmax = o.itrmax; rr.ea.rtol = o.rtol; rr.ea.abstol = o.abstol;
    return rr;
  };
  int launches = 0;
  // r = b - A x; s = M^-1 r; bnorm, rnorm, rho0 = <s, r>   (pcg.f90:442-478)
  spmv<T, T>(S.A, x, R, SPMV_RES, b, nullptr, st);
  S.M.apply(np, R, Sv, nullptr, st);
  PB_CUDA(cudaMemsetAsync(P, 0, sizeof(T) * np, st));
  DotSel sel;
  sel.a[0] = 1; sel.b[0] = 1;   // <b, b>
  sel.a[1] = 2; sel.b[1] = 2;   // <r, r>
  sel.a[2] = 3; sel.b[2] = 2;   // <s, r>
  lincomb_dot<T>(np, nullptr, b, cimm(0), R, cimm(0), Sv, cimm(0), nullptr, nullptr, sel, 3,
                 red(EPI_CG_INIT), nullptr, st);
  launches += 3;
  const int chunk = 16;
  auto iterations = [&] {
    for (int it = 0; it < chunk; ++it) {
      cg_axpy2<T>(np, x, P, Sv, K, gdone, st);                            // x += alpha p; p = s + beta p
      int sa[2] = {1, 0}, sb[2] = {0, 0};
      spmv_dot<T, T>(S.A, P, Q, SPMV_Y, nullptr, nullptr, 1, sa, sb, red(EPI_CG_GAMMA), gdone, st);
      lincomb<T>(np, R, Q, cdev(&K->tmp[0]), R, cimm(1.0), nullptr, cimm(0), gdone, st);  // r = -alpha q + r
      S.M.apply(np, R, Sv, gdone, st);                                    // s = M^-1 r
      DotSel d2;
      d2.a[0] = 1; d2.b[0] = 2;   // <s, r>
      d2.a[1] = 2; d2.b[1] = 2;   // <r, r>
      lincomb_dot<T>(np, nullptr, Sv, cimm(0), R, cimm(0), nullptr, cimm(0), nullptr, nullptr, d2, 2,
                     red(EPI_CG_DOT2), gdone, st);
    }
  };
  GraphRunner G;
  const int max_chunks = o.itrmax / chunk + 2;
  for (int c = 0; c < max_chunks; ++c) {
    if (read_done(K, st)) break;
    G.launch(iterations, o.use_graphs, st);
    launches += 5 * chunk;
  }
  // x = alpha p + x   (pcg.f90:733)
  lincomb<T>(np, x, P, cdev(&K->alpha), x, cimm(1.0), nullptr, cimm(0), nullptr, st);
  launches += 1;
  KState h = read_state(K);
  SolveOut out;
  out.niter = h.niter;
  out.iret = h.iret;
  out.breakdown = h.breakdown;
  out.launches = launches;
  return out;
}

// ------------------------------------------------------------------ BiCGStab
template <class T>
static SolveOut run_bicg(const Options& o, const System<T>& S, const T* b, T* x, double* hist,
                         Workspace& W) {
  cudaStream_t st = stream();
  const int64_t np = S.np;
  const size_t vb = sizeof(T) * np;
  DBuf r(vb), r0(vb), p(vb), q(vb), pp(vb), e(vb), pe(vb), v(vb);
  T *R = dp<T>(r), *R0 = dp<T>(r0), *P = dp<T>(p), *Q = dp<T>(q), *PP = dp<T>(pp),
    *E = dp<T>(e), *PE = dp<T>(pe), *V = dp<T>(v);
  KState* K = W.st();
  init_state(W, 1);
  const int* gdone = &K->done;
  auto red = [&](int epi) {
    Red rr = W.red(epi);
    rr.ea.hist = hist; rr.ea.itrmax = o.itrmax; rr.ea.rtol = o.rtol;
    return rr;
  };
  int launches = 0;
  spmv<T, T>(S.A, x, R, SPMV_RES, b, nullptr, st);
  DotSel sel;
  sel.a[0] = 1; sel.b[0] = 1;   // <b, b>
  sel.a[1] = 2; sel.b[1] = 2;   // <r, r>
  lincomb_dot<T>(np, nullptr, b, cimm(0), R, cimm(0), nullptr, cimm(0), nullptr, nullptr, sel, 2,
                 red(EPI_BICG_INIT), nullptr, st);
  d2d(R0, R, vb);
  d2d(P, R, vb);
  launches += 2;
  const int chunk = 8;
  auto iterations = [&] {
    for (int it = 0; it < chunk; ++it) {
      S.M.apply(np, P, PP, gdone, st);                                        // pp = M^-1 p
      int sa[2] = {2, 0}, sb[2] = {0, 0};
      spmv_dot<T, T>(S.A, PP, Q, SPMV_Y, nullptr, R0, 1, sa, sb, red(EPI_BICG_C2), gdone, st);  // q, c2
      lincomb<T>(np, E, R, cimm(1.0), Q, cdev(&K->tmp[0]), nullptr, cimm(0), gdone, st);      // e = r - alpha q
      S.M.apply(np, E, PE, gdone, st);                                        // pe = M^-1 e
      int sa2[2] = {2, 0}, sb2[2] = {0, 0};
      spmv_dot<T, T>(S.A, PE, V, SPMV_Y, nullptr, E, 2, sa2, sb2, red(EPI_BICG_C3), gdone, st);  // v, <e,v>, <v,v>
      lincomb<T>(np, x, PP, cdev(&K->alpha), PE, cdev(&K->c3), x, cimm(1.0), gdone, st);   // x += alpha pp + c3 pe
      DotSel d3;
      d3.a[0] = 0; d3.b[0] = 4;   // <r, r0>
      d3.a[1] = 0; d3.b[1] = 0;   // <r, r>
      lincomb_dot<T>(np, R, E, cimm(1.0), V, cdev(&K->tmp[1]), nullptr, cimm(0), R0, nullptr, d3, 2,
                     red(EPI_BICG_END), gdone, st);                           // r = e - c3 v
      lincomb<T>(np, P, R, cimm(1.0), Q, cdev(&K->tmp[2]), P, cdev(&K->beta), gdone, st);  // p = r - beta c3 q + beta p
    }
  };
  GraphRunner G;
  const int max_chunks = o.itrmax / chunk + 2;
  for (int c = 0; c < max_chunks; ++c) {
    if (read_done(K, st)) break;
    G.launch(iterations, o.use_graphs, st);
    launches += 8 * chunk;
  }
  KState h = read_state(K);
  SolveOut out;
  out.niter = h.niter;
  out.iret = h.iret;
  out.breakdown = h.breakdown;
  out.launches = launches;
  return out;
}

// ------------------------------------------------------------------ GMRES(m)
template <class T>
static SolveOut run_gmres(const Options& o, const System<T>& S, const T* b, T* x, double* hist,
                          Workspace& W) {
  cudaStream_t st = stream();
  const int64_t np = S.np;
  const int m = o.m;
  PB_CHECK(m >= 1 && m < kMaxRed, PARCEL_B_E_ARG, "GMRES restart length %d outside [1, %d)", m, kMaxRed);
  const int64_t ldv = (np + 31) & ~int64_t(31);
  const size_t vb = sizeof(T) * np;
  DBuf r(vb), Vb(sizeof(T) * ldv * (m + 1)), pv(vb), w(vb), v0(vb), x0(vb);
  // Flexible GMRES keeps z_j = M_j^-1 v_j (the preconditioner may change between
  // columns) and updates x with Z y instead of M^-1 V y.
  const bool flex = o.flexible || S.extra != nullptr;
  DBuf Zb;
  if (flex) Zb.alloc(sizeof(T) * ldv * m);
  T* Z = dp<T>(Zb);
  // precon(in, out, az): out = M^-1 in (+ the extra stage); with the extra stage and az
  // given, az = A out comes from the stage and the caller's SpMV is skipped.
  auto precon = [&](const T* in, T* out, T* az, const int* gate) {
    if (S.extra) S.extra->begin(S, in, gate, st);
    S.M.apply(np, in, out, gate, st);
    if (S.extra) S.extra->apply(S, in, out, az, gate, st);
  };
  const int precon_launches = 1 + (S.extra ? S.extra->launches() : 0);
  DBuf hb(sizeof(double) * (m + 1) * m), eb(sizeof(double) * (m + 1)), csb(sizeof(double) * (m + 1)),
      snb(sizeof(double) * (m + 1)), yb(sizeof(double) * (m + 1));
  T *R = dp<T>(r), *V = dp<T>(Vb), *PV = dp<T>(pv), *Wv = dp<T>(w), *V0 = dp<T>(v0),
    *X0 = dp<T>(x0);
  PB_CUDA(cudaMemsetAsync(V, 0, sizeof(T) * ldv * (m + 1), st));
  KState* K = W.st();
  init_state(W, 1);
  const int* gdone = &K->done;
  const int* gskip = &K->skip_inner;
  auto red = [&](int epi, int k = 0, int j = 0) {
    Red rr = W.red(epi);
    rr.ea.hist = hist; rr.ea.itrmax = o.itrmax; rr.ea.rtol = o.rtol; rr.ea.abstol = o.abstol;
    rr.ea.h = dp<double>(hb); rr.ea.e = dp<double>(eb); rr.ea.cs = dp<double>(csb);
    rr.ea.sn = dp<double>(snb); rr.ea.m = m; rr.ea.k = k; rr.ea.j = j;
    return rr;
  };
  int launches = 0;
  {  // bnorm = ||b||
    Red rr = red(EPI_NORM2);
    rr.ea.out = &K->bnorm;
    DotSel sel;
    sel.a[0] = 1; sel.b[0] = 1;
    lincomb_dot<T>(np, nullptr, b, cimm(0), nullptr, cimm(0), nullptr, cimm(0), nullptr, nullptr, sel, 1,
                   rr, nullptr, st);
    launches += 1;
  }
  // Fused one-launch MGS (pb_mgs.cu) when the vector fits its register tiling.
  const bool fused_mgs = o.gs != PARCEL_B_GS_CGS && o.fused_mgs && mgs_supported<T>(np);
  // The staged variant reduces through per-(column, pass, CTA) slots that start every
  // cycle as all-ones bytes; the others through per-(column, pass) counters that start at 0.
  const bool staged_mgs = fused_mgs && mgs_staged<T>(np);
  const size_t nslots = (size_t)m * (m + 2) * (size_t)(num_sms() + 1);   // partials, then totals
  DBuf mparts(sizeof(double) * 2 * (size_t)std::max(1, mgs_grid<T>())),
      mctr(sizeof(unsigned) * (size_t)m * (m + 2)), merr(sizeof(int)),
      mslots(staged_mgs ? sizeof(double) * nslots : 0);
  PB_CUDA(cudaMemsetAsync(merr.p, 0, sizeof(int), st));
  int per_cycle = 0;
  auto cycle = [&] {
    per_cycle = 0;
    if (staged_mgs) {
      PB_CUDA(cudaMemsetAsync(mslots.p, 0xFF, sizeof(double) * nslots, st));
      ++per_cycle;
    } else if (fused_mgs) {
      PB_CUDA(cudaMemsetAsync(mctr.p, 0, sizeof(unsigned) * (size_t)m * (m + 2), st));
      ++per_cycle;
    }
    int sa[2] = {0, 0}, sb[2] = {0, 0};
    spmv_dot<T, T>(S.A, x, R, SPMV_RES, b, nullptr, 1, sa, sb, red(EPI_GM_RESTART), gdone, st);
    ++per_cycle;
    for (int j = 1; j <= m; ++j) {
      T* Vj = V + (size_t)(j - 1) * ldv;
      if (j == 1) {
        lincomb<T>(np, Vj, R, cdev(&K->tmp[0]), nullptr, cimm(0), nullptr, cimm(0), gskip, st);
        ++per_cycle;
      }
      T* Pj = flex ? Z + (size_t)(j - 1) * ldv : PV;
      const bool az_from_stage = S.extra && S.extra->provides_az() && fused_mgs && o.gs != PARCEL_B_GS_CGS;
      precon(Vj, Pj, az_from_stage ? Wv : nullptr, gskip);
      per_cycle += precon_launches;
      if (o.gs == PARCEL_B_GS_CGS) {
        spmv<T, T>(S.A, Pj, Wv, SPMV_Y, nullptr, gskip, st);
        multidot<T>(np, j, Wv, V, ldv, red(EPI_GM_HCGS, 0, j), gskip, st);
        cgs_update<T>(np, j, Wv, V, ldv, dp<double>(hb) + (size_t)(j - 1) * (m + 1), red(EPI_GM_NORM, 0, j),
                      gskip, st);
        per_cycle += 3;
      } else if (fused_mgs) {
        if (!az_from_stage) spmv<T, T>(S.A, Pj, Wv, SPMV_Y, nullptr, gskip, st);
        MgsArgs<T> ma;
        ma.np = np; ma.j = j; ma.w = Wv; ma.V = V; ma.ldv = ldv;
        ma.vnext = (j < m) ? V + (size_t)j * ldv : nullptr;
        ma.parts = dp<double>(mparts);
        ma.ctr = dp<unsigned>(mctr) + (size_t)(j - 1) * (m + 2);
        if (staged_mgs) {
          ma.slots = dp<double>(mslots) + (size_t)(j - 1) * (m + 2) * num_sms();
          ma.totals = dp<double>(mslots) + (size_t)m * (m + 2) * num_sms() + (size_t)(j - 1) * (m + 2);
        }
        ma.err = dp<int>(merr);
        ma.gate = gskip;
        ma.red = red(EPI_GM_NORM, 0, j);
        mgs_column<T>(ma, st);
        per_cycle += az_from_stage ? 1 : 2;
      } else {
        int sa1[2] = {0, 0}, sb1[2] = {2, 0};   // <w, v_1>
        spmv_dot<T, T>(S.A, Pj, Wv, SPMV_Y, nullptr, V, 1, sa1, sb1, red(EPI_GM_H, 1, j), gskip, st);
        ++per_cycle;
        for (int k = 1; k <= j; ++k) {
          const T* Vk = V + (size_t)(k - 1) * ldv;
          DotSel d;
          if (k < j) { d.a[0] = 0; d.b[0] = 4; }   // <w, v_{k+1}>
          else { d.a[0] = 0; d.b[0] = 0; }         // <w, w>
          const T* Vnext = (k < j) ? V + (size_t)k * ldv : nullptr;
          lincomb_dot<T>(np, Wv, Vk, cdev(&K->tmp[1]), Wv, cimm(1.0), nullptr, cimm(0), Vnext, nullptr, d, 1,
                         (k < j) ? red(EPI_GM_H, k + 1, j) : red(EPI_GM_NORM, 0, j), gskip, st);
          ++per_cycle;
        }
      }
      if (j < m && !(fused_mgs && o.gs != PARCEL_B_GS_CGS)) {
        lincomb<T>(np, V + (size_t)j * ldv, Wv, cdev(&K->tmp[2]), nullptr, cimm(0), nullptr, cimm(0), gskip, st);
        ++per_cycle;
      }
    }
    // update_xVec: y = H^-1 e; v0 = V y; x0 = M^-1 v0; x = x0 + x
    gm_backsolve(dp<double>(hb), dp<double>(eb), dp<double>(yb), m, K, gdone, st);
    if (flex) {
      sum_vec<T>(np, X0, Z, ldv, dp<double>(yb), K, gdone, st);
    } else {
      sum_vec<T>(np, V0, V, ldv, dp<double>(yb), K, gdone, st);
      S.M.apply(np, V0, X0, gdone, st);
      ++per_cycle;
    }
    lincomb<T>(np, x, X0, cimm(1.0), x, cimm(1.0), nullptr, cimm(0), gdone, st);
    gm_post(K, m, o.itrmax, st);
    per_cycle += 4;
  };
  GraphRunner G;
  const int max_cycles = o.itrmax / m + 2;
  for (int c = 0; c < max_cycles; ++c) {
    if (read_done(K, st)) break;
    G.launch(cycle, o.use_graphs, st);
    launches += per_cycle;
    if (o.on_cycle) (*o.on_cycle)(c);
  }
  KState h = read_state(K);
  int merr_h = 0;
  d2h(&merr_h, merr.p, sizeof(int));
  PB_CHECK(merr_h == 0, PARCEL_B_E_CUDA, "MGS grid barrier timed out");
  SolveOut out;
  out.niter = h.niter;
  out.iret = h.iret;
  out.breakdown = h.breakdown;
  out.launches = launches;
  return out;
}

template <class T>
SolveOut run_krylov(const Options& o, const System<T>& S, const T* b, T* x, double* hist_dev) {
  Workspace W;
  W.init();
  switch (o.solver) {
    case PARCEL_B_SOLVER_CG: return run_pcg<T>(o, S, b, x, hist_dev, W);
    case PARCEL_B_SOLVER_BICG: return run_bicg<T>(o, S, b, x, hist_dev, W);
    case PARCEL_B_SOLVER_GMRES: return run_gmres<T>(o, S, b, x, hist_dev, W);
    default:
      PB_CHECK(false, PARCEL_B_E_UNSUPPORTED, "solver %d is not provided by this build", o.solver);
  }
  return SolveOut{};
}

template void build_system<double>(const Options&, const parcel_b_crs&, bool, System<double>&);
template void build_system<float>(const Options&, const parcel_b_crs&, bool, System<float>&);
template SolveOut run_krylov<double>(const Options&, const System<double>&, const double*, double*,
                                     double*);
template SolveOut run_krylov<float>(const Options&, const System<float>&, const float*, float*,
                                    double*);

}  // namespace pb
