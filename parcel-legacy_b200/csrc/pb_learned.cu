// pb_learned.cu -- C ABI of the learned two-level preconditioner stage (no counterpart in
// the reference).
//
// Life cycle: parcel_b_learned_create fixes the grid and the coarsening factor;
// parcel_b_learned_collect runs the plain solver (GMRES with the block-Jacobi ILU or Jacobi
// preconditioner of the caller's parameters) and turns the residual after every restart
// cycle into a training pair; parcel_b_learned_train fits the network with Adam on the GPU;
// parcel_b_learned_set_stage chooses the coarse solve (Jacobi-PCG steps, network guess on
// or off); parcel_b_solve_learned runs flexible GMRES with z = M^-1 v + P y, in FP64 or in
// FP32 inside the FP64 refinement loop, and falls back to the plain PGMRES/ILU path from
// the current iterate when the learned solve does not reach the tolerance.
//
// A training pair for a residual r = b - A x_k of the plain solve: the coarse residual
// rc = P^T r and the coarse error y* with A_c y* = rc (A_c = P^T A P, solved by many
// coarse PCG steps):  input = [bf16(rc / sigma), bf16(dhat)],  target = y* / sigma,
// sigma = rms(rc).  In the stage the network's output is the coarse PCG's starting guess.
#include <algorithm>
#include <cmath>
#include <memory>
#include <random>

#include "pb_api.cuh"
#include "pb_cnn.cuh"
#include "pb_coarse.cuh"

namespace pb {

struct Learned {
  int nx = 0, ny = 0, nz = 0, c = 1;
  cnn::Geo g;
  cnn::Net net;
  cnn::Acts train;           // training batches
  cnn::Acts kern;            // kernel-level forward / gradient calls
  DBuf tgt, loss;
  double scale = 0.0;        // target scale s: 1 / rms of the collected targets
  std::vector<DBuf> pu, pt;  // training pairs: inputs bf16 [V][2], targets float [V]
  int coarse_steps = 8;      // Jacobi-PCG iterations of the stage's coarse solve
  bool use_net = true;       // start the coarse solve from the network's guess
};

// Coarse PCG iterations behind a training target (the coarse error A_c^-1 rc).
constexpr int kTargetSteps = 400;

namespace {

void check_grid(const Learned& L, const parcel_b_crs* A) {
  PB_CHECK((int64_t)L.nx * L.ny * L.nz == (int64_t)A->n, PARCEL_B_E_ARG,
           "matrix has %d rows, the learned stage's grid %d x %d x %d", A->n, L.nx, L.ny, L.nz);
}

// Normalised coarse mean of log|diag A|: zero mean and unit variance over the coarse grid.
void make_dhat(const Learned& L, const DevMat<double>& A, DBuf& out) {
  const int64_t V = L.g.V();
  out.alloc(sizeof(float) * V);
  cnn::coarse_log_diag(L.nx, L.ny, L.nz, L.c, A.rowptr, A.col, A.val, A.cbase, dp<float>(out), stream());
  std::vector<float> h((size_t)V);
  d2h(h.data(), out.p, sizeof(float) * V);
  double m = 0.0, q = 0.0;
  for (float v : h) m += v;
  m /= (double)V;
  for (float v : h) q += (v - m) * (v - m);
  const double sd = std::sqrt(q / (double)V);
  for (float& v : h) v = sd > 1e-12 ? (float)((v - m) / sd) : 0.f;
  h2d(out.p, h.data(), sizeof(float) * V);
}

// The Galerkin coarse operator of a matrix on the handle's grid, FP64 and FP32.
struct CoarseOp {
  coarse::Grid g;
  DBuf ac64, ac32, dinv;
  void build(const Learned& L, const DevMat<double>& A) {
    g = coarse::Grid(L.nx, L.ny, L.nz, L.c);
    coarse::check_grid(g);
    const int64_t V = g.Vc();
    ac64.alloc(sizeof(double) * coarse::kTaps * V);
    ac32.alloc(sizeof(float) * coarse::kTaps * V);
    dinv.alloc(sizeof(float) * V);
    coarse::galerkin(g, A, dp<double>(ac64), stream());
    coarse::to_f32(V, dp<double>(ac64), dp<float>(ac32), dp<float>(dinv), stream());
  }
  coarse::PcgArgs args(const float* rc, const float* g0, float* y, int steps, const int* gate) const {
    coarse::PcgArgs a;
    a.g = g; a.ac = dp<float>(ac32); a.dinv = dp<float>(dinv);
    a.rc = rc; a.g0 = g0; a.y = y; a.steps = steps; a.gate = gate;
    return a;
  }
};

// Additive two-level stage: z = M^-1 v + P y with y from `steps` Jacobi-PCG iterations on
// A_c y = P^T v, started from the network's guess (use_net) or from zero.  The coarse
// branch (restriction, network, coarse solve) runs on a side stream while the ILU sweep
// runs on the solver's stream (the sweep uses one CTA per block-Jacobi block and leaves the
// other SMs idle); the prolongation joins the two.
template <class T>
struct TwoLevelStage final : ExtraStage<T> {
  const Learned* L;
  CoarseOp op;
  DBuf hc, rc, y, scal, dhat, code;
  cnn::Acts acts;
  const int* pos = nullptr;
  int64_t np = 0;
  int steps = 0;
  bool net = false;
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  TwoLevelStage(const Learned* l, const System<T>& S) : L(l) {
    op.build(*L, S.Anat);
    steps = L->coarse_steps;
    net = L->use_net;
    np = S.np;
    if (S.permuted) pos = dp<int>(S.pos);
    code.alloc(sizeof(int) * np);
    coarse::pack_coords(op.g, np, S.permuted ? dp<int>(S.rowAt) : nullptr, dp<int>(code), stream());
    const int64_t V = op.g.Vc();
    hc.alloc(sizeof(float) * 8 * op.g.Vh());
    rc.alloc(sizeof(float) * V);
    y.alloc(sizeof(float) * V);
    scal.alloc(sizeof(float) * 2);
    if (net) {
      make_dhat(*L, S.Anat, dhat);
      acts.ensure(L->g, 1, false);
      cnn::init_kernels();
    }
    PB_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    PB_CUDA(cudaEventCreateWithFlags(&ev_fork, cudaEventDisableTiming));
    PB_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
  }
  ~TwoLevelStage() override {
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (side) cudaStreamDestroy(side);
  }
  void begin(const System<T>&, const T* r, const int* gate, cudaStream_t st) override {
    PB_CUDA(cudaEventRecord(ev_fork, st));
    PB_CUDA(cudaStreamWaitEvent(side, ev_fork, 0));
    coarse::restrict_fine<T>(op.g, r, pos, dp<float>(hc), dp<float>(rc), gate, side);
    const float* g0 = nullptr;
    if (net) {
      coarse::rms(op.g.Vc(), dp<float>(rc), dp<float>(scal), gate, side);
      cnn::prep_input(L->g, dp<float>(rc), dp<float>(dhat), dp<float>(scal), dp<__nv_bfloat16>(acts.u), gate, side);
      cnn::forward(L->net, acts, gate, side);
      g0 = dp<float>(acts.y);
    }
    coarse::pcg(op.args(dp<float>(rc), g0, dp<float>(y), steps, gate), side);
    PB_CUDA(cudaEventRecord(ev_join, side));
  }
  void apply(const System<T>&, const T*, T* z, T*, const int* gate, cudaStream_t st) override {
    PB_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
    coarse::prolong_add<T>(op.g, np, dp<float>(y), dp<int>(code), z, gate, st);
  }
  bool provides_az() const override { return false; }
  int launches() const override { return net ? 12 : 4; }
};

// The caller's natural CRS matrix on the device (uploaded if its arrays live on the host).
struct NatMat {
  DBuf rp, ci, va;
  DevMat<double> A;
  explicit NatMat(const parcel_b_crs& c) {
    A.n = c.n; A.nnz = c.nnz; A.rbase = 1; A.cbase = c.istart;
    if (is_device_ptr(c.val)) {
      A.rowptr = c.rowptr; A.col = c.col; A.val = c.val;
      return;
    }
    rp.alloc(sizeof(int) * (c.n + 1)); h2d(rp.p, c.rowptr, sizeof(int) * (c.n + 1));
    ci.alloc(sizeof(int) * c.nnz); h2d(ci.p, c.col, sizeof(int) * c.nnz);
    va.alloc(sizeof(double) * c.nnz); h2d(va.p, c.val, sizeof(double) * c.nnz);
    A.rowptr = dp<int>(rp); A.col = dp<int>(ci); A.val = dp<double>(va);
  }
};

// A host or device float array of n entries as a device pointer (uploaded if needed).
struct FVec {
  DBuf own;
  const float* p = nullptr;
  FVec(const float* src, size_t n) {
    if (is_device_ptr(src)) { p = src; return; }
    own.alloc(sizeof(float) * n);
    h2d(own.p, src, sizeof(float) * n);
    p = dp<float>(own);
  }
};

// A tensor-core kernel that gave up waiting for its MMAs leaves a code in net.err.
void check_net(const Learned& L) {
  int e = 0;
  d2h(&e, L.net.err.p, sizeof(int));
  PB_CHECK(e == 0, PARCEL_B_E_CUDA, "network kernel: tensor-core completion wait timed out (code %d)", e);
}

void copy_out(float* dst, const void* src, size_t bytes) {
  if (is_device_ptr(dst)) { d2d(dst, src, bytes); sync(); }
  else d2h(dst, src, bytes);
}

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" {

int64_t parcel_b_learned_num_params(void) { return cnn::kNumParams; }

int parcel_b_learned_create(int nx, int ny, int nz, int coarsen, uint64_t seed, parcel_b_learned* out) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(out, PARCEL_B_E_ARG, "NULL handle pointer");
    PB_CHECK(nx > 0 && ny > 0 && nz > 0 && coarsen >= 1, PARCEL_B_E_ARG, "bad grid %d x %d x %d / %d", nx, ny,
             nz, coarsen);
    PB_CHECK(nx % coarsen == 0 && ny % coarsen == 0 && nz % coarsen == 0, PARCEL_B_E_ARG,
             "grid %d x %d x %d is not divisible by the coarsening factor %d", nx, ny, nz, coarsen);
    auto L = std::make_unique<Learned>();
    L->nx = nx; L->ny = ny; L->nz = nz; L->c = coarsen;
    L->g.gx = nx / coarsen; L->g.gy = ny / coarsen; L->g.gz = nz / coarsen;
    L->net.init(seed);
    L->loss.alloc(sizeof(double));
    sync();
    *out = reinterpret_cast<parcel_b_learned>(L.release());
    return 0;
  });
}

int parcel_b_learned_destroy(parcel_b_learned h) {
  return guarded([&]() -> int {
    if (h) {
      sync();
      delete reinterpret_cast<Learned*>(h);
    }
    return 0;
  });
}

int parcel_b_learned_get_params(parcel_b_learned h, float* params, double* target_scale) {
  return guarded([&]() -> int {
    PB_CHECK(h, PARCEL_B_E_ARG, "NULL handle");
    Learned& L = *reinterpret_cast<Learned*>(h);
    if (params) copy_out(params, L.net.master.p, sizeof(float) * cnn::kNumParams);
    if (target_scale) *target_scale = L.scale;
    return 0;
  });
}

int parcel_b_learned_set_params(parcel_b_learned h, const float* params, double target_scale) {
  return guarded([&]() -> int {
    PB_CHECK(h, PARCEL_B_E_ARG, "NULL handle");
    Learned& L = *reinterpret_cast<Learned*>(h);
    if (params) {
      FVec p(params, cnn::kNumParams);
      d2d(L.net.master.p, p.p, sizeof(float) * cnn::kNumParams);
      L.net.repack(stream());
    }
    if (target_scale > 0.0) L.scale = target_scale;
    sync();
    return 0;
  });
}

int parcel_b_learned_forward(parcel_b_learned h, int batch, const float* u, float* y) {
  return guarded([&]() -> int {
    PB_CHECK(h && u && y && batch >= 1, PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    const size_t M = (size_t)L.g.V() * batch;
    L.kern.ensure(L.g, batch, false);
    FVec uv(u, 2 * M);
    cnn::to_bf16(2 * M, uv.p, dp<__nv_bfloat16>(L.kern.u), stream());
    cnn::forward(L.net, L.kern, nullptr, stream());
    check_net(L);
    copy_out(y, L.kern.y.p, sizeof(float) * M);
    return 0;
  });
}

int parcel_b_learned_grad(parcel_b_learned h, int batch, const float* u, const float* target, double* loss,
                          float* grad) {
  return guarded([&]() -> int {
    PB_CHECK(h && u && target && batch >= 1, PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    const size_t M = (size_t)L.g.V() * batch;
    L.kern.ensure(L.g, batch, true);
    FVec uv(u, 2 * M), tv(target, M);
    cnn::to_bf16(2 * M, uv.p, dp<__nv_bfloat16>(L.kern.u), stream());
    cnn::loss_grad(L.net, L.kern, tv.p, 1.f, dp<double>(L.loss), stream());
    check_net(L);
    if (loss) d2h(loss, L.loss.p, sizeof(double));
    if (grad) copy_out(grad, L.net.grad.p, sizeof(float) * cnn::kNumParams);
    sync();
    return 0;
  });
}

int parcel_b_learned_adam(parcel_b_learned h, double lr) {
  return guarded([&]() -> int {
    PB_CHECK(h, PARCEL_B_E_ARG, "NULL handle");
    Learned& L = *reinterpret_cast<Learned*>(h);
    cnn::adam(L.net, (float)lr, stream());
    sync();
    return 0;
  });
}

int parcel_b_learned_collect(parcel_b_learned h, const parcel_b_input* prm, const parcel_b_crs* A, const double* b,
                             int max_pairs, int* npairs) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(h && b, PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    validate(A);
    check_grid(L, A);
    Options o = resolve_options(prm);
    PB_CHECK(o.solver == PARCEL_B_SOLVER_GMRES, PARCEL_B_E_UNSUPPORTED,
             "training pairs come from the plain GMRES solve (solver %d given)", o.solver);
    o.flexible = false;
    cudaStream_t st = stream();
    System<double> S;
    build_system<double>(o, *A, is_device_ptr(A->val), S);
    DBuf dhat;
    make_dhat(L, S.Anat, dhat);
    const int n = A->n, np = S.np;
    const int64_t V = L.g.V();
    NatVec bv(b, n, is_device_ptr(b));
    DBuf bi(sizeof(double) * np), xi(sizeof(double) * np);
    PB_CUDA(cudaMemsetAsync(bi.p, 0, sizeof(double) * np, st));
    PB_CUDA(cudaMemsetAsync(xi.p, 0, sizeof(double) * np, st));
    if (S.permuted) scatter_perm<double>(n, dp<double>(bi), bv.p, dp<int>(S.pos), st);
    else d2d(bi.p, bv.p, sizeof(double) * n);
    const int cap = std::max(1, max_pairs);
    std::vector<DBuf> xs;
    xs.emplace_back(sizeof(double) * np);   // x_0 = 0
    PB_CUDA(cudaMemsetAsync(xs.back().p, 0, sizeof(double) * np, st));
    std::function<void(int)> hook = [&](int) {
      if ((int)xs.size() < cap + 1) {
        xs.emplace_back(sizeof(double) * np);
        d2d(xs.back().p, xi.p, sizeof(double) * np);
      }
    };
    o.on_cycle = &hook;
    DBuf hist(sizeof(double) * (o.itrmax + 2));
    SolveOut so = run_krylov<double>(o, S, dp<double>(bi), dp<double>(xi), dp<double>(hist));
    PB_CHECK(so.iret == 0, PARCEL_B_E_BREAKDOWN, "the plain solve did not converge (iret %d): no training pairs",
             so.iret);
    const double bnorm = std::sqrt(dev_dot<double>(np, dp<double>(bi), dp<double>(bi)));
    CoarseOp op;
    op.build(L, S.Anat);
    DBuf r(sizeof(double) * np), hc(sizeof(float) * 8 * op.g.Vh()), rc(sizeof(float) * V), ys(sizeof(float) * V),
        scal(sizeof(float) * 2);
    PB_CUDA(cudaMemsetAsync(r.p, 0, sizeof(double) * np, st));
    const int* pos = S.permuted ? dp<int>(S.pos) : nullptr;
    int added = 0;
    for (const DBuf& xk : xs) {
      if (added >= cap) break;
      spmv<double, double>(S.A, dp<double>(xk), dp<double>(r), SPMV_RES, dp<double>(bi), nullptr, st);
      const double rel = std::sqrt(dev_dot<double>(np, dp<double>(r), dp<double>(r))) / bnorm;
      if (!(rel > 1e-8)) continue;   // converged iterates carry no error to learn
      coarse::restrict_fine<double>(op.g, dp<double>(r), pos, dp<float>(hc), dp<float>(rc), nullptr, st);
      coarse::rms(V, dp<float>(rc), dp<float>(scal), nullptr, st);
      coarse::pcg(op.args(dp<float>(rc), nullptr, dp<float>(ys), kTargetSteps, nullptr), st);
      L.pu.emplace_back(sizeof(__nv_bfloat16) * 2 * V);
      L.pt.emplace_back(sizeof(float) * V);
      cnn::prep_input(L.g, dp<float>(rc), dp<float>(dhat), dp<float>(scal), dp<__nv_bfloat16>(L.pu.back()),
                      nullptr, st);
      cnn::scale_by(V, dp<float>(ys), dp<float>(scal), dp<float>(L.pt.back()), st);
      ++added;
    }
    sync();
    if (npairs) *npairs = added;
    return 0;
  });
}

int parcel_b_learned_set_stage(parcel_b_learned h, int coarse_steps, int use_net) {
  return guarded([&]() -> int {
    PB_CHECK(h && coarse_steps >= 0 && (use_net == 0 || use_net == 1), PARCEL_B_E_ARG,
             "bad arguments (coarse_steps %d, use_net %d)", coarse_steps, use_net);
    Learned& L = *reinterpret_cast<Learned*>(h);
    L.coarse_steps = coarse_steps;
    L.use_net = use_net != 0;
    return 0;
  });
}

int parcel_b_learned_galerkin(parcel_b_learned h, const parcel_b_crs* A, double* ac) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(h && ac, PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    validate(A);
    check_grid(L, A);
    NatMat M(*A);
    CoarseOp op;
    op.build(L, M.A);
    const size_t bytes = sizeof(double) * coarse::kTaps * op.g.Vc();
    if (is_device_ptr(ac)) { d2d(ac, op.ac64.p, bytes); sync(); }
    else d2h(ac, op.ac64.p, bytes);
    return 0;
  });
}

int parcel_b_learned_coarse_solve(parcel_b_learned h, const parcel_b_crs* A, const float* rc, const float* g0,
                                  int steps, float* y) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(h && rc && y && steps >= 0, PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    validate(A);
    check_grid(L, A);
    NatMat M(*A);
    CoarseOp op;
    op.build(L, M.A);
    const int64_t V = op.g.Vc();
    FVec r(rc, V);
    std::unique_ptr<FVec> gv;
    if (g0) gv = std::make_unique<FVec>(g0, V);
    DBuf out(sizeof(float) * V);
    coarse::pcg(op.args(r.p, gv ? gv->p : nullptr, dp<float>(out), steps, nullptr), stream());
    copy_out(y, out.p, sizeof(float) * V);
    return 0;
  });
}

int parcel_b_learned_transfer(parcel_b_learned h, int to_coarse, const double* in, double* out) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(h && in && out && (to_coarse == 0 || to_coarse == 1), PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    const coarse::Grid g(L.nx, L.ny, L.nz, L.c);
    coarse::check_grid(g);
    const int64_t n = (int64_t)L.nx * L.ny * L.nz, V = g.Vc();
    cudaStream_t st = stream();
    if (to_coarse) {
      NatVec v(in, (int)n, is_device_ptr(in));
      DBuf hc(sizeof(float) * 8 * g.Vh()), rc(sizeof(float) * V);
      coarse::restrict_fine<double>(g, v.p, nullptr, dp<float>(hc), dp<float>(rc), nullptr, st);
      std::vector<float> hr((size_t)V);
      d2h(hr.data(), rc.p, sizeof(float) * V);
      std::vector<double> hd(hr.begin(), hr.end());
      if (is_device_ptr(out)) { h2d(out, hd.data(), sizeof(double) * V); sync(); }
      else memcpy(out, hd.data(), sizeof(double) * V);
    } else {
      std::vector<double> hin((size_t)V);
      if (is_device_ptr(in)) d2h(hin.data(), in, sizeof(double) * V);
      else memcpy(hin.data(), in, sizeof(double) * V);
      std::vector<float> hf(hin.begin(), hin.end());
      DBuf yc(sizeof(float) * V), z(sizeof(double) * n), code(sizeof(int) * n);
      h2d(yc.p, hf.data(), sizeof(float) * V);
      PB_CUDA(cudaMemsetAsync(z.p, 0, sizeof(double) * n, st));
      coarse::pack_coords(g, n, nullptr, dp<int>(code), st);
      coarse::prolong_add<double>(g, n, dp<float>(yc), dp<int>(code), dp<double>(z), nullptr, st);
      if (is_device_ptr(out)) { d2d(out, z.p, sizeof(double) * n); sync(); }
      else d2h(out, z.p, sizeof(double) * n);
    }
    return 0;
  });
}

int parcel_b_learned_num_pairs(parcel_b_learned h) {
  return h ? (int)reinterpret_cast<Learned*>(h)->pu.size() : 0;
}

int parcel_b_learned_train(parcel_b_learned h, int steps, int batch, double lr, uint64_t seed, double* first_loss,
                           double* last_loss) {
  return guarded([&]() -> int {
    PB_CHECK(h && steps >= 1 && batch >= 1 && lr > 0.0, PARCEL_B_E_ARG, "bad arguments");
    Learned& L = *reinterpret_cast<Learned*>(h);
    const int np = (int)L.pu.size();
    PB_CHECK(np > 0, PARCEL_B_E_ARG, "no training pairs: call parcel_b_learned_collect first");
    cudaStream_t st = stream();
    const int64_t V = L.g.V();
    if (L.scale <= 0.0) {
      double q = 0.0;
      std::vector<float> hv((size_t)V);
      for (const DBuf& p : L.pt) {
        d2h(hv.data(), p.p, sizeof(float) * V);
        for (float v : hv) q += (double)v * v;
      }
      const double rms = std::sqrt(q / ((double)V * np));
      L.scale = rms > 0.0 ? 1.0 / rms : 1.0;
    }
    L.train.ensure(L.g, batch, true);
    L.tgt.alloc(sizeof(float) * V * batch);
    std::mt19937_64 rng(seed);
    for (int s = 0; s < steps; ++s) {
      for (int b = 0; b < batch; ++b) {
        const int k = (int)(rng() % (uint64_t)np);
        d2d(dp<char>(L.train.u) + sizeof(__nv_bfloat16) * 2 * V * b, L.pu[k].p, sizeof(__nv_bfloat16) * 2 * V);
        d2d(dp<float>(L.tgt) + V * b, L.pt[k].p, sizeof(float) * V);
      }
      cnn::loss_grad(L.net, L.train, dp<float>(L.tgt), (float)L.scale, dp<double>(L.loss), st);
      if (s == 0 && first_loss) d2h(first_loss, L.loss.p, sizeof(double));
      cnn::adam(L.net, (float)lr, st);
    }
    if (last_loss) {
      cnn::loss_grad(L.net, L.train, dp<float>(L.tgt), (float)L.scale, dp<double>(L.loss), st);
      d2h(last_loss, L.loss.p, sizeof(double));
    }
    check_net(L);
    return 0;
  });
}

}  // extern "C"

namespace pb {
namespace {

// nrhs solves of A x_k = b_k with one set-up (layout, ILU factors, learned stage).  B and X
// hold the right-hand sides and solutions one after the other (natural layout).
int solve_learned_impl(const parcel_b_input* prm, const parcel_b_crs* A, Learned* L, int nrhs, const double* B,
                       double* X, double* reshistory, int* niter, int* iret) {
  ensure_init();
  validate(A);
  PB_CHECK(B && X && nrhs >= 1, PARCEL_B_E_ARG, "b and x must not be NULL, nrhs >= 1");
  if (L) check_grid(*L, A);
  Options o = resolve_options(prm);
  PB_CHECK(o.solver == PARCEL_B_SOLVER_GMRES, PARCEL_B_E_UNSUPPORTED,
           "the learned stage runs inside flexible GMRES (solver %d given)", o.solver);
  PB_CHECK(o.precon >= 0 && o.precon <= 2, PARCEL_B_E_UNSUPPORTED, "ipreflag=%d is not provided", o.precon);
  o.flexible = true;
  const double t0 = now_s();
  const int n = A->n;
  const bool dev = is_device_ptr(A->val);
  const bool bdev = is_device_ptr(B), xdev = is_device_ptr(X);
  parcel_b_stats stt;
  memset(&stt, 0, sizeof(stt));
  const bool mixed = o.inner == PARCEL_B_INNER_FP32_REFINE;
  std::unique_ptr<System<float>> S32;
  std::unique_ptr<System<double>> S64;
  std::unique_ptr<TwoLevelStage<float>> st32;
  std::unique_ptr<TwoLevelStage<double>> st64;
  if (mixed) {
    S32 = std::make_unique<System<float>>();
    build_system<float>(o, *A, dev, *S32);
    if (L) { st32 = std::make_unique<TwoLevelStage<float>>(L, *S32); S32->extra = st32.get(); }
    stt.ilu_levels_max = S32->ilu_levels_max;
    stt.ilu_nblocks = S32->ilu_nblocks;
  } else {
    S64 = std::make_unique<System<double>>();
    build_system<double>(o, *A, dev, *S64);
    if (L) { st64 = std::make_unique<TwoLevelStage<double>>(L, *S64); S64->extra = st64.get(); }
    stt.ilu_levels_max = S64->ilu_levels_max;
    stt.ilu_nblocks = S64->ilu_nblocks;
  }
  // natural matrix on the device for the true residual (the FP64 system keeps one)
  DevMat<double> An;
  An.n = n; An.nnz = A->nnz; An.rbase = 1; An.cbase = A->istart;
  DBuf up_rp, up_ci, up_va;
  if (S64) {
    An = S64->Anat;
  } else if (dev) {
    An.rowptr = A->rowptr; An.col = A->col; An.val = A->val;
  } else {
    up_rp.alloc(sizeof(int) * (n + 1)); h2d(up_rp.p, A->rowptr, sizeof(int) * (n + 1));
    up_ci.alloc(sizeof(int) * A->nnz); h2d(up_ci.p, A->col, sizeof(int) * A->nnz);
    up_va.alloc(sizeof(double) * A->nnz); h2d(up_va.p, A->val, sizeof(double) * A->nnz);
    An.rowptr = dp<int>(up_rp); An.col = dp<int>(up_ci); An.val = dp<double>(up_va);
  }
  sync();
  const double t1 = now_s();
  std::unique_ptr<System<double>> Sfb;   // plain system, built only if a fallback is needed
  int total = 0, worst = 0;
  double worst_rel = 0.0;
  std::vector<double> hist;
  for (int k = 0; k < nrhs; ++k) {
    NatVec bv(B + (size_t)k * n, n, bdev), xv(X + (size_t)k * n, n, xdev);
    hist.clear();
    SolveOut so;
    if (mixed) {
      MixedResult mr = solve_mixed_on(o, *S32, bv.p, xv.p, hist, nullptr);
      so.niter = mr.niter; so.iret = mr.iret; so.launches = mr.launches;
      stt.refine_steps += mr.refine_steps;
      stt.true_relres_dd = std::max(stt.true_relres_dd, mr.true_relres_dd);
    } else {
      so = solve_on_system(o, *S64, bv.p, xv.p, hist, nullptr);
    }
    // The true FP64 residual decides; the plain PGMRES/ILU path finishes what the
    // learned solve left.
    double rel = true_relres(An, bv.p, xv.p);
    if (!(rel < o.rtol) && so.iret >= 0 && so.niter < o.itrmax) {
      Options op = resolve_options(prm);
      op.itrmax = o.itrmax - so.niter;
      if (!Sfb) {
        Sfb = std::make_unique<System<double>>();
        build_system<double>(op, *A, dev, *Sfb);
      }
      std::vector<double> h2;
      SolveOut s2 = solve_on_system(op, *Sfb, bv.p, xv.p, h2, nullptr);
      for (double v : h2) hist.push_back(v);
      so.niter += s2.niter;
      so.iret = s2.iret;
      so.launches += s2.launches;
      stt.fallback += 1;
      rel = true_relres(An, bv.p, xv.p);
    }
    if (!xdev) d2h(X + (size_t)k * n, xv.p, sizeof(double) * n);
    if (niter) niter[k] = so.niter;
    if (iret) iret[k] = so.iret;
    if (so.iret < 0) { worst = so.iret; break; }
    if (so.iret > worst) worst = so.iret;
    total += so.niter;
    stt.kernel_launches += so.launches;
    worst_rel = std::max(worst_rel, rel);
  }
  if (nrhs == 1 && reshistory && !hist.empty()) {
    size_t cnt = std::min<size_t>(hist.size(), (size_t)std::max(o.itrmax, 0));
    if (is_device_ptr(reshistory)) { h2d(reshistory, hist.data(), sizeof(double) * cnt); sync(); }
    else memcpy(reshistory, hist.data(), sizeof(double) * cnt);
  }
  const double t2 = now_s();
  stt.true_relres = worst_rel;
  stt.setup_s = t1 - t0;
  stt.solve_s = t2 - t1;
  stt.total_s = t2 - t0;
  stt.niter = total;
  stt.iret = worst;
  set_stats(stt);
  return worst < 0 ? worst : 0;
}

}  // namespace
}  // namespace pb

extern "C" {

int parcel_b_solve_learned(const parcel_b_input* prm, const parcel_b_crs* A, parcel_b_learned h, const double* b,
                           double* x, double* reshistory, int* niter, int* iret) {
  int rc = guarded([&]() -> int {
    return solve_learned_impl(prm, A, reinterpret_cast<Learned*>(h), 1, b, x, reshistory, niter, iret);
  });
  if (rc < 0 && iret) *iret = rc;
  return rc;
}

int parcel_b_solve_learned_many(const parcel_b_input* prm, const parcel_b_crs* A, parcel_b_learned h, int nrhs,
                                const double* b, double* x, int* niter, int* iret) {
  int rc = guarded([&]() -> int {
    return solve_learned_impl(prm, A, reinterpret_cast<Learned*>(h), nrhs, b, x, nullptr, niter, iret);
  });
  if (rc < 0 && iret) *iret = rc;
  return rc;
}

}  // extern "C"
