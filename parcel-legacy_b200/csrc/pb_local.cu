// pb_local.cu -- one process's share of a row-distributed system: the GPU side of the
// multi-process solve (parcel_b/dist.py).
//
// The reference splits the rows of A contiguously over MPI ranks (src/krylov.f90:447-470),
// exchanges the halo of x before every product (src/comm.f90:153-403, 528-597) and keeps
// the block-Jacobi blocks inside each rank, so the preconditioner needs no communication
// (src/matrix.f90:8074-8134).  A local operator holds this rank's rows with the columns
// renumbered locally (owned rows 1..n, halo values n+1..n_ext) for the product, and the
// block-Jacobi preconditioner of the owned-owned submatrix (divide_region over the owned
// rows, as every rank of the reference does).  The Krylov recurrences and the collectives
// run on the host side (parcel_b/dist.py).
#include <memory>
#include <vector>

#include "pb_api.cuh"

namespace pb {
namespace {

struct LocalOp {
  int n = 0, n_ext = 0;
  int64_t nnz = 0;
  DBuf rp, ci, va;        // rows with local column ids, 1-based
  DevMat<double> Aext;
  System<double> S;       // owned-owned submatrix (preconditioner)
  bool has_precon = false;
  DBuf rperm, zperm;
};

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" {

int parcel_b_local_create(const parcel_b_input* prm, const parcel_b_crs* A, int n_ext, parcel_b_local* out) {
  return guarded([&]() -> int {
    ensure_init();
    PB_CHECK(out && A && A->rowptr && A->col && A->val, PARCEL_B_E_ARG, "NULL argument");
    PB_CHECK(A->n > 0 && n_ext >= A->n && A->nnz >= 0 && A->nnz < (int64_t)INT32_MAX, PARCEL_B_E_ARG,
             "bad sizes: n = %d, n_ext = %d, nnz = %lld", A->n, n_ext, (long long)A->nnz);
    PB_CHECK(A->istart == 1, PARCEL_B_E_ARG, "local column ids are 1-based (istart = %d)", A->istart);
    Options o = resolve_options(prm);
    PB_CHECK(o.precon >= 0 && o.precon <= 2, PARCEL_B_E_UNSUPPORTED, "ipreflag=%d", o.precon);
    auto L = std::make_unique<LocalOp>();
    const int n = A->n;
    const int64_t nnz = A->nnz;
    L->n = n; L->n_ext = n_ext; L->nnz = nnz;
    // host copies (the arrays may live on either side)
    std::vector<int> hrp(n + 1), hci(nnz);
    std::vector<double> hva(nnz);
    auto fetch = [](void* dst, const void* src, size_t bytes) {
      if (is_device_ptr(src)) d2h(dst, src, bytes);
      else memcpy(dst, src, bytes);
    };
    fetch(hrp.data(), A->rowptr, sizeof(int) * (n + 1));
    fetch(hci.data(), A->col, sizeof(int) * nnz);
    fetch(hva.data(), A->val, sizeof(double) * nnz);
    PB_CHECK(hrp[0] == 1 && hrp[n] - 1 == nnz, PARCEL_B_E_ARG, "row pointer must run from 1 to nnz + 1");
    for (int64_t k = 0; k < nnz; ++k)
      PB_CHECK(hci[k] >= 1 && hci[k] <= n_ext, PARCEL_B_E_ARG, "column %d outside 1..%d", hci[k], n_ext);
    L->rp.alloc(sizeof(int) * (n + 1)); h2d(L->rp.p, hrp.data(), sizeof(int) * (n + 1));
    L->ci.alloc(sizeof(int) * std::max<int64_t>(nnz, 1)); h2d(L->ci.p, hci.data(), sizeof(int) * nnz);
    L->va.alloc(sizeof(double) * std::max<int64_t>(nnz, 1)); h2d(L->va.p, hva.data(), sizeof(double) * nnz);
    L->Aext.n = n; L->Aext.nnz = nnz; L->Aext.rbase = 1; L->Aext.cbase = 1;
    L->Aext.rowptr = dp<int>(L->rp); L->Aext.col = dp<int>(L->ci); L->Aext.val = dp<double>(L->va);
    // owned-owned submatrix: the halo columns dropped, row order and column order kept
    std::vector<int> orp(n + 1), oci;
    std::vector<double> ova;
    oci.reserve(nnz); ova.reserve(nnz);
    orp[0] = 1;
    for (int i = 0; i < n; ++i) {
      for (int k = hrp[i] - 1; k < hrp[i + 1] - 1; ++k)
        if (hci[k] <= n) { oci.push_back(hci[k]); ova.push_back(hva[k]); }
      orp[i + 1] = (int)oci.size() + 1;
    }
    parcel_b_crs Aoo;
    memset(&Aoo, 0, sizeof(Aoo));
    Aoo.n = n; Aoo.gn = n; Aoo.nnz = (int64_t)oci.size(); Aoo.istart = 1;
    Aoo.rowptr = orp.data(); Aoo.col = oci.data(); Aoo.val = ova.data();
    if (o.precon != PARCEL_B_PRECON_NONE) {
      build_system<double>(o, Aoo, false, L->S);
      L->has_precon = true;
      if (L->S.permuted) {
        L->rperm.alloc(sizeof(double) * L->S.np);
        L->zperm.alloc(sizeof(double) * L->S.np);
        PB_CUDA(cudaMemsetAsync(L->rperm.p, 0, sizeof(double) * L->S.np, stream()));
      }
    }
    sync();
    *out = reinterpret_cast<parcel_b_local>(L.release());
    return 0;
  });
}

int parcel_b_local_create_blocks(const parcel_b_input* prm, const parcel_b_crs* A, int n_ext, int nblocks,
                                 const int32_t* starts, parcel_b_local* out) {
  std::vector<int> s;
  const int rc = guarded([&]() -> int {
    PB_CHECK(starts != nullptr && nblocks >= 1, PARCEL_B_E_ARG, "explicit blocks: nblocks = %d, starts %s", nblocks,
             starts ? "given" : "NULL");
    s.assign(starts, starts + nblocks + 1);
    return 0;
  });
  if (rc < 0) return rc;
  ScopedBlockStarts blocks(&s);   // the owned-owned system's block split (block_split checks it)
  return parcel_b_local_create(prm, A, n_ext, out);
}

int parcel_b_local_spmv(parcel_b_local h, const double* x_ext, double* y) {
  return guarded([&]() -> int {
    PB_CHECK(h && x_ext && y, PARCEL_B_E_ARG, "NULL argument");
    PB_CHECK(is_device_ptr(x_ext) && is_device_ptr(y), PARCEL_B_E_ARG, "x_ext and y must be device arrays");
    LocalOp& L = *reinterpret_cast<LocalOp*>(h);
    spmv<double, double>(L.Aext, x_ext, y, SPMV_Y, nullptr, nullptr, stream());
    sync();
    return 0;
  });
}

int parcel_b_local_precon(parcel_b_local h, const double* r, double* z) {
  return guarded([&]() -> int {
    PB_CHECK(h && r && z, PARCEL_B_E_ARG, "NULL argument");
    PB_CHECK(is_device_ptr(r) && is_device_ptr(z), PARCEL_B_E_ARG, "r and z must be device arrays");
    LocalOp& L = *reinterpret_cast<LocalOp*>(h);
    cudaStream_t st = stream();
    if (!L.has_precon) {
      d2d(z, r, sizeof(double) * L.n);
    } else if (L.S.permuted) {
      scatter_perm<double>(L.n, dp<double>(L.rperm), r, dp<int>(L.S.pos), st);
      L.S.M.apply(L.S.np, dp<double>(L.rperm), dp<double>(L.zperm), nullptr, st);
      gather_perm<double>(L.n, z, dp<double>(L.zperm), dp<int>(L.S.pos), st);
      int err = 0;
      d2h(&err, L.S.M.ilu.err.p, sizeof(int));
      PB_CHECK(err == 0, PARCEL_B_E_CUDA, "ILU sweep kernel reported wait timeout %d", err);
    } else {
      L.S.M.apply(L.n, r, z, nullptr, st);
    }
    sync();
    return 0;
  });
}

int parcel_b_local_destroy(parcel_b_local h) {
  return guarded([&]() -> int {
    if (h) {
      sync();
      delete reinterpret_cast<LocalOp*>(h);
    }
    return 0;
  });
}

}  // extern "C"
