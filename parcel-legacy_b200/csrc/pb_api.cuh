// pb_api.cuh -- helpers shared by the C-ABI translation units (pb_capi.cu, pb_learned.cu).
#pragma once

#include <new>
#include <vector>

#include "pb_mixed.cuh"
#include "pb_solvers.cuh"

namespace pb {

// Runs f() and turns library exceptions into status codes (the reference stops the
// process on hard errors; this library returns them).
template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const Error& e) {
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error(PARCEL_B_E_NOMEM, "host allocation failed");
    return PARCEL_B_E_NOMEM;
  } catch (...) {
    set_last_error(PARCEL_B_E_ARG, "unexpected exception");
    return PARCEL_B_E_ARG;
  }
}

// Checks a CRS argument for what one process on one GPU supports.
void validate(const parcel_b_crs* A);
void set_stats(const parcel_b_stats& s);

// ||b - A x|| / ||b|| in FP64, natural layout, device arrays.
double true_relres(const DevMat<double>& A, const double* b, const double* x);

// Natural-layout vector on the device: the caller's pointer or an uploaded copy.
struct NatVec {
  DBuf own;
  double* p = nullptr;
  NatVec(const double* src, int n, bool dev) {
    if (dev) { p = const_cast<double*>(src); return; }
    own.alloc(sizeof(double) * n);
    h2d(own.p, src, sizeof(double) * n);
    p = dp<double>(own);
  }
};

// One FP64 solve on a built system.  b, x natural-layout device arrays; x in/out.
SolveOut solve_on_system(const Options& o, System<double>& S, const double* b_dev, double* x_dev,
                         std::vector<double>& hist_out, double* setup_t);

}  // namespace pb
