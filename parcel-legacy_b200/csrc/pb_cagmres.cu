// pb_cagmres.cu -- CA-GMRES(s, t) (placeholder until the s-step kernels land).
#include "pb_mixed.cuh"

namespace pb {

SolveOut solve_cagmres(const Options& o, System<double>& S, const double* b, double* x,
                       std::vector<double>& hist, double* setup_t) {
  (void)o; (void)S; (void)b; (void)x; (void)hist; (void)setup_t;
  PB_CHECK(false, PARCEL_B_E_UNSUPPORTED, "CA-GMRES is not built yet");
  return SolveOut{};
}

}  // namespace pb
