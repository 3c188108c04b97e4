// Tiled Cartesian kernels. Placeholder until the tiled kernel lands: the
// structured mesh is served by the general element kernel.
#include "sf_cartesian.cuh"

namespace sf {

bool cartesian_prepare(CartesianPlan& plan, int SB, int SQ, const double* A, const double* B,
                       const double* w1, const double* G0, int nx, int ny, int nz) {
  plan.ready = false;
  return false;
}

bool cartesian_supported(const CartesianPlan& plan, int dtype) { return false; }

int cartesian_launches(const CartesianPlan& plan) { return 1; }

void cartesian_apply(const CartesianPlan& plan, int dtype, const void* x, void* y,
                     cudaStream_t stream) {
  throw Error(SF_ERR_UNSUPPORTED, "tiled Cartesian kernel not available");
}

void cartesian_release(CartesianPlan& plan) { plan.ready = false; }

}  // namespace sf
