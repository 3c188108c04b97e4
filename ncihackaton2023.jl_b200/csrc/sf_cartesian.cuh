// Tiled Cartesian kernels (kernels_cartesian.cu): constant-coefficient
// axis-aligned affine cells on a structured mesh.
#pragma once

#include "sf_internal.cuh"

namespace sf {

struct CartesianPlan {
  bool ready = false;
  int SB = 0, SQ = 0, nx = 0, ny = 0, nz = 0;
  double M[kMaxSB * kMaxSB] = {0};  // 1D element mass A^T W A, lexicographic order
  double K[kMaxSB * kMaxSB] = {0};  // 1D element stiffness B^T W B
  double c[3] = {0, 0, 0};          // G0 diagonal: xx, yy, zz
  int choice[2] = {0, 0};           // tile candidate per dtype (0: FP64, 1: FP32)
  // z-slab of a larger mesh: nz cells of it; vectors hold the grid levels z0 p .. (z0 + nz + 1) p
  // (one halo plane below, p above); outputs on levels z0 p + 1 .. (z0 + nz) p, the last one
  // left out when it is the mesh's Dirichlet boundary (slab_top)
  bool slab = false, slab_top = false;
  int D = 3;  // 2: an nx x ny quadrilateral mesh (nz unused)
};

// A Chebyshev smoothing step of the multigrid smoother fused into an FP32 apply of z
// (the apply's x): with az = (A z) at every point,
//   d = c2 dinv (r - az) (mode 1) or c1 d + c2 dinv (r - az) (mode 2),  z_out = z + d,
// and nothing is written to the apply's y. z_out is another buffer than z.
struct CartCheb {
  const void* r = nullptr;
  const void* dinv = nullptr;
  void* d = nullptr;
  void* z_out = nullptr;
  double c1 = 0.0, c2 = 0.0;
  int mode = 0;  // 0: none
};

// Optional work fused into one apply of the CG loop.
struct CartFuse {
  double* dot = nullptr;  // per-tile partial sums of x*y (cartesian_tiles entries)
  int tz0 = 0, tz1 = -1;  // tz1 >= 0: apply only the tile rows tz0 <= tz < tz1 (z-rows of tiles)
  // x and y in another numbering of the free points: num[i] is the index of lexicographic
  // point i (a whole mesh; no dot or tile-row range with it)
  const int32_t* num = nullptr;
  CartCheb cheb;  // mode != 0: the Chebyshev step instead of writing y (FP32, whole mesh)
};

// Builds the 1D operators; returns false when no tiled kernel exists for SB.
bool cartesian_prepare(CartesianPlan& plan, int SB, int SQ, const double* A, const double* B,
                       const double* w1, const double* G0, int nx, int ny, int nz, int D = 3);
bool cartesian_supported(const CartesianPlan& plan, int dtype);
// Tile-shape candidates for the plan's order and dtype (timed by sf_autotune).
int cartesian_candidates(const CartesianPlan& plan, int dtype);
const char* cartesian_candidate_name(const CartesianPlan& plan, int dtype, int k);
void cartesian_apply_candidate(const CartesianPlan& plan, int dtype, int k, const void* x, void* y,
                               cudaStream_t stream);
int cartesian_launches(const CartesianPlan& plan);  // kernel launches per apply

// Batched (persistent) form. A problem descriptor of cartesian_batch_desc_bytes(dtype)
// bytes is written per problem; the call returns the problem's work items
// (tiles of candidate `cand` x nrhs). One launch then applies every problem
// of a group that shares `proto`'s order and 1D operators, with CTAs taking
// work items from *d_counter (which must be zero at launch).
size_t cartesian_batch_desc_bytes(int dtype);
long long cartesian_batch_desc(const CartesianPlan& plan, int dtype, int cand, const void* x,
                               void* y, long long ldx, long long ldy, int nrhs, long long first,
                               void* out);
void cartesian_batch_launch(const CartesianPlan& proto, int dtype, int cand, const void* d_desc,
                            int nprob, long long total, unsigned long long* d_counter, bool iso,
                            cudaStream_t st);
void cartesian_apply(const CartesianPlan& plan, int dtype, const void* x, void* y,
                     cudaStream_t stream, const CartFuse& fuse = CartFuse{});
// diag(A) at the points an apply writes (same layout as y; other points untouched).
void cartesian_diag(const CartesianPlan& plan, double* d, cudaStream_t stream);
// Cells per tile along z of the chosen candidate (a tile row covers EZ cell layers).
int cartesian_tile_ez(const CartesianPlan& plan, int dtype);
// Tiles (CTAs) of one apply with the chosen candidate: the entries CartFuse::dot receives.
long long cartesian_tiles(const CartesianPlan& plan, int dtype);
void cartesian_release(CartesianPlan& plan);

}  // namespace sf
