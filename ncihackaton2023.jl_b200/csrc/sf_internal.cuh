// Internal declarations shared by the sfb200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/sfb200.h"

namespace sf {

constexpr int kMaxSB = 10;
constexpr int kMaxSQ = 10;

enum MeshKind { MESH_NONE = 0, MESH_CSR = 1, MESH_STRUCTURED = 2 };
enum GeomKind { GEOM_NONE = 0, GEOM_SEPARABLE = 1, GEOM_TABLE = 2 };

// Error carried from the internals to the ABI layer.
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define SF_CUDA_CHECK(expr)                                                              \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      throw ::sf::Error(SF_ERR_CUDA, std::string(#expr " failed: ") + cudaGetErrorString(_e)); \
  } while (0)

#define SF_REQUIRE(cond, status, msg)                   \
  do {                                                  \
    if (!(cond)) throw ::sf::Error((status), (msg));    \
  } while (0)

// Device geometry shared by the element kernels.
struct Geometry {
  int kind = GEOM_NONE;
  double w1[kMaxSQ] = {0};   // separable: 1D weights, G(q) = w_i w_j w_k G0
  double G0[6] = {0};        // xx, yy, zz, xy, xz, yz
  const double* table = nullptr;  // table: [cell][6][SQ^3]
  long long table_stride = 0;     // doubles per cell (0 = one cell shared by all)
  // FP32 copy of the table for the FP32 element kernel: [cell][6][SQ^3], rows padded to
  // table32_stride floats (a multiple of 4; 0 = one cell shared by all)
  const float* table32 = nullptr;
  long long table32_stride = 0;
  const double* kappa = nullptr;  // [cell][SQ^3] or null
  const double* wdet = nullptr;   // w_q |det J| at the points, [cell][SQ^3] (the right-hand side)
  long long wdet_stride = 0;      // doubles per cell (0 = one cell shared by all)
};

// Gather/scatter description shared by the element kernels.
struct Cells {
  int mesh = MESH_NONE;
  long long ncells = 0;
  const int32_t* ids = nullptr;  // CSR: [cell][SB^3] tensor order, 0-based free id or -1
  int nx = 0, ny = 0, nz = 0;    // structured
  int p = 0;
};

// Launchers implemented in kernels_general.cu. A, B: SQ x SB row-major
// ([qp][basis]) in the kernel's 1D order.
// b += sum over cells of P_e^T (A^T (x) A^T (x) A^T) (w |det J| f) with f at the points,
// fq [cell][SQ^3] (FP64; b must be zeroed first).
void launch_general_rhs(int SB, int SQ, const double* A, const double* B, const Cells& cells,
                        const Geometry& geom, const double* fq, double* b, cudaStream_t stream);
void launch_general_apply(int dtype, int SB, int SQ, const double* A, const double* B,
                          const Cells& cells, const Geometry& geom, const void* x, void* y,
                          cudaStream_t stream);
void launch_general_diag(int dtype, int SB, int SQ, const double* A, const double* B,
                         const Cells& cells, const Geometry& geom, void* d, cudaStream_t stream);
// kbar[cell][q] = (grad ybar)_q^T G_q (grad x)_q, G without kappa (FP64 output).
void launch_kappa_vjp(int dtype, int SB, int SQ, const double* A, const double* B,
                      const Cells& cells, const Geometry& geom, const void* x, const void* ybar,
                      double* kbar, cudaStream_t stream);
// Cell-local evaluation: x_cells/y_cells [cell][SB^3] in local order; t2l (device) maps
// tensor position -> local dof.
void launch_general_evaluate(int dtype, int SB, int SQ, const double* A, const double* B,
                             long long ncells, const int32_t* t2l, const Geometry& geom,
                             const void* x_cells, void* y_cells, cudaStream_t stream);

// dst[c * dst_stride + k] = src[c * per + k] in FP32 for c < ncopy, k < per.
void convert_table32(const double* src, long long ncopy, int per, long long dst_stride, float* dst,
                     cudaStream_t stream);

// Access to an operator handle from other translation units (sfb200.cu).
struct OpShape {
  bool structured = false;  // whole 3D structured mesh, own numbering, geometry set
  int nx = 0, ny = 0, nz = 0, p = 0;
  long long n_free = 0;
};
OpShape op_shape(const sf_op* op);
// y = A x (dtype SF_F64 / SF_F32) on the stream; throws Error on failure.
void op_apply(sf_op* op, int dtype, const void* x, void* y, cudaStream_t st);
// FP64 diag(A) into d (n_free entries, written in full).
void op_diag(sf_op* op, double* d, cudaStream_t st);
// y = A x (FP64) and *out = (x, y), a fixed-order sum through `partials`
// (op_dot_partials(op) entries); s[9] holds the reduction's block counter (zero
// between calls). Nothing is summed while *skip != 0.
void op_apply_dot(sf_op* op, const double* x, double* y, double* partials, double* out, double* s,
                  const double* skip, cudaStream_t st);
long long op_dot_partials(const sf_op* op);
// A Chebyshev step fused into an FP32 apply of z on the tiled kernel: d = c2 dinv (r - A z)
// (mode 1) or c1 d + c2 dinv (r - A z) (mode 2), z_out = z + d. Returns false (and does
// nothing) when the operator does not run the tiled kernel.
bool op_cheb_apply(sf_op* op, const float* z, const float* r, const float* dinv, float* d,
                   float* z_out, double c1, double c2, int mode, cudaStream_t st);

}  // namespace sf
