// Device-side conjugate-gradient building blocks (kernels_vec.cu).
#pragma once

#include "sf_internal.cuh"

namespace sf {

// Slots of the device scalar array used by the CG kernels.
enum CgSlot {
  CG_RZ = 0,      // current (r, z)
  CG_PQ = 1,      // (p, A p)
  CG_RZ_NEW = 2,  // (r, z) after the update; CG_RR must follow it
  CG_RR = 3,      // (r, r)
  CG_BB = 4,      // (b, b); must follow CG_RR
  CG_DONE = 5,    // 0 running; 1 converged by this iteration's update; 2 finished; 3 non-finite
  CG_ITERS = 6,   // completed iterations
  CG_TOL2 = 7,    // stopping threshold on (r, r); negative: never stop on the device
  CG_REPORTS = 8,   // direction steps run since cg_init (the number of the last report)
  CG_COUNTER = 9,   // storage of the unsigned block counter of the last-block reductions
  CG_PART_PQ = 10,  // distributed CG: this rank's (p, q), then (after the caller's sum) all ranks'
  CG_PART_RZ = 11,  // distributed CG: (r, dinv r), likewise
  CG_PART_RR = 12,  // distributed CG: (r, r), likewise
  CG_NSLOTS = 16
};

constexpr int kRedBlocks = 148 * 8;  // reduction grid: 8 blocks of 256 threads per SM

// One CG iteration on the device is:
//   q = A p and (p, q) -> s[PQ] (the tiled apply writes per-tile partial sums and
//                 dot_finish adds them; the general apply is followed by vec_dot);
//   cg_update:    alpha = RZ / PQ; r -= alpha q; sums (r, dinv r), (r, r) -> RZ_NEW, RR,
//                 and DONE = 1 once RR <= TOL2 (3 if RR is not finite);
//   cg_direction: x += alpha p; p = dinv r + beta p (beta = RZ_NEW / RZ) unless DONE = 1;
//                 then RZ = RZ_NEW, ITERS += 1, DONE 1 -> 2, REPORTS += 1, and (with a
//                 report buffer) RR, DONE, ITERS, REPORTS written to mapped host memory.
// Every kernel of an iteration does nothing once DONE >= 2 (all but the direction step
// once DONE != 0), so the host may queue iterations past convergence and poll the
// reports a few iterations behind the device without changing the result.
// The reductions end in the last block to finish, which uses the counter at
// s[CG_COUNTER]: cg_reset or cg_init must zero it before the first reduction.

// out = sum of partials[0..nparts) in a fixed order; nothing while *skip != 0
void dot_finish(const double* partials, long long nparts, double* out, const double* skip,
                cudaStream_t st);
// Zeroes all scalars (and the counter) of a solve.
void cg_reset(double* s, cudaStream_t st);
// *out = (a, b); nothing while *skip != 0. s: the scalar array (its counter is used).
template <typename T>
void vec_dot(const T* a, const T* b, long long n, double* partials, double* out, double* s,
             const double* skip, cudaStream_t st);
template <typename T>
void cg_start(const T* b, const T* q, const T* dinv, T* r, T* p, long long n, double* partials,
              double* s, cudaStream_t st);
// After cg_start or mixed_residual: RZ = RZ_NEW, ITERS = 0, TOL2 = reltol2 * max(BB, 1 if
// BB = 0) (or -1 for reltol2 < 0), DONE = 2 if RR <= TOL2 already (3 if RR is not finite).
void cg_init(double* s, double reltol2, cudaStream_t st);
// distributed: alpha = RZ / s[PART_PQ] (then PQ = PART_PQ), sums into PART_RZ, PART_RR and
// no stopping test (cg_check does it once the caller has summed them over ranks)
template <typename T>
void cg_update(double* s, T* r, const T* q, const T* dinv, long long n, double* partials,
               cudaStream_t st, bool distributed = false);
// distributed: RZ_NEW = PART_RZ, RR = PART_RR and the stopping test (nothing once DONE != 0)
void cg_check(double* s, cudaStream_t st);
template <typename T>
void cg_direction(double* s, T* x, T* p, const T* r, const T* dinv, long long n, double* report,
                  cudaStream_t st);
template <typename T>
void vec_invert(const double* d, T* dinv, long long n, cudaStream_t st);

// Inverse Jacobi diagonal of a whole-mesh 3D Cartesian operator as a table: on such a
// mesh diag(A) at a free point depends only on the point's position inside its cell,
// so D^-1 at free point (x, y, z) (flat index x + nfx (y + nfy z)) is
// tab[((z+1) % p) p^2 + ((y+1) % p) p + (x+1) % p], p^3 FP64 entries on the device.
struct JacobiTable {
  const double* tab = nullptr;
  int p = 0, nfx = 0, nfy = 0;
};
// cg_update and cg_direction (non-distributed) with D^-1 from the table instead of a
// vector: two vector sweeps fewer per iteration.
template <typename T>
void cg_update_table(double* s, T* r, const T* q, const JacobiTable& J, long long n,
                     double* partials, cudaStream_t st);
template <typename T>
void cg_direction_table(double* s, T* x, T* p, const T* r, const JacobiTable& J, long long n,
                        double* report, cudaStream_t st);
// y[i] = x[idx[i]] for a vector of dtype SF_F64 / SF_F32 (n entries, idx a permutation
// of 0..n-1; the inverse permutation undoes it).
void permute_gather(int dtype, const void* x, const int32_t* idx, void* y, long long n,
                    cudaStream_t st);
// Reliable update: r32 = float(b - q), xs32 = 0, optionally p32 = dinv r32;
// writes s[CG_RZ_NEW] = (r32, dinv r32) and s[CG_RR] = FP64 (r, r).
void mixed_residual(const double* b, const double* q, const float* dinv, float* r32, float* xs32,
                    float* p32, bool set_p, long long n, double* partials, double* s,
                    cudaStream_t st);
// x += xs32
void mixed_fold(double* x, const float* xs32, long long n, cudaStream_t st);
void copy_scalar(double* s, int dst, int src, cudaStream_t st);

}  // namespace sf
