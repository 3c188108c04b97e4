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
  CG_RES64 = 5,   // mixed precision: FP64 outer residual (r, r)
  CG_NSLOTS = 8
};

constexpr int kRedBlocks = 148 * 4;  // reduction grid: 4 blocks per SM

template <typename T>
void vec_dot(const T* a, const T* b, long long n, double* partials, double* out, cudaStream_t st);
template <typename T>
void cg_start(const T* b, const T* q, const T* dinv, T* r, T* p, long long n, double* partials,
              double* s, cudaStream_t st);
template <typename T>
void cg_update(const double* s_in, T* x, const T* p, T* r, const T* q, const T* dinv, long long n,
               double* partials, double* s, cudaStream_t st);
template <typename T>
void cg_direction(double* s, T* p, const T* r, const T* dinv, long long n, cudaStream_t st);
template <typename T>
void vec_invert(const double* d, T* dinv, long long n, cudaStream_t st);
void mixed_residual(const double* b, const double* q, double* r, long long n, double* partials,
                    double* s, int slot, cudaStream_t st);
void mixed_scale(const double* s, int slot, const double* r, float* r32, float* d32, long long n,
                 cudaStream_t st);
void mixed_correct(const double* s, int slot, double* x, const float* d32, long long n,
                   cudaStream_t st);

}  // namespace sf
