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
// Reliable update: r32 = float(b - q), xs32 = 0, optionally p32 = dinv r32;
// writes s[CG_RZ_NEW] = (r32, dinv r32) and s[CG_RR] = FP64 (r, r).
void mixed_residual(const double* b, const double* q, const float* dinv, float* r32, float* xs32,
                    float* p32, bool set_p, long long n, double* partials, double* s,
                    cudaStream_t st);
// x += xs32
void mixed_fold(double* x, const float* xs32, long long n, cudaStream_t st);
void copy_scalar(double* s, int dst, int src, cudaStream_t st);

}  // namespace sf
