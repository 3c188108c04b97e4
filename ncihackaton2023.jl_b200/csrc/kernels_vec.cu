// Vector kernels of the device conjugate-gradient solver.
//
// These replace the host BLAS-1 work of IterativeSolvers.cg! (called at
// profiling/drivers.jl:85-95). The CG scalars (alpha, beta, dot products)
// live in a small device array, so an iteration launches without a host
// round trip. Reductions are deterministic: a fixed grid writes per-block
// partial sums (FP64 for both vector types), and a one-block kernel adds
// them in a fixed order.
#include "sf_cg.cuh"

namespace sf {
namespace {

constexpr int kThreads = 256;

// Block-wide sum of NV doubles; returns the totals in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][kThreads / 32];
#pragma unroll
  for (int k = 0; k < NV; ++k) {
    double s = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double s = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) s += sh[k][w];
      v[k] = s;
    }
  }
}

// partials[b*NV + k]: per-block sums. One block adds them and stores to out[k].
template <int NV>
__global__ void k_finish(const double* __restrict__ partials, int nblocks, double* __restrict__ out) {
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kThreads) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += partials[b * NV + k];
  }
  block_sum<NV>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = v[k];
  }
}

// out = a . b
template <typename T>
__global__ void k_dot(const T* __restrict__ a, const T* __restrict__ b, long long n,
                      double* __restrict__ partials) {
  double v[1] = {0.0};
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads)
    v[0] += (double)a[i] * (double)b[i];
  block_sum<1>(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
}

// Start of CG: r = b - q (q = A x0, or q = null for x0 = 0), z = dinv r, p = z.
// Sums: (r,z), (r,r), (b,b).
template <typename T>
__global__ void k_cg_start(const T* __restrict__ b, const T* __restrict__ q,
                           const T* __restrict__ dinv, T* __restrict__ r, T* __restrict__ p,
                           long long n, double* __restrict__ partials) {
  double v[3] = {0.0, 0.0, 0.0};
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    const T bi = b[i];
    const T ri = q ? (T)(bi - q[i]) : bi;
    const T zi = dinv ? (T)(dinv[i] * ri) : ri;
    r[i] = ri;
    p[i] = zi;
    v[0] += (double)ri * (double)zi;
    v[1] += (double)ri * (double)ri;
    v[2] += (double)bi * (double)bi;
  }
  block_sum<3>(v);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 3 + 0] = v[0];
    partials[blockIdx.x * 3 + 1] = v[1];
    partials[blockIdx.x * 3 + 2] = v[2];
  }
}

// alpha = s[RZ] / s[PQ]; x += alpha p; r -= alpha q. Sums: (r, dinv r), (r, r).
template <typename T>
__global__ void k_cg_update(const double* __restrict__ s, T* __restrict__ x,
                            const T* __restrict__ p, T* __restrict__ r, const T* __restrict__ q,
                            const T* __restrict__ dinv, long long n, double* __restrict__ partials) {
  const double alpha_d = s[CG_RZ] / s[CG_PQ];
  const T alpha = (T)alpha_d;
  double v[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    x[i] = fma(alpha, p[i], x[i]);
    const T ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    const T zi = dinv ? (T)(dinv[i] * ri) : ri;
    v[0] += (double)ri * (double)zi;
    v[1] += (double)ri * (double)ri;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2 + 0] = v[0];
    partials[blockIdx.x * 2 + 1] = v[1];
  }
}

// beta = s[RZ_NEW] / s[RZ]; p = dinv r + beta p; then RZ <- RZ_NEW (one thread, after use).
template <typename T>
__global__ void k_cg_direction(const double* __restrict__ s, T* __restrict__ p,
                               const T* __restrict__ r, const T* __restrict__ dinv, long long n) {
  const T beta = (T)(s[CG_RZ_NEW] / s[CG_RZ]);
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    const T zi = dinv ? (T)(dinv[i] * r[i]) : r[i];
    p[i] = fma(beta, p[i], zi);
  }
}

__global__ void k_copy_scalar(double* __restrict__ s, int dst, int src) {
  if (threadIdx.x == 0 && blockIdx.x == 0) s[dst] = s[src];
}

// dinv = 1 / d (FP64 in, T out)
template <typename T>
__global__ void k_invert(const double* __restrict__ d, T* __restrict__ dinv, long long n) {
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads)
    dinv[i] = (T)(1.0 / d[i]);
}

// Reliable update of the mixed-precision CG: the FP64 true residual
// r = b - A64 x replaces the FP32 recurrence residual. Writes r32 = (float) r,
// zeroes the FP32 partial solution xs32, and (when set_p) starts the search
// direction p32 = dinv r32. Sums: (r32, dinv r32) and the FP64 (r, r).
__global__ void k_mixed_residual(const double* __restrict__ b, const double* __restrict__ q,
                                 const float* __restrict__ dinv, float* __restrict__ r32,
                                 float* __restrict__ xs32, float* __restrict__ p32, int set_p,
                                 long long n, double* __restrict__ partials) {
  double v[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads) {
    const double ri = b[i] - q[i];
    const float rf = (float)ri;
    const float zf = dinv[i] * rf;
    r32[i] = rf;
    xs32[i] = 0.0f;
    if (set_p) p32[i] = zf;
    v[0] += (double)rf * (double)zf;
    v[1] += ri * ri;
  }
  block_sum<2>(v);
  if (threadIdx.x == 0) {
    partials[blockIdx.x * 2 + 0] = v[0];
    partials[blockIdx.x * 2 + 1] = v[1];
  }
}

// x64 += xs32 (fold the FP32 partial solution into the FP64 solution)
__global__ void k_fold(double* __restrict__ x, const float* __restrict__ xs32, long long n) {
  for (long long i = (long long)blockIdx.x * kThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kThreads)
    x[i] += (double)xs32[i];
}

int grid_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b > kRedBlocks) b = kRedBlocks;
  if (b < 1) b = 1;
  return (int)b;
}

}  // namespace

template <typename T>
void vec_dot(const T* a, const T* b, long long n, double* partials, double* out,
             cudaStream_t st) {
  const int g = grid_for(n);
  k_dot<T><<<g, kThreads, 0, st>>>(a, b, n, partials);
  k_finish<1><<<1, kThreads, 0, st>>>(partials, g, out);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_start(const T* b, const T* q, const T* dinv, T* r, T* p, long long n, double* partials,
              double* s, cudaStream_t st) {
  const int g = grid_for(n);
  k_cg_start<T><<<g, kThreads, 0, st>>>(b, q, dinv, r, p, n, partials);
  k_finish<3><<<1, kThreads, 0, st>>>(partials, g, s + CG_RZ_NEW);  // RZ_NEW, RR, BB
  k_copy_scalar<<<1, 32, 0, st>>>(s, CG_RZ, CG_RZ_NEW);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_update(const double* s_in, T* x, const T* p, T* r, const T* q, const T* dinv, long long n,
               double* partials, double* s, cudaStream_t st) {
  const int g = grid_for(n);
  k_cg_update<T><<<g, kThreads, 0, st>>>(s_in, x, p, r, q, dinv, n, partials);
  k_finish<2><<<1, kThreads, 0, st>>>(partials, g, s + CG_RZ_NEW);  // RZ_NEW, RR
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_direction(double* s, T* p, const T* r, const T* dinv, long long n, cudaStream_t st) {
  const int g = grid_for(n);
  k_cg_direction<T><<<g, kThreads, 0, st>>>(s, p, r, dinv, n);
  k_copy_scalar<<<1, 32, 0, st>>>(s, CG_RZ, CG_RZ_NEW);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void vec_invert(const double* d, T* dinv, long long n, cudaStream_t st) {
  k_invert<T><<<grid_for(n), kThreads, 0, st>>>(d, dinv, n);
  SF_CUDA_CHECK(cudaGetLastError());
}

void mixed_residual(const double* b, const double* q, const float* dinv, float* r32, float* xs32,
                    float* p32, bool set_p, long long n, double* partials, double* s,
                    cudaStream_t st) {
  const int g = grid_for(n);
  k_mixed_residual<<<g, kThreads, 0, st>>>(b, q, dinv, r32, xs32, p32, set_p ? 1 : 0, n, partials);
  k_finish<2><<<1, kThreads, 0, st>>>(partials, g, s + CG_RZ_NEW);  // RZ_NEW, RR (FP64 true)
  SF_CUDA_CHECK(cudaGetLastError());
}

void mixed_fold(double* x, const float* xs32, long long n, cudaStream_t st) {
  k_fold<<<grid_for(n), kThreads, 0, st>>>(x, xs32, n);
  SF_CUDA_CHECK(cudaGetLastError());
}

void copy_scalar(double* s, int dst, int src, cudaStream_t st) {
  k_copy_scalar<<<1, 32, 0, st>>>(s, dst, src);
  SF_CUDA_CHECK(cudaGetLastError());
}

template void vec_dot<double>(const double*, const double*, long long, double*, double*, cudaStream_t);
template void vec_dot<float>(const float*, const float*, long long, double*, double*, cudaStream_t);
template void cg_start<double>(const double*, const double*, const double*, double*, double*,
                               long long, double*, double*, cudaStream_t);
template void cg_start<float>(const float*, const float*, const float*, float*, float*, long long,
                              double*, double*, cudaStream_t);
template void cg_update<double>(const double*, double*, const double*, double*, const double*,
                                const double*, long long, double*, double*, cudaStream_t);
template void cg_update<float>(const double*, float*, const float*, float*, const float*,
                               const float*, long long, double*, double*, cudaStream_t);
template void cg_direction<double>(double*, double*, const double*, const double*, long long,
                                   cudaStream_t);
template void cg_direction<float>(double*, float*, const float*, const float*, long long,
                                  cudaStream_t);
template void vec_invert<double>(const double*, double*, long long, cudaStream_t);
template void vec_invert<float>(const double*, float*, long long, cudaStream_t);

}  // namespace sf
