// Vector kernels of the device conjugate-gradient solver.
//
// These replace the host BLAS-1 work of IterativeSolvers.cg! (called at
// profiling/drivers.jl:85-95). The CG scalars (alpha, beta, dot products)
// live in a small device array, so an iteration launches without a host
// round trip. Reductions are deterministic: every block stores its partial
// sums (FP64 for both vector types), and the block that finishes last adds
// all of them in block order, so the result does not depend on which block
// that is. Elementwise loops take kUnroll elements per thread per round and
// issue all their loads first, which keeps enough bytes in flight for FP32
// vectors too.
#include "sf_cg.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <utility>

namespace sf {
namespace {

constexpr int kThreads = 256;
constexpr int kUnroll = 4;

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

// Fixed-order sum of partials[b*NV + k] over b < nparts; totals in thread 0.
template <int NV>
__device__ __forceinline__ void sum_partials(const double* partials, long long nparts,
                                             double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
#pragma unroll 4
  for (long long b = threadIdx.x; b < nparts; b += kThreads) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += __ldcg(partials + b * NV + k);
  }
  block_sum<NV>(v);
}

// Each block stores its sums v; the last block to finish adds every block's
// sums and returns true (in all its threads) with the totals in v (thread 0).
// The counter is back at zero when the kernel ends.
template <int NV>
__device__ __forceinline__ bool last_block_sum(double (&v)[NV], double* partials,
                                               unsigned int* count) {
  __shared__ bool is_last;
  block_sum<NV>(v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) partials[blockIdx.x * NV + k] = v[k];
    __threadfence();
    is_last = atomicAdd(count, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!is_last) return false;
  __threadfence();
  sum_partials<NV>(partials, gridDim.x, v);
  if (threadIdx.x == 0) *count = 0u;
  return true;
}

__device__ __forceinline__ unsigned int* cg_counter(double* s) {
  return reinterpret_cast<unsigned int*>(s + CG_COUNTER);
}

// Publishes RR, DONE, ITERS and then the report number to mapped host memory.
__device__ __forceinline__ void publish(const double* s, double* report) {
  if (!report) return;
  report[0] = s[CG_RR];
  report[1] = s[CG_DONE];
  report[2] = s[CG_ITERS];
  __threadfence_system();
  report[3] = s[CG_REPORTS];
}

// out = sum of partials in a fixed order (nothing while *skip != 0)
template <int NV>
__global__ void k_finish(const double* __restrict__ partials, long long nparts,
                         double* __restrict__ out, const double* __restrict__ skip) {
  if (skip && *skip != 0.0) return;
  double v[NV];
  sum_partials<NV>(partials, nparts, v);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) out[k] = v[k];
  }
}

// *out = a . b
template <typename T>
__global__ void k_dot(const T* __restrict__ a, const T* __restrict__ b, long long n,
                      double* __restrict__ partials, double* __restrict__ out, double* s_count,
                      const double* __restrict__ skip) {
  if (skip && *skip != 0.0) return;
  const long long S = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  double v[1] = {0.0};
  for (; i + (kUnroll - 1) * S < n; i += kUnroll * S) {
    T av[kUnroll], bv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      av[u] = a[i + u * S];
      bv[u] = b[i + u * S];
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) v[0] += (double)av[u] * (double)bv[u];
  }
  for (; i < n; i += S) v[0] += (double)a[i] * (double)b[i];
  if (last_block_sum<1>(v, partials, cg_counter(s_count)) && threadIdx.x == 0) *out = v[0];
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

__global__ void k_cg_init(double* __restrict__ s, double reltol2) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  s[CG_RZ] = s[CG_RZ_NEW];
  s[CG_ITERS] = 0.0;
  s[CG_REPORTS] = 0.0;
  *cg_counter(s) = 0u;
  const double bb = s[CG_BB];
  s[CG_TOL2] = reltol2 < 0.0 ? -1.0 : reltol2 * (bb > 0.0 ? bb : 1.0);
  const double rr = s[CG_RR];
  s[CG_DONE] = isfinite(rr) ? (rr <= s[CG_TOL2] ? 2.0 : 0.0) : 3.0;
}

// alpha = RZ / PQ; r -= alpha q. Sums (r, dinv r) -> RZ_NEW, (r, r) -> RR; then
// DONE = 1 at convergence, 3 if a sum is not finite.
template <typename T>
__global__ void k_cg_update(double* __restrict__ s, T* __restrict__ r, const T* __restrict__ q,
                            const T* __restrict__ dinv, long long n,
                            double* __restrict__ partials, int distributed) {
  if (s[CG_DONE] != 0.0) return;
  const double pq = distributed ? s[CG_PART_PQ] : s[CG_PQ];
  const T alpha = (T)(s[CG_RZ] / pq);
  const long long S = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  double v[2] = {0.0, 0.0};
  for (; i + (kUnroll - 1) * S < n; i += kUnroll * S) {
    T qv[kUnroll], rv[kUnroll], dv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      qv[u] = q[i + u * S];
      rv[u] = r[i + u * S];
      dv[u] = dinv ? dinv[i + u * S] : T(1);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const T ri = fma(-alpha, qv[u], rv[u]);
      r[i + u * S] = ri;
      const T zi = dinv ? (T)(dv[u] * ri) : ri;
      v[0] += (double)ri * (double)zi;
      v[1] += (double)ri * (double)ri;
    }
  }
  for (; i < n; i += S) {
    const T ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    const T zi = dinv ? (T)(dinv[i] * ri) : ri;
    v[0] += (double)ri * (double)zi;
    v[1] += (double)ri * (double)ri;
  }
  if (last_block_sum<2>(v, partials, cg_counter(s)) && threadIdx.x == 0) {
    if (distributed) {
      s[CG_PQ] = pq;
      s[CG_PART_RZ] = v[0];
      s[CG_PART_RR] = v[1];
    } else {
      s[CG_RZ_NEW] = v[0];
      s[CG_RR] = v[1];
      if (!isfinite(v[1]) || !isfinite(v[0])) s[CG_DONE] = 3.0;
      else if (v[1] <= s[CG_TOL2]) s[CG_DONE] = 1.0;
    }
  }
}

// distributed CG: the summed (r, dinv r) and (r, r), and the stopping test
__global__ void k_cg_check(double* __restrict__ s) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || s[CG_DONE] != 0.0) return;
  const double rz = s[CG_PART_RZ], rr = s[CG_PART_RR];
  s[CG_RZ_NEW] = rz;
  s[CG_RR] = rr;
  if (!isfinite(rr) || !isfinite(rz)) s[CG_DONE] = 3.0;
  else if (rr <= s[CG_TOL2]) s[CG_DONE] = 1.0;
}

// x += alpha p; then p = dinv r + beta p unless this iteration converged. The
// last block ends the iteration: RZ = RZ_NEW, ITERS += 1, DONE 1 -> 2, and a
// report. A finished solve only reports.
template <typename T>
__global__ void k_cg_direction(double* __restrict__ s, T* __restrict__ x, T* __restrict__ p,
                               const T* __restrict__ r, const T* __restrict__ dinv, long long n,
                               double* __restrict__ report) {
  const double done = s[CG_DONE];
  if (done >= 2.0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      s[CG_REPORTS] += 1.0;
      publish(s, report);
    }
    return;
  }
  const T alpha = (T)(s[CG_RZ] / s[CG_PQ]);
  const T beta = (T)(s[CG_RZ_NEW] / s[CG_RZ]);
  const long long S = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (done == 0.0) {
    for (; i + (kUnroll - 1) * S < n; i += kUnroll * S) {
      T pv[kUnroll], xv[kUnroll], rv[kUnroll], dv[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        pv[u] = p[i + u * S];
        xv[u] = x[i + u * S];
        rv[u] = r[i + u * S];
        dv[u] = dinv ? dinv[i + u * S] : T(1);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        x[i + u * S] = fma(alpha, pv[u], xv[u]);
        const T zi = dinv ? (T)(dv[u] * rv[u]) : rv[u];
        p[i + u * S] = fma(beta, pv[u], zi);
      }
    }
    for (; i < n; i += S) {
      const T pi = p[i];
      x[i] = fma(alpha, pi, x[i]);
      const T zi = dinv ? (T)(dinv[i] * r[i]) : r[i];
      p[i] = fma(beta, pi, zi);
    }
  } else {
    for (; i < n; i += S) x[i] = fma(alpha, p[i], x[i]);
  }
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(cg_counter(s), 1u) == gridDim.x - 1;
    if (is_last) {
      *cg_counter(s) = 0u;
      s[CG_RZ] = s[CG_RZ_NEW];
      s[CG_ITERS] += 1.0;
      if (done == 1.0) s[CG_DONE] = 2.0;
      s[CG_REPORTS] += 1.0;
      publish(s, report);
    }
  }
}

// Free-grid position (x, y, z) of a flat index. A grid-stride loop advances it by the
// position of the stride with one carry per axis, so no division per element.
struct GridPos {
  int x, y, z;
  __device__ __forceinline__ void set(long long i, int nfx, int nfy) {
    x = (int)(i % nfx);
    const long long t = i / nfx;
    y = (int)(t % nfy);
    z = (int)(t / nfy);
  }
  __device__ __forceinline__ void add(const GridPos& d, int nfx, int nfy) {
    x += d.x;
    if (x >= nfx) {
      x -= nfx;
      ++y;
    }
    y += d.y;
    if (y >= nfy) {
      y -= nfy;
      ++z;
    }
    z += d.z;
  }
};

template <int P>
__device__ __forceinline__ double table_dinv(const JacobiTable& J, const GridPos& g) {
  return __ldg(J.tab + ((g.z + 1) % P) * P * P + ((g.y + 1) % P) * P + (g.x + 1) % P);
}

// k_cg_update (non-distributed) with D^-1 from the table.
template <typename T, int P>
__global__ void k_cg_update_table(double* __restrict__ s, T* __restrict__ r,
                                  const T* __restrict__ q, const JacobiTable J, long long n,
                                  double* __restrict__ partials) {
  if (s[CG_DONE] != 0.0) return;
  const T alpha = (T)(s[CG_RZ] / s[CG_PQ]);
  const long long S = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  GridPos g, st;
  g.set(i, J.nfx, J.nfy);
  st.set(S, J.nfx, J.nfy);
  double v[2] = {0.0, 0.0};
  for (; i + (kUnroll - 1) * S < n; i += kUnroll * S) {
    T qv[kUnroll], rv[kUnroll], dv[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      qv[u] = q[i + u * S];
      rv[u] = r[i + u * S];
      dv[u] = (T)table_dinv<P>(J, g);
      g.add(st, J.nfx, J.nfy);
    }
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) {
      const T ri = fma(-alpha, qv[u], rv[u]);
      r[i + u * S] = ri;
      const T zi = (T)(dv[u] * ri);
      v[0] += (double)ri * (double)zi;
      v[1] += (double)ri * (double)ri;
    }
  }
  for (; i < n; i += S) {
    const T ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    const T zi = (T)((T)table_dinv<P>(J, g) * ri);
    g.add(st, J.nfx, J.nfy);
    v[0] += (double)ri * (double)zi;
    v[1] += (double)ri * (double)ri;
  }
  if (last_block_sum<2>(v, partials, cg_counter(s)) && threadIdx.x == 0) {
    s[CG_RZ_NEW] = v[0];
    s[CG_RR] = v[1];
    if (!isfinite(v[1]) || !isfinite(v[0])) s[CG_DONE] = 3.0;
    else if (v[1] <= s[CG_TOL2]) s[CG_DONE] = 1.0;
  }
}

// k_cg_direction with D^-1 from the table.
template <typename T, int P>
__global__ void k_cg_direction_table(double* __restrict__ s, T* __restrict__ x,
                                     T* __restrict__ p, const T* __restrict__ r,
                                     const JacobiTable J, long long n,
                                     double* __restrict__ report) {
  const double done = s[CG_DONE];
  if (done >= 2.0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      s[CG_REPORTS] += 1.0;
      publish(s, report);
    }
    return;
  }
  const T alpha = (T)(s[CG_RZ] / s[CG_PQ]);
  const T beta = (T)(s[CG_RZ_NEW] / s[CG_RZ]);
  const long long S = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  if (done == 0.0) {
    GridPos g, st;
    g.set(i, J.nfx, J.nfy);
    st.set(S, J.nfx, J.nfy);
    for (; i + (kUnroll - 1) * S < n; i += kUnroll * S) {
      T pv[kUnroll], xv[kUnroll], rv[kUnroll], dv[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        pv[u] = p[i + u * S];
        xv[u] = x[i + u * S];
        rv[u] = r[i + u * S];
        dv[u] = (T)table_dinv<P>(J, g);
        g.add(st, J.nfx, J.nfy);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        x[i + u * S] = fma(alpha, pv[u], xv[u]);
        const T zi = (T)(dv[u] * rv[u]);
        p[i + u * S] = fma(beta, pv[u], zi);
      }
    }
    for (; i < n; i += S) {
      const T pi = p[i];
      x[i] = fma(alpha, pi, x[i]);
      const T zi = (T)((T)table_dinv<P>(J, g) * r[i]);
      g.add(st, J.nfx, J.nfy);
      p[i] = fma(beta, pi, zi);
    }
  } else {
    for (; i < n; i += S) x[i] = fma(alpha, p[i], x[i]);
  }
  __shared__ bool is_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    is_last = atomicAdd(cg_counter(s), 1u) == gridDim.x - 1;
    if (is_last) {
      *cg_counter(s) = 0u;
      s[CG_RZ] = s[CG_RZ_NEW];
      s[CG_ITERS] += 1.0;
      if (done == 1.0) s[CG_DONE] = 2.0;
      s[CG_REPORTS] += 1.0;
      publish(s, report);
    }
  }
}

// y[i] = x[idx[i]]: the index stream and y are coalesced, kUnroll entries per thread
// in flight.
template <typename T>
__global__ void k_permute(const T* __restrict__ x, const int32_t* __restrict__ idx,
                          T* __restrict__ y, long long n) {
  const long long S = (long long)gridDim.x * kThreads;
  long long i = (long long)blockIdx.x * kThreads + threadIdx.x;
  for (; i + (kUnroll - 1) * S < n; i += kUnroll * S) {
    int32_t k[kUnroll];
    T v[kUnroll];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) k[u] = idx[i + u * S];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) v[u] = x[k[u]];
#pragma unroll
    for (int u = 0; u < kUnroll; ++u) y[i + u * S] = v[u];
  }
  for (; i < n; i += S) y[i] = x[idx[i]];
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

// Blocks of `kernel` resident on the current device at once (cached per device and kernel).
int resident_blocks(const void* kernel) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> cache;
  int dev = 0;
  SF_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({dev, kernel});
  if (it != cache.end()) return it->second;
  int sms = 0, per_sm = 0;
  SF_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0));
  const int blocks = std::max(1, sms * std::max(1, per_sm));
  cache[{dev, kernel}] = blocks;
  return blocks;
}

// One wave of `kernel` (at most kRedBlocks blocks, the capacity of the partial sums).
template <typename K>
int grid_for(K kernel, long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  b = std::min<long long>(b, std::min(kRedBlocks, resident_blocks((const void*)kernel)));
  return (int)std::max(1LL, b);
}

}  // namespace

void dot_finish(const double* partials, long long nparts, double* out, const double* skip,
                cudaStream_t st) {
  k_finish<1><<<1, kThreads, 0, st>>>(partials, nparts, out, skip);
  SF_CUDA_CHECK(cudaGetLastError());
}

void cg_reset(double* s, cudaStream_t st) {
  SF_CUDA_CHECK(cudaMemsetAsync(s, 0, CG_NSLOTS * sizeof(double), st));
}

template <typename T>
void vec_dot(const T* a, const T* b, long long n, double* partials, double* out, double* s,
             const double* skip, cudaStream_t st) {
  k_dot<T><<<grid_for(k_dot<T>, n), kThreads, 0, st>>>(a, b, n, partials, out, s, skip);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_start(const T* b, const T* q, const T* dinv, T* r, T* p, long long n, double* partials,
              double* s, cudaStream_t st) {
  const int g = grid_for(k_cg_start<T>, n);
  k_cg_start<T><<<g, kThreads, 0, st>>>(b, q, dinv, r, p, n, partials);
  k_finish<3><<<1, kThreads, 0, st>>>(partials, g, s + CG_RZ_NEW, nullptr);  // RZ_NEW, RR, BB
  SF_CUDA_CHECK(cudaGetLastError());
}

void cg_init(double* s, double reltol2, cudaStream_t st) {
  k_cg_init<<<1, 32, 0, st>>>(s, reltol2);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_update(double* s, T* r, const T* q, const T* dinv, long long n, double* partials,
               cudaStream_t st, bool distributed) {
  k_cg_update<T><<<grid_for(k_cg_update<T>, n), kThreads, 0, st>>>(s, r, q, dinv, n, partials,
                                                                   distributed ? 1 : 0);
  SF_CUDA_CHECK(cudaGetLastError());
}

void cg_check(double* s, cudaStream_t st) {
  k_cg_check<<<1, 32, 0, st>>>(s);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_direction(double* s, T* x, T* p, const T* r, const T* dinv, long long n, double* report,
                  cudaStream_t st) {
  k_cg_direction<T><<<grid_for(k_cg_direction<T>, n), kThreads, 0, st>>>(s, x, p, r, dinv, n, report);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void vec_invert(const double* d, T* dinv, long long n, cudaStream_t st) {
  k_invert<T><<<grid_for(k_invert<T>, n), kThreads, 0, st>>>(d, dinv, n);
  SF_CUDA_CHECK(cudaGetLastError());
}

void mixed_residual(const double* b, const double* q, const float* dinv, float* r32, float* xs32,
                    float* p32, bool set_p, long long n, double* partials, double* s,
                    cudaStream_t st) {
  const int g = grid_for(k_mixed_residual, n);
  k_mixed_residual<<<g, kThreads, 0, st>>>(b, q, dinv, r32, xs32, p32, set_p ? 1 : 0, n, partials);
  k_finish<2><<<1, kThreads, 0, st>>>(partials, g, s + CG_RZ_NEW, nullptr);  // RZ_NEW, RR (FP64)
  SF_CUDA_CHECK(cudaGetLastError());
}

void mixed_fold(double* x, const float* xs32, long long n, cudaStream_t st) {
  k_fold<<<grid_for(k_fold, n), kThreads, 0, st>>>(x, xs32, n);
  SF_CUDA_CHECK(cudaGetLastError());
}

void copy_scalar(double* s, int dst, int src, cudaStream_t st) {
  k_copy_scalar<<<1, 32, 0, st>>>(s, dst, src);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_update_table(double* s, T* r, const T* q, const JacobiTable& J, long long n,
                     double* partials, cudaStream_t st) {
  switch (J.p) {
#define SF_CASE(P_)                                                                            \
  case P_:                                                                                     \
    k_cg_update_table<T, P_><<<grid_for(k_cg_update_table<T, P_>, n), kThreads, 0, st>>>(    \
        s, r, q, J, n, partials);                                                              \
    break;
    SF_CASE(1) SF_CASE(2) SF_CASE(3) SF_CASE(4) SF_CASE(5) SF_CASE(6) SF_CASE(7) SF_CASE(8)
#undef SF_CASE
    default: throw Error(SF_ERR_UNSUPPORTED, "no Jacobi table for this order");
  }
  SF_CUDA_CHECK(cudaGetLastError());
}

template <typename T>
void cg_direction_table(double* s, T* x, T* p, const T* r, const JacobiTable& J, long long n,
                        double* report, cudaStream_t st) {
  switch (J.p) {
#define SF_CASE(P_)                                                                            \
  case P_:                                                                                     \
    k_cg_direction_table<T, P_><<<grid_for(k_cg_direction_table<T, P_>, n), kThreads, 0,     \
                                  st>>>(s, x, p, r, J, n, report);                             \
    break;
    SF_CASE(1) SF_CASE(2) SF_CASE(3) SF_CASE(4) SF_CASE(5) SF_CASE(6) SF_CASE(7) SF_CASE(8)
#undef SF_CASE
    default: throw Error(SF_ERR_UNSUPPORTED, "no Jacobi table for this order");
  }
  SF_CUDA_CHECK(cudaGetLastError());
}

void permute_gather(int dtype, const void* x, const int32_t* idx, void* y, long long n,
                    cudaStream_t st) {
  if (n <= 0) return;
  if (dtype == SF_F64) {
    k_permute<double><<<grid_for(k_permute<double>, n), kThreads, 0, st>>>(
        static_cast<const double*>(x), idx, static_cast<double*>(y), n);
  } else if (dtype == SF_F32) {
    k_permute<float><<<grid_for(k_permute<float>, n), kThreads, 0, st>>>(
        static_cast<const float*>(x), idx, static_cast<float*>(y), n);
  } else {
    throw Error(SF_ERR_ARG, "dtype must be SF_F64 or SF_F32");
  }
  SF_CUDA_CHECK(cudaGetLastError());
}


#define SF_INST(T)                                                                            \
  template void vec_dot<T>(const T*, const T*, long long, double*, double*, double*,            \
                           const double*, cudaStream_t);                                        \
  template void cg_start<T>(const T*, const T*, const T*, T*, T*, long long, double*, double*,  \
                            cudaStream_t);                                                      \
  template void cg_update<T>(double*, T*, const T*, const T*, long long, double*, cudaStream_t,  \
                             bool);                                                             \
  template void cg_direction<T>(double*, T*, T*, const T*, const T*, long long, double*,        \
                                cudaStream_t);                                                  \
  template void vec_invert<T>(const double*, T*, long long, cudaStream_t);                   \
  template void cg_update_table<T>(double*, T*, const T*, const JacobiTable&, long long,       \
                                   double*, cudaStream_t);                                      \
  template void cg_direction_table<T>(double*, T*, T*, const T*, const JacobiTable&, long long, \
                                      double*, cudaStream_t);
SF_INST(double)
SF_INST(float)
#undef SF_INST

}  // namespace sf
