// Multigrid-preconditioned flexible CG on structured meshes (sf_mg_*).
//
// The reference solves with IterativeSolvers.cg! and no preconditioner
// (profiling/drivers.jl:85-95). The iteration count of that CG grows like the
// square root of the condition number: about 2400 Jacobi-preconditioned
// iterations for a rough right-hand side at Q4 on 64^3 cells, and more than
// 9000 already on 3^3 cells for equispaced Q8 on perturbed cells. This solver
// keeps the FP64 CG on the caller's operator and preconditions it with one
// V-cycle per iteration:
//
//   levels    the caller's structured operators, finest first: lower orders on
//             the same cells (p-coarsening) and then coarser meshes (h-coarsening);
//   transfers prolongation P from level l+1 to level l is the interpolation of
//             the coarse space into the fine one. On a structured grid it is the
//             tensor product of one 1D matrix along each axis, so it runs as three
//             1D passes; the restriction is P^T, the same passes transposed;
//   smoother  Chebyshev polynomial of D^-1 A (D the diagonal) of a fixed degree
//             over [lmax / ratio, 1.1 lmax], with lmax estimated by power
//             iteration at set-up; the coarsest level gets a longer Chebyshev run;
//   basis     optionally, the hierarchy works in another nodal basis of the
//             finest space (Gauss-Lobatto nodes, for equispaced high order): with
//             T the change of basis (values at the caller's nodes of the
//             hierarchy's basis functions, again a tensor product of a 1D matrix),
//             the caller's operator is A = T^-T A_h T^-1 and the preconditioner is
//             T V(T^T r);
//   outer     flexible CG, FCG(1): z = M r, p = z - ((z, q_old) / (p, q_old)) p,
//             q = A p, alpha = (p, r) / (p, q). The flexible form tolerates a
//             preconditioner that is not exactly linear, e.g. one run in FP32.
//
// In the mixed mode the whole V-cycle (level applies, smoothing, transfers)
// runs in FP32 and the outer CG (the caller's FP64 apply, the residual, the
// dot products and x) stays in FP64; the reached residual is the FP64 one.
// One outer iteration is captured once in a CUDA graph and replayed; all CG
// scalars stay on the device and the host reads the convergence flag after every
// iteration. The reductions are deterministic (fixed-order sums).
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "sf_internal.cuh"

namespace sf {
namespace {

constexpr int kT = 256;
constexpr int kMgBlocks = 148 * 8;   // reduction grid: the partial-sum capacity
constexpr int kMaxW = 256;           // 1D transfer table entries
// Iterations replayed between reads of the convergence flag. An iteration takes milliseconds
// and a read microseconds; with 4, a deformed Q8 32^3 solve of 18 iterations ran 20.
constexpr int kChunk = 1;

// Scalar slots of the outer FCG.
// S_COUNTER is slot 9, where op_apply_dot's reductions keep their block counter.
enum MgSlot {
  S_ZQ = 0, S_PR, S_PQ, S_RR, S_BB, S_TOL2, S_DONE, S_ITERS, S_FIRST, S_COUNTER, S_NSLOTS = 16
};
static_assert(S_COUNTER == 9, "the reduction counter slot of op_apply_dot");

// ---------------------------------------------------------------------------
// 1D transfer pass along one axis of a structured free-point grid, cell by cell.
// Prolongation from level l+1 to level l: the coarse grid has ncc cells of pc
// points along the axis, the fine grid ncc cells of F points (F = r pf: r fine
// cells of order pf per coarse cell); W[l][m] ((F+1) x (pc+1), row-major) is the
// coarse cell's basis function m at its fine node l. Fine point g = c F + l
// (l < F, grid index 1 .. ncc F - 1) takes cell c's value
//     out[g] = sum_m W[l][m] in[c pc + m]      (coarse points 1 .. ncc pc - 1),
// and the restriction is the exact transpose: coarse point c pc + m (0 < m < pc)
// sums W[l][m] in[c F + l] over cell c's fine points, and the vertex (c+1) pc
// sums column pc over cell c and column 0 over cell c+1.
// A thread takes one coarse cell of one grid line, so it loads each input of the
// cell once; W is read from the kernel parameters (the same entry across a warp).
// ---------------------------------------------------------------------------
constexpr int kMaxPc = 8;     // coarse order (pc + 1 values per cell in registers)
constexpr int kCellRows = 4;  // blocks of 32 x 4 threads

template <typename T>
struct CellPassParams {
  T W[kMaxW];              // (F + 1) x (pc + 1), row-major
  int F, pc, ncc;          // fine points per coarse cell, coarse order, cells along the axis
  int n0, n1, n2;          // output grid (x fastest); the third index <= 65535
  int n_in;                // input points along the axis
  int axis;                // 0 x, 1 y, 2 z
  int transpose, accumulate, subtract;  // restriction; out += ; in - in2
};

// One coarse cell c of a line: ld(k) reads input point k (free index along the
// axis), emit(k, v) writes output point k. Every output point of the line is
// emitted by exactly one cell.
template <typename T, typename Load, typename Emit>
__device__ __forceinline__ void cell_pass(const CellPassParams<T>& Q, int c, const Load& ld,
                                          const Emit& emit) {
  const int pc = Q.pc, F = Q.F, ncc = Q.ncc;
  if (!Q.transpose) {
    T u[kMaxPc + 1];
#pragma unroll
    for (int m = 0; m <= kMaxPc; ++m) {
      const int j = c * pc + m;  // coarse grid point (0 and ncc pc are boundary points)
      u[m] = (m <= pc && j > 0 && j < ncc * pc) ? ld(j - 1) : T(0);
    }
    for (int l = 0; l < F; ++l) {
      const int g = c * F + l;
      if (g == 0) continue;
      const T* w = Q.W + l * (pc + 1);
      T acc = T(0);
#pragma unroll
      for (int m = 0; m <= kMaxPc; ++m)
        if (m <= pc) acc = fma(w[m], u[m], acc);
      emit(g - 1, acc);
    }
  } else {
    T acc[kMaxPc + 1];
#pragma unroll
    for (int m = 0; m <= kMaxPc; ++m) acc[m] = T(0);
    for (int l = 0; l < F; ++l) {
      const int g = c * F + l;
      const T v = g > 0 ? ld(g - 1) : T(0);
      const T* w = Q.W + l * (pc + 1);
#pragma unroll
      for (int m = 1; m <= kMaxPc; ++m)
        if (m <= pc) acc[m] = fma(w[m], v, acc[m]);
    }
    T vtx = T(0);  // the right vertex's part from cell c + 1 (column 0)
    if (c + 1 < ncc)
      for (int l = 0; l < F; ++l) vtx = fma(Q.W[l * (pc + 1)], ld((c + 1) * F + l - 1), vtx);
#pragma unroll
    for (int m = 1; m <= kMaxPc; ++m) {
      const int j = c * pc + m;
      if (m <= pc && j < ncc * pc) emit(j - 1, m == pc ? acc[m] + vtx : acc[m]);
    }
  }
}

// Passes along y (axis 1) or z (axis 2): thread (x, cell, third index); the loads
// and stores of a warp are consecutive along x.
template <typename T>
__global__ void k_cellpass(const __grid_constant__ CellPassParams<T> Q, const T* __restrict__ in,
                           const T* __restrict__ in2, T* __restrict__ out) {
  const int i0 = blockIdx.x * 32 + threadIdx.x;
  const int c = blockIdx.y * kCellRows + threadIdx.y;
  const int io = blockIdx.z;  // z for a pass along y, y for a pass along z
  if (i0 >= Q.n0 || c >= Q.ncc) return;
  long long ib, ob, stride;
  if (Q.axis == 1) {
    stride = Q.n0;
    ib = i0 + (long long)Q.n0 * Q.n_in * io;
    ob = i0 + (long long)Q.n0 * Q.n1 * io;
  } else {
    stride = (long long)Q.n0 * Q.n1;
    ib = ob = i0 + (long long)Q.n0 * io;
  }
  cell_pass<T>(
      Q, c,
      [&](int k) {
        const long long o = ib + k * stride;
        return Q.subtract ? in[o] - in2[o] : in[o];
      },
      [&](int k, T v) {
        const long long o = ob + k * stride;
        out[o] = Q.accumulate ? out[o] + v : v;
      });
}

// The pass along x: a warp per grid row stages the row's inputs (in - in2) in
// shared memory with coalesced loads, assembles the output row there cell by
// cell, and stores it coalesced.
template <typename T>
__global__ void k_cellpass_x(const __grid_constant__ CellPassParams<T> Q,
                             const T* __restrict__ in, const T* __restrict__ in2,
                             T* __restrict__ out) {
  extern __shared__ __align__(16) unsigned char cp_smem[];
  T* srow = reinterpret_cast<T*>(cp_smem) + threadIdx.y * (Q.n_in + Q.n0);
  T* sout = srow + Q.n_in;
  const int i1 = blockIdx.y * kCellRows + threadIdx.y, i2 = blockIdx.z;
  if (i1 >= Q.n1) return;  // the whole warp
  const long long ib = (long long)Q.n_in * (i1 + (long long)Q.n1 * i2);
  const long long ob = (long long)Q.n0 * (i1 + (long long)Q.n1 * i2);
  for (int k = threadIdx.x; k < Q.n_in; k += 32)
    srow[k] = Q.subtract ? in[ib + k] - in2[ib + k] : in[ib + k];
  __syncwarp();
  for (int c = threadIdx.x; c < Q.ncc; c += 32)
    cell_pass<T>(Q, c, [&](int k) { return srow[k]; }, [&](int k, T v) { sout[k] = v; });
  __syncwarp();
  for (int k = threadIdx.x; k < Q.n0; k += 32)
    out[ob + k] = Q.accumulate ? out[ob + k] + sout[k] : sout[k];
}

// ---------------------------------------------------------------------------
// Chebyshev smoothing steps (first kind) of D^-1 A:
//   mode 0: d = c2 dinv r,              z = d           (start from z = 0)
//   mode 1: d = c2 dinv (r - az),       z += d          (start from a given z)
//   mode 2: d = c1 d + c2 dinv (r - az), z += d         (later steps)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_cheb(int mode, long long n, const T* __restrict__ r, const T* __restrict__ az,
                       const T* __restrict__ dinv, T* __restrict__ z, T* __restrict__ d, T c1,
                       T c2) {
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT) {
    const T res = mode == 0 ? r[i] : r[i] - az[i];
    T dv = c2 * dinv[i] * res;
    if (mode == 2) dv = fma(c1, d[i], dv);
    d[i] = dv;
    z[i] = mode == 0 ? dv : z[i] + dv;
  }
}

template <typename T>
__global__ void k_invert(const double* __restrict__ d, T* __restrict__ dinv, long long n) {
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT)
    dinv[i] = (T)(d[i] != 0.0 ? 1.0 / d[i] : 0.0);
}

template <typename TO, typename TI>
__global__ void k_convert(const TI* __restrict__ a, TO* __restrict__ b, long long n) {
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT)
    b[i] = (TO)a[i];
}

// ---------------------------------------------------------------------------
// Deterministic reductions: each block stores its partial sums, and the last
// block to finish adds all of them in block order.
// ---------------------------------------------------------------------------
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
  __shared__ double sh[NV][kT / 32];
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
      for (int w = 0; w < kT / 32; ++w) s += sh[k][w];
      v[k] = s;
    }
  }
  __syncthreads();
}

// True in every thread of the last block to finish; the totals are then in v
// (thread 0). The counter (in the scalar array) is back at zero afterwards.
template <int NV>
__device__ __forceinline__ bool last_block(double (&v)[NV], double* partials, double* s) {
  __shared__ bool is_last;
  unsigned int* count = reinterpret_cast<unsigned int*>(s + S_COUNTER);
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
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (long long b = threadIdx.x; b < gridDim.x; b += kT) {
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += __ldcg(partials + b * NV + k);
  }
  block_sum<NV>(v);
  if (threadIdx.x == 0) *count = 0u;
  return true;
}

// r = b - q (q = A x0), rl = r in the hierarchy's type; (r, r), (b, b); the
// stopping threshold and the flag.
template <typename TL>
__global__ void k_fcg_start(const double* __restrict__ b, const double* __restrict__ q,
                            double* __restrict__ r, TL* __restrict__ rl, long long n,
                            double reltol2, double* __restrict__ partials,
                            double* __restrict__ s) {
  double v[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT) {
    const double bi = b[i], ri = bi - q[i];
    r[i] = ri;
    rl[i] = (TL)ri;
    v[0] = fma(ri, ri, v[0]);
    v[1] = fma(bi, bi, v[1]);
  }
  if (last_block<2>(v, partials, s) && threadIdx.x == 0) {
    s[S_RR] = v[0];
    s[S_BB] = v[1];
    s[S_TOL2] = reltol2 * (v[1] > 0.0 ? v[1] : 1.0);
    s[S_ITERS] = 0.0;
    s[S_FIRST] = 1.0;
    s[S_DONE] = !isfinite(v[0]) ? 3.0 : (v[0] <= s[S_TOL2] ? 2.0 : 0.0);
  }
}

// (z, q_old): nothing on the first iteration or once done.
template <typename TZ>
__global__ void k_fcg_zq(const TZ* __restrict__ z, const double* __restrict__ q, long long n,
                         double* __restrict__ partials, double* __restrict__ s) {
  if (s[S_DONE] != 0.0 || s[S_FIRST] != 0.0) return;
  double v[1] = {0.0};
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT)
    v[0] = fma((double)z[i], q[i], v[0]);
  if (last_block<1>(v, partials, s) && threadIdx.x == 0) s[S_ZQ] = v[0];
}

// p = z - beta p (beta = (z, q_old) / (p_old, q_old), 0 first); (p, r).
template <typename TZ>
__global__ void k_fcg_dir(const TZ* __restrict__ z, double* __restrict__ p,
                          const double* __restrict__ r, long long n,
                          double* __restrict__ partials, double* __restrict__ s) {
  if (s[S_DONE] != 0.0) return;
  const double beta = s[S_FIRST] != 0.0 ? 0.0 : s[S_ZQ] / s[S_PQ];
  double v[1] = {0.0};
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT) {
    const double pi = beta != 0.0 ? fma(-beta, p[i], (double)z[i]) : (double)z[i];
    p[i] = pi;
    v[0] = fma(pi, r[i], v[0]);
  }
  if (last_block<1>(v, partials, s) && threadIdx.x == 0) s[S_PR] = v[0];
}

// alpha = (p, r) / (p, q); x += alpha p; r -= alpha q; rl = r; (r, r) and the test.
template <typename TL>
__global__ void k_fcg_update(double* __restrict__ x, double* __restrict__ r,
                             const double* __restrict__ p, const double* __restrict__ q,
                             TL* __restrict__ rl, long long n, double* __restrict__ partials,
                             double* __restrict__ s) {
  if (s[S_DONE] != 0.0) return;
  const double alpha = s[S_PR] / s[S_PQ];
  double v[1] = {0.0};
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT) {
    x[i] = fma(alpha, p[i], x[i]);
    const double ri = fma(-alpha, q[i], r[i]);
    r[i] = ri;
    rl[i] = (TL)ri;
    v[0] = fma(ri, ri, v[0]);
  }
  if (last_block<1>(v, partials, s) && threadIdx.x == 0) {
    s[S_RR] = v[0];
    s[S_ITERS] += 1.0;
    s[S_FIRST] = 0.0;
    if (!isfinite(v[0]) || !isfinite(alpha)) s[S_DONE] = 3.0;
    else if (v[0] <= s[S_TOL2]) s[S_DONE] = 2.0;
  }
}

// Power iteration step of D^-1 A: w = dinv (A v) is given; (w, w) and (v, v).
__global__ void k_pow_norms(const double* __restrict__ w, const double* __restrict__ v,
                            long long n, double* __restrict__ partials, double* __restrict__ s,
                            double* __restrict__ out) {
  double a[2] = {0.0, 0.0};
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT) {
    a[0] = fma(w[i], w[i], a[0]);
    a[1] = fma(v[i], v[i], a[1]);
  }
  if (last_block<2>(a, partials, s) && threadIdx.x == 0) {
    out[0] = a[0];
    out[1] = a[1];
  }
}

// v = dinv (A v) / |dinv A v| (the input w = A v); a deterministic start vector when init.
__global__ void k_pow_next(double* __restrict__ v, const double* __restrict__ av,
                           const double* __restrict__ dinv, long long n, const double* norms,
                           int init) {
  const double sc = init ? 1.0 : 1.0 / sqrt(norms[0] > 0.0 ? norms[0] : 1.0);
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT) {
    if (init) {  // a fixed pseudo-random vector in [-1, 1]
      unsigned long long h = (unsigned long long)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
      h ^= h >> 31;
      h *= 0xBF58476D1CE4E5B9ull;
      h ^= h >> 27;
      v[i] = (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    } else {
      v[i] = sc * dinv[i] * av[i];
    }
  }
}

__global__ void k_dinv_apply(double* __restrict__ w, const double* __restrict__ av,
                             const double* __restrict__ dinv, long long n) {
  for (long long i = (long long)blockIdx.x * kT + threadIdx.x; i < n;
       i += (long long)gridDim.x * kT)
    w[i] = dinv[i] * av[i];
}

int grid_of(long long n) {
  return (int)std::max(1LL, std::min<long long>((n + kT - 1) / kT, kMgBlocks));
}


}  // namespace
}  // namespace sf

// ---------------------------------------------------------------------------
// The hierarchy.
// ---------------------------------------------------------------------------
struct sf_mg {
  struct Level {
    sf_op* op = nullptr;
    int nx = 0, ny = 0, nz = 0, p = 0;
    long long n = 0;
    double lmax = 0.0;
    double* dinv64 = nullptr;  // FP64 D^-1 (set-up)
    void* dinv = nullptr;      // D^-1 in the cycle's type
    void* r = nullptr;         // input (the restricted residual below level 0)
    void* zb[2] = {nullptr, nullptr};  // output (two buffers: a fused Chebyshev step
    int cur = 0;                        // writes z + d into the other one); zb[cur] is current
    void* z() const { return zb[cur]; }
    void* d = nullptr;         // Chebyshev direction
    void* t = nullptr;         // A z
  };
  // transfer between level l (fine) and l + 1 (coarse): per-axis 1D table
  struct Transfer {
    int r = 1, F = 0, pc = 0;
    std::vector<double> W;  // (F + 1) x (pc + 1)
  };
  sf_op* A = nullptr;  // the caller's operator (the outer FP64 CG)
  long long n = 0;
  std::vector<Level> lv;
  std::vector<Transfer> tr;
  bool has_basis = false;
  Transfer basis;  // change of basis at level 0 (F = pc = p)
  // Chebyshev degree and range: measured best together on Q4 64^3 (Cartesian, equispaced)
  // and deformed Q8 32^3 (Gauss-Lobatto); with ratio 30 the Q8 solve took twice the iterations.
  int degree = 4;
  double ratio = 20.0;
  int coarse_steps = 10;
  double coarse_ratio = 100.0;
  int dtype = -1;  // type of the allocated cycle buffers
  bool ready = false;
  // cycle buffers: transfer temporaries, level-0 input/output in the caller's basis
  void* tmp1 = nullptr;
  void* tmp2 = nullptr;
  size_t tmp_bytes = 0;
  void* rl = nullptr;  // the residual in the cycle's type (caller's basis)
  void* zl = nullptr;  // the preconditioned residual (caller's basis)
  // outer FP64 CG vectors and scalars
  double *x = nullptr, *r = nullptr, *p = nullptr, *q = nullptr;
  double* s = nullptr;
  double* partials = nullptr;
  long long partials_n = 0;  // entries of partials
  // power-iteration work vectors (largest level) and the two norms
  double *pw_v = nullptr, *pw_w = nullptr, *pw_av = nullptr, *pw_norms = nullptr;
  double* h_s = nullptr;  // pinned copy of the scalars
  cudaStream_t cs = nullptr;  // the solver's own stream (graph capture and replay)
  cudaEvent_t ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_dtype = -1;
  bool use_graph = true;  // false: capture failed, the iteration is launched kernel by kernel
  std::vector<void*> owned;  // device allocations
  std::string err;
};

namespace {

using sf::Error;

void* mg_alloc(sf_mg* mg, size_t bytes) {
  void* p = nullptr;
  SF_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
  mg->owned.push_back(p);
  return p;
}

void mg_release(sf_mg* mg) {
  if (mg->exec) cudaGraphExecDestroy(mg->exec);
  if (mg->graph) cudaGraphDestroy(mg->graph);
  mg->exec = nullptr;
  mg->graph = nullptr;
  for (void* p : mg->owned) cudaFree(p);
  mg->owned.clear();
  if (mg->h_s) cudaFreeHost(mg->h_s);
  mg->h_s = nullptr;
  if (mg->ev_in) cudaEventDestroy(mg->ev_in);
  if (mg->ev_out) cudaEventDestroy(mg->ev_out);
  if (mg->cs) cudaStreamDestroy(mg->cs);
  mg->ev_in = mg->ev_out = nullptr;
  mg->cs = nullptr;
}

template <typename F>
int mg_guarded(sf_mg* mg, F&& f) {
  try {
    f();
    if (mg) mg->err.clear();
    return SF_OK;
  } catch (const Error& e) {
    if (mg) mg->err = e.what();
    return e.status;
  } catch (const std::exception& e) {
    if (mg) mg->err = e.what();
    return SF_ERR_ARG;
  }
}

size_t esize(int dtype) { return dtype == SF_F64 ? 8 : 4; }

// One 1D pass of transfer t along `axis` (ncc coarse cells along it). out dims
// (n0, n1, n2); the input has n_in points along the axis.
template <typename T>
void pass(const sf_mg::Transfer& t, int axis, bool transpose, long long n0, long long n1,
          long long n2, int n_in, int ncc, const T* in, const T* in2, T* out, bool acc,
          cudaStream_t st) {
  if (n0 <= 0 || n1 <= 0 || n2 <= 0) return;
  sf::CellPassParams<T> Q{};
  for (size_t i = 0; i < t.W.size(); ++i) Q.W[i] = (T)t.W[i];
  Q.F = t.F;
  Q.pc = t.pc;
  Q.ncc = ncc;
  Q.n0 = (int)n0;
  Q.n1 = (int)n1;
  Q.n2 = (int)n2;
  Q.axis = axis;
  Q.n_in = n_in;
  Q.transpose = transpose ? 1 : 0;
  Q.accumulate = acc ? 1 : 0;
  Q.subtract = in2 ? 1 : 0;
  const dim3 block(32, sf::kCellRows);
  if (axis == 0) {  // rows staged in shared memory: kCellRows x (n_in + n0) values
    SF_REQUIRE(n_in <= 767 && n0 <= 767 && n2 <= 65535, SF_ERR_UNSUPPORTED,
               "multigrid transfer: at most 767 free points per grid row");
    const size_t smem = (size_t)sf::kCellRows * (n_in + n0) * sizeof(T);
    sf::k_cellpass_x<T><<<dim3(1, (unsigned)((n1 + sf::kCellRows - 1) / sf::kCellRows),
                               (unsigned)n2),
                          block, smem, st>>>(Q, in, in2, out);
  } else {
    const long long third = axis == 1 ? n2 : n1;
    SF_REQUIRE(third <= 65535, SF_ERR_UNSUPPORTED, "multigrid transfer: grid too large");
    sf::k_cellpass<T><<<dim3((unsigned)((n0 + 31) / 32),
                             (unsigned)((ncc + sf::kCellRows - 1) / sf::kCellRows),
                             (unsigned)third),
                        block, 0, st>>>(Q, in, in2, out);
  }
  SF_CUDA_CHECK(cudaGetLastError());
}

// out (fine grid, fx x fy x fz free points) (+)= P in (coarse grid cx x cy x cz);
// ncc: coarse cells per axis.
template <typename T>
void prolong(sf_mg* mg, const sf_mg::Transfer& t, const int ncc[3], const T* in, T* out, bool acc,
             cudaStream_t st) {
  const long long c[3] = {(long long)ncc[0] * t.pc - 1, (long long)ncc[1] * t.pc - 1,
                          (long long)ncc[2] * t.pc - 1};
  const long long f[3] = {(long long)ncc[0] * t.F - 1, (long long)ncc[1] * t.F - 1,
                          (long long)ncc[2] * t.F - 1};
  T* a = static_cast<T*>(mg->tmp1);
  T* b = static_cast<T*>(mg->tmp2);
  pass<T>(t, 2, false, c[0], c[1], f[2], (int)c[2], ncc[2], in, nullptr, a, false, st);
  pass<T>(t, 1, false, c[0], f[1], f[2], (int)c[1], ncc[1], a, nullptr, b, false, st);
  pass<T>(t, 0, false, f[0], f[1], f[2], (int)c[0], ncc[0], b, nullptr, out, acc, st);
}

// out (coarse) = P^T (in - in2) (fine); in2 may be null.
template <typename T>
void restrict_(sf_mg* mg, const sf_mg::Transfer& t, const int ncc[3], const T* in, const T* in2,
               T* out, cudaStream_t st) {
  const long long c[3] = {(long long)ncc[0] * t.pc - 1, (long long)ncc[1] * t.pc - 1,
                          (long long)ncc[2] * t.pc - 1};
  const long long f[3] = {(long long)ncc[0] * t.F - 1, (long long)ncc[1] * t.F - 1,
                          (long long)ncc[2] * t.F - 1};
  T* a = static_cast<T*>(mg->tmp1);
  T* b = static_cast<T*>(mg->tmp2);
  pass<T>(t, 0, true, c[0], f[1], f[2], (int)f[0], ncc[0], in, in2, a, false, st);
  pass<T>(t, 1, true, c[0], c[1], f[2], (int)f[1], ncc[1], a, nullptr, b, false, st);
  pass<T>(t, 2, true, c[0], c[1], c[2], (int)f[2], ncc[2], b, nullptr, out, false, st);
}

template <typename T>
void cheb_step(int mode, const sf_mg::Level& L, T c1, T c2, cudaStream_t st) {
  sf::k_cheb<T><<<sf::grid_of(L.n), sf::kT, 0, st>>>(
      mode, L.n, static_cast<const T*>(L.r), static_cast<const T*>(L.t),
      static_cast<const T*>(L.dinv), static_cast<T*>(L.z()), static_cast<T*>(L.d), c1, c2);
  SF_CUDA_CHECK(cudaGetLastError());
}

// One Chebyshev step after z = zb[cur] (mode 1 or 2): on an FP32 tiled level, fused
// into the apply's store phase, which writes z + d into the other buffer; otherwise
// an apply into t and the step kernel.
template <typename T>
void cheb_apply_step(sf_mg::Level& L, int dt, int mode, double c1, double c2, cudaStream_t st) {
  if constexpr (sizeof(T) == 4) {
    if (sf::op_cheb_apply(L.op, static_cast<const float*>(L.z()), static_cast<const float*>(L.r),
                          static_cast<const float*>(L.dinv), static_cast<float*>(L.d),
                          static_cast<float*>(L.zb[L.cur ^ 1]), c1, c2, mode, st)) {
      L.cur ^= 1;
      return;
    }
  }
  sf::op_apply(L.op, dt, L.z(), L.t, st);
  cheb_step<T>(mode, L, T(c1), T(c2), st);
}

// `deg` Chebyshev steps on level L over [lmax / ratio, 1.1 lmax]; zero_start: z = 0 first.
template <typename T>
void smooth(sf_mg::Level& L, int dt, int deg, double ratio, bool zero_start, cudaStream_t st) {
  const double b = 1.1 * L.lmax, a = b / (1.1 * ratio);
  const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
  double rho = 1.0 / sigma;
  if (zero_start) cheb_step<T>(0, L, T(0), T(1.0 / theta), st);
  else cheb_apply_step<T>(L, dt, 1, 0.0, 1.0 / theta, st);
  for (int k = 1; k < deg; ++k) {
    const double rho_n = 1.0 / (2.0 * sigma - rho);
    cheb_apply_step<T>(L, dt, 2, rho_n * rho, 2.0 * rho_n / delta, st);
    rho = rho_n;
  }
}

template <typename T>
void vcycle(sf_mg* mg, int l, int dt, cudaStream_t st) {
  sf_mg::Level& L = mg->lv[l];
  if (l + 1 == (int)mg->lv.size()) {
    smooth<T>(L, dt, mg->coarse_steps, mg->coarse_ratio, true, st);
    return;
  }
  smooth<T>(L, dt, mg->degree, mg->ratio, true, st);
  sf::op_apply(L.op, dt, L.z(), L.t, st);
  sf_mg::Level& C = mg->lv[l + 1];
  const int ncc[3] = {C.nx, C.ny, C.nz};
  restrict_<T>(mg, mg->tr[l], ncc, static_cast<const T*>(L.r), static_cast<const T*>(L.t),
               static_cast<T*>(C.r), st);
  vcycle<T>(mg, l + 1, dt, st);
  prolong<T>(mg, mg->tr[l], ncc, static_cast<const T*>(C.z()), static_cast<T*>(L.z()), true, st);
  smooth<T>(L, dt, mg->degree, mg->ratio, false, st);
}

// zl = M rl in the caller's basis.
template <typename T>
void precondition(sf_mg* mg, int dt, cudaStream_t st) {
  sf_mg::Level& L0 = mg->lv[0];
  const int ncc[3] = {L0.nx, L0.ny, L0.nz};
  if (mg->has_basis) {  // r_h = T^T r, z = T z_h
    restrict_<T>(mg, mg->basis, ncc, static_cast<const T*>(mg->rl), nullptr,
                 static_cast<T*>(L0.r), st);
    vcycle<T>(mg, 0, dt, st);
    prolong<T>(mg, mg->basis, ncc, static_cast<const T*>(L0.z()), static_cast<T*>(mg->zl), false,
               st);
  } else {
    vcycle<T>(mg, 0, dt, st);
  }
}

// D^-1 in the cycle's type from the FP64 set-up copy.
void cycle_dinv(sf_mg::Level& L, int dt, cudaStream_t st) {
  if (dt == SF_F64)
    SF_CUDA_CHECK(cudaMemcpyAsync(L.dinv, L.dinv64, L.n * 8, cudaMemcpyDeviceToDevice, st));
  else
    sf::k_convert<float, double><<<sf::grid_of(L.n), sf::kT, 0, st>>>(
        L.dinv64, static_cast<float*>(L.dinv), L.n);
  SF_CUDA_CHECK(cudaGetLastError());
}

// The captured iteration holds the smoother's coefficients and the kernels chosen for
// the levels' operators; it is captured again on the next solve.
void drop_graph(sf_mg* mg) {
  if (mg->exec) cudaGraphExecDestroy(mg->exec);
  if (mg->graph) cudaGraphDestroy(mg->graph);
  mg->exec = nullptr;
  mg->graph = nullptr;
  mg->graph_dtype = -1;
}

// Partial-sum slots for the reductions and the operator's fused (p, A p) sums.
void ensure_partials(sf_mg* mg) {
  const long long need = std::max<long long>(2 * sf::kMgBlocks, sf::op_dot_partials(mg->A));
  if (need <= mg->partials_n) return;
  mg->partials = static_cast<double*>(mg_alloc(mg, need * sizeof(double)));
  mg->partials_n = need;
}

// Buffers of the cycle in type dt (allocated on the first solve of that type).
void ensure_buffers(sf_mg* mg, int dt) {
  if (mg->dtype == dt) return;
  SF_REQUIRE(mg->dtype < 0, SF_ERR_STATE, "internal: cycle buffers of another type");
  const size_t es = esize(dt);
  size_t tmax = 0;
  for (size_t l = 0; l + 1 < mg->lv.size(); ++l) {  // largest transfer intermediate
    const auto& C = mg->lv[l + 1];
    const auto& t = mg->tr[l];
    const long long cx = (long long)C.nx * t.pc - 1, cy = (long long)C.ny * t.pc - 1;
    const long long fy = (long long)C.ny * t.F - 1, fz = (long long)C.nz * t.F - 1;
    const long long fx = (long long)C.nx * t.F - 1;
    tmax = std::max<size_t>(tmax, (size_t)std::max(cx * cy * fz, std::max(cx * fy * fz, fx * cy * fz)));
    tmax = std::max<size_t>(tmax, (size_t)(cx * fy * fz));
  }
  const auto& L0 = mg->lv[0];
  if (mg->has_basis) tmax = std::max<size_t>(tmax, (size_t)L0.n);
  mg->tmp1 = mg_alloc(mg, tmax * es);
  mg->tmp2 = mg_alloc(mg, tmax * es);
  for (size_t l = 0; l < mg->lv.size(); ++l) {
    auto& L = mg->lv[l];
    L.dinv = mg_alloc(mg, L.n * es);
    L.zb[0] = mg_alloc(mg, L.n * es);
    L.zb[1] = mg_alloc(mg, L.n * es);
    L.d = mg_alloc(mg, L.n * es);
    L.t = mg_alloc(mg, L.n * es);
    L.r = (l == 0 && !mg->has_basis) ? nullptr : mg_alloc(mg, L.n * es);
    cycle_dinv(L, dt, mg->cs);
  }
  mg->rl = mg_alloc(mg, mg->n * es);
  mg->zl = mg->has_basis ? mg_alloc(mg, mg->n * es) : nullptr;  // else level 0's current z
  if (!mg->has_basis) mg->lv[0].r = mg->rl;
  mg->dtype = dt;
}

// D^-1 and lmax of every level (FP64, power iteration on D^-1 A), from the levels'
// operators as they are now. The vectors are allocated on the first call.
void setup_levels(sf_mg* mg, cudaStream_t st) {
  if (!mg->pw_norms) {
    long long nmax = 0;
    for (auto& L : mg->lv) nmax = std::max(nmax, L.n);
    mg->pw_norms = static_cast<double*>(mg_alloc(mg, 2 * sizeof(double)));
    mg->pw_v = static_cast<double*>(mg_alloc(mg, nmax * 8));
    mg->pw_w = static_cast<double*>(mg_alloc(mg, nmax * 8));
    mg->pw_av = static_cast<double*>(mg_alloc(mg, nmax * 8));
    for (auto& L : mg->lv) L.dinv64 = static_cast<double*>(mg_alloc(mg, L.n * 8));
  }
  double* norms = mg->pw_norms;
  double *v = mg->pw_v, *w = mg->pw_w, *av = mg->pw_av;
  double h[2];
  for (auto& L : mg->lv) {
    sf::op_diag(L.op, av, st);
    sf::k_invert<double><<<sf::grid_of(L.n), sf::kT, 0, st>>>(av, L.dinv64, L.n);
    sf::k_pow_next<<<sf::grid_of(L.n), sf::kT, 0, st>>>(v, nullptr, nullptr, L.n, nullptr, 1);
    SF_CUDA_CHECK(cudaGetLastError());
    double lam = 0.0;
    for (int it = 0; it < 20; ++it) {
      sf::op_apply(L.op, SF_F64, v, av, st);
      sf::k_dinv_apply<<<sf::grid_of(L.n), sf::kT, 0, st>>>(w, av, L.dinv64, L.n);
      sf::k_pow_norms<<<sf::grid_of(L.n), sf::kT, 0, st>>>(w, v, L.n, mg->partials, mg->s, norms);
      sf::k_pow_next<<<sf::grid_of(L.n), sf::kT, 0, st>>>(v, av, L.dinv64, L.n, norms, 0);
      SF_CUDA_CHECK(cudaGetLastError());
      if (it >= 16) {
        SF_CUDA_CHECK(cudaMemcpyAsync(h, norms, sizeof(h), cudaMemcpyDeviceToHost, st));
        SF_CUDA_CHECK(cudaStreamSynchronize(st));
        lam = std::max(lam, std::sqrt(h[0] / (h[1] > 0 ? h[1] : 1.0)));
      }
    }
    SF_REQUIRE(std::isfinite(lam) && lam > 0.0, SF_ERR_NONFINITE,
               "multigrid set-up: no eigenvalue estimate of D^-1 A");
    L.lmax = lam;
  }
}

// One FCG iteration (everything after the residual is known).
template <typename TL>
void fcg_iteration(sf_mg* mg, int dt, cudaStream_t st) {
  const long long n = mg->n;
  precondition<TL>(mg, dt, st);
  const TL* z = static_cast<const TL*>(mg->has_basis ? mg->zl : mg->lv[0].z());
  const int g = sf::grid_of(n);
  sf::k_fcg_zq<TL><<<g, sf::kT, 0, st>>>(z, mg->q, n, mg->partials, mg->s);
  sf::k_fcg_dir<TL><<<g, sf::kT, 0, st>>>(z, mg->p, mg->r, n, mg->partials, mg->s);
  sf::op_apply_dot(mg->A, mg->p, mg->q, mg->partials, mg->s + sf::S_PQ, mg->s,
                   mg->s + sf::S_DONE, st);  // q = A p and (p, q)
  sf::k_fcg_update<TL><<<g, sf::kT, 0, st>>>(mg->x, mg->r, mg->p, mg->q,
                                              static_cast<TL*>(mg->rl), n, mg->partials, mg->s);
  SF_CUDA_CHECK(cudaGetLastError());
}

// Captures one iteration into a graph; returns false (and launches nothing) when the
// capture fails, in which case the iterations are launched directly.
bool capture(sf_mg* mg, int dt) {
  if (!mg->use_graph) return false;
  if (mg->exec && mg->graph_dtype == dt) return true;
  if (mg->exec) cudaGraphExecDestroy(mg->exec);
  if (mg->graph) cudaGraphDestroy(mg->graph);
  mg->exec = nullptr;
  mg->graph = nullptr;
  SF_CUDA_CHECK(cudaStreamBeginCapture(mg->cs, cudaStreamCaptureModeThreadLocal));
  bool ok = true;
  try {
    if (dt == SF_F64) fcg_iteration<double>(mg, dt, mg->cs);
    else fcg_iteration<float>(mg, dt, mg->cs);
  } catch (const Error&) {
    ok = false;
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(mg->cs, &g);
  if (!ok || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
    mg->use_graph = false;
    return false;
  }
  mg->graph = g;
  SF_CUDA_CHECK(cudaGraphInstantiate(&mg->exec, mg->graph, 0));
  mg->graph_dtype = dt;
  return true;
}

void check_level(const sf_op* op, const char* what) {
  SF_REQUIRE(op, SF_ERR_ARG, std::string("null ") + what);
  const sf::OpShape s = sf::op_shape(op);
  SF_REQUIRE(s.structured, SF_ERR_UNSUPPORTED,
             std::string(what) + " must be a whole 3D structured mesh (sf_set_structured) with "
                                 "its geometry set");
}

}  // namespace

extern "C" {

int sf_mg_create(sf_mg** out, sf_op* A, int nlevels, sf_op* const* levels,
                 const double* const* transfer, const double* basis_change) {
  if (!out) return SF_ERR_ARG;
  *out = nullptr;
  sf_mg* mg = new (std::nothrow) sf_mg();
  if (!mg) return SF_ERR_ARG;
  const int st = mg_guarded(mg, [&] {
    check_level(A, "operator");
    SF_REQUIRE(nlevels >= 1 && levels, SF_ERR_ARG, "need at least one level");
    mg->A = A;
    const sf::OpShape sa = sf::op_shape(A);
    mg->n = sa.n_free;
    for (int l = 0; l < nlevels; ++l) {
      check_level(levels[l], "level");
      const sf::OpShape s = sf::op_shape(levels[l]);
      sf_mg::Level L;
      L.op = levels[l];
      L.nx = s.nx;
      L.ny = s.ny;
      L.nz = s.nz;
      L.p = s.p;
      L.n = s.n_free;
      mg->lv.push_back(L);
    }
    const auto& L0 = mg->lv[0];
    SF_REQUIRE(L0.nx == sa.nx && L0.ny == sa.ny && L0.nz == sa.nz && L0.p == sa.p &&
                   L0.n == sa.n_free,
               SF_ERR_ARG, "level 0 must be the operator's mesh and order");
    for (int l = 0; l + 1 < nlevels; ++l) {
      const auto &F = mg->lv[l], &C = mg->lv[l + 1];
      SF_REQUIRE(transfer && transfer[l], SF_ERR_ARG, "missing transfer table");
      SF_REQUIRE(C.nx > 0 && F.nx % C.nx == 0 && F.ny % C.ny == 0 && F.nz % C.nz == 0,
                 SF_ERR_ARG, "coarse cells must split the fine cells evenly");
      const int r = F.nx / C.nx;
      SF_REQUIRE(F.ny / C.ny == r && F.nz / C.nz == r, SF_ERR_ARG,
                 "the coarsening ratio must be the same along every axis");
      SF_REQUIRE(C.p <= r * F.p, SF_ERR_ARG, "the coarse space must lie in the fine one");
      sf_mg::Transfer t;
      t.r = r;
      t.F = r * F.p;
      t.pc = C.p;
      SF_REQUIRE((t.F + 1) * (t.pc + 1) <= sf::kMaxW && t.pc <= sf::kMaxPc, SF_ERR_ARG,
                 "transfer table too large");
      SF_REQUIRE(F.nx * F.p <= 768 && F.nz * F.p <= 65535, SF_ERR_UNSUPPORTED,
                 "multigrid transfer: at most 767 free points per grid row");
      t.W.assign(transfer[l], transfer[l] + (t.F + 1) * (t.pc + 1));
      mg->tr.push_back(t);
    }
    if (basis_change) {
      mg->has_basis = true;
      mg->basis.r = 1;
      mg->basis.F = L0.p;
      mg->basis.pc = L0.p;
      SF_REQUIRE((L0.p + 1) * (L0.p + 1) <= sf::kMaxW && L0.p <= sf::kMaxPc, SF_ERR_ARG,
                 "basis table too large");
      SF_REQUIRE(L0.nx * L0.p <= 768, SF_ERR_UNSUPPORTED,
                 "multigrid transfer: at most 767 free points per grid row");
      mg->basis.W.assign(basis_change, basis_change + (L0.p + 1) * (L0.p + 1));
    }
    SF_CUDA_CHECK(cudaStreamCreateWithFlags(&mg->cs, cudaStreamNonBlocking));
    SF_CUDA_CHECK(cudaEventCreateWithFlags(&mg->ev_in, cudaEventDisableTiming));
    SF_CUDA_CHECK(cudaEventCreateWithFlags(&mg->ev_out, cudaEventDisableTiming));
    mg->s = static_cast<double*>(mg_alloc(mg, sf::S_NSLOTS * sizeof(double)));
    ensure_partials(mg);
    SF_CUDA_CHECK(cudaMemsetAsync(mg->s, 0, sf::S_NSLOTS * sizeof(double), mg->cs));
    SF_CUDA_CHECK(cudaMallocHost(&mg->h_s, sf::S_NSLOTS * sizeof(double)));
    mg->x = static_cast<double*>(mg_alloc(mg, mg->n * 8));
    mg->r = static_cast<double*>(mg_alloc(mg, mg->n * 8));
    mg->p = static_cast<double*>(mg_alloc(mg, mg->n * 8));
    mg->q = static_cast<double*>(mg_alloc(mg, mg->n * 8));
    setup_levels(mg, mg->cs);
    SF_CUDA_CHECK(cudaStreamSynchronize(mg->cs));
    mg->ready = true;
  });
  if (st != SF_OK) {
    // keep the handle so that the caller can read the message
    mg_release(mg);
    *out = mg;
    return st;
  }
  *out = mg;
  return SF_OK;
}

int sf_mg_destroy(sf_mg* mg) {
  if (!mg) return SF_OK;
  cudaDeviceSynchronize();
  mg_release(mg);
  delete mg;
  return SF_OK;
}

const char* sf_mg_last_error(const sf_mg* mg) { return mg ? mg->err.c_str() : "null handle"; }

int sf_mg_set_option(sf_mg* mg, const char* name, double value) {
  if (!mg || !name) return SF_ERR_ARG;
  return mg_guarded(mg, [&] {
    const std::string k(name);
    if (k == "degree") {
      SF_REQUIRE(value >= 1 && value <= 16, SF_ERR_ARG, "degree must be in 1..16");
      mg->degree = (int)value;
    } else if (k == "ratio") {
      SF_REQUIRE(value > 1.0, SF_ERR_ARG, "ratio must be > 1");
      mg->ratio = value;
    } else if (k == "coarse_steps") {
      SF_REQUIRE(value >= 1 && value <= 1000, SF_ERR_ARG, "coarse_steps must be in 1..1000");
      mg->coarse_steps = (int)value;
    } else if (k == "coarse_ratio") {
      SF_REQUIRE(value > 1.0, SF_ERR_ARG, "coarse_ratio must be > 1");
      mg->coarse_ratio = value;
    } else {
      throw Error(SF_ERR_ARG, "unknown multigrid option '" + k + "'");
    }
    drop_graph(mg);
  });
}

int sf_mg_refresh(sf_mg* mg, void* stream) {
  if (!mg) return SF_ERR_ARG;
  return mg_guarded(mg, [&] {
    SF_REQUIRE(!mg->lv.empty() && mg->cs, SF_ERR_STATE, "the multigrid set-up failed");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SF_CUDA_CHECK(cudaEventRecord(mg->ev_in, st));
    SF_CUDA_CHECK(cudaStreamWaitEvent(mg->cs, mg->ev_in, 0));
    mg->ready = false;  // until the new diagonals and estimates are in
    drop_graph(mg);
    ensure_partials(mg);
    setup_levels(mg, mg->cs);
    if (mg->dtype >= 0)
      for (auto& L : mg->lv) cycle_dinv(L, mg->dtype, mg->cs);
    SF_CUDA_CHECK(cudaStreamSynchronize(mg->cs));
    mg->ready = true;
  });
}

int sf_mg_get_info(const sf_mg* mg, const char* key, double* value) {
  if (!mg || !key || !value) return SF_ERR_ARG;
  const std::string k(key);
  if (k == "levels") *value = (double)mg->lv.size();
  else if (k.rfind("lmax", 0) == 0 && k.size() > 4) {
    const int l = std::atoi(k.c_str() + 4);
    if (l < 0 || l >= (int)mg->lv.size()) return SF_ERR_ARG;
    *value = mg->lv[l].lmax;
  } else if (k == "graph") {
    *value = mg->use_graph && mg->exec ? 1.0 : 0.0;
  } else if (k.rfind("n", 0) == 0 && k.size() > 1 && std::isdigit((unsigned char)k[1])) {
    const int l = std::atoi(k.c_str() + 1);
    if (l < 0 || l >= (int)mg->lv.size()) return SF_ERR_ARG;
    *value = (double)mg->lv[l].n;
  } else return SF_ERR_ARG;
  return SF_OK;
}

int sf_mg_cg(sf_mg* mg, int mode, const double* b, double* x, double reltol, int maxiter,
             int* iters, double* relres, void* stream) {
  if (!mg) return SF_ERR_ARG;
  return mg_guarded(mg, [&] {
    SF_REQUIRE(mg->ready, SF_ERR_STATE, "the multigrid set-up failed");
    SF_REQUIRE(b && x, SF_ERR_ARG, "null b or x");
    SF_REQUIRE(reltol > 0 && maxiter >= 0, SF_ERR_ARG, "bad reltol / maxiter");
    SF_REQUIRE(mode == SF_MG_MIXED || mode == SF_MG_F64, SF_ERR_ARG, "unknown multigrid mode");
    const int dt = mode == SF_MG_F64 ? SF_F64 : SF_F32;
    SF_REQUIRE(mg->dtype < 0 || mg->dtype == dt, SF_ERR_UNSUPPORTED,
               "a multigrid handle solves in one mode only (create another for the other)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = mg->n;
    // the caller's stream first, then the solver's own stream
    SF_CUDA_CHECK(cudaEventRecord(mg->ev_in, st));
    SF_CUDA_CHECK(cudaStreamWaitEvent(mg->cs, mg->ev_in, 0));
    ensure_buffers(mg, dt);
    const bool graph = capture(mg, dt);
    cudaStream_t cs = mg->cs;
    SF_CUDA_CHECK(cudaMemcpyAsync(mg->x, x, n * 8, cudaMemcpyDeviceToDevice, cs));
    sf::op_apply(mg->A, SF_F64, mg->x, mg->q, cs);
    const int g = sf::grid_of(n);
    if (dt == SF_F64)
      sf::k_fcg_start<double><<<g, sf::kT, 0, cs>>>(b, mg->q, mg->r, static_cast<double*>(mg->rl),
                                                    n, reltol * reltol, mg->partials, mg->s);
    else
      sf::k_fcg_start<float><<<g, sf::kT, 0, cs>>>(b, mg->q, mg->r, static_cast<float*>(mg->rl),
                                                   n, reltol * reltol, mg->partials, mg->s);
    SF_CUDA_CHECK(cudaGetLastError());
    SF_CUDA_CHECK(cudaMemcpyAsync(mg->h_s, mg->s, sf::S_NSLOTS * sizeof(double),
                                  cudaMemcpyDeviceToHost, cs));
    SF_CUDA_CHECK(cudaStreamSynchronize(cs));
    double done = mg->h_s[sf::S_DONE];
    for (int queued = 0; queued < maxiter && done == 0.0;) {
      const int chunk = std::min(sf::kChunk, maxiter - queued);
      for (int k = 0; k < chunk; ++k) {
        if (graph) SF_CUDA_CHECK(cudaGraphLaunch(mg->exec, cs));
        else if (dt == SF_F64) fcg_iteration<double>(mg, dt, cs);
        else fcg_iteration<float>(mg, dt, cs);
      }
      queued += chunk;
      SF_CUDA_CHECK(cudaMemcpyAsync(mg->h_s, mg->s, sf::S_NSLOTS * sizeof(double),
                                    cudaMemcpyDeviceToHost, cs));
      SF_CUDA_CHECK(cudaStreamSynchronize(cs));
      done = mg->h_s[sf::S_DONE];
    }
    SF_CUDA_CHECK(cudaMemcpyAsync(x, mg->x, n * 8, cudaMemcpyDeviceToDevice, cs));
    SF_CUDA_CHECK(cudaEventRecord(mg->ev_out, cs));
    SF_CUDA_CHECK(cudaStreamWaitEvent(st, mg->ev_out, 0));
    SF_REQUIRE(done != 3.0, SF_ERR_NONFINITE, "non-finite residual in the multigrid CG");
    const double bb = mg->h_s[sf::S_BB];
    const double rel = std::sqrt(mg->h_s[sf::S_RR]) / (bb > 0 ? std::sqrt(bb) : 1.0);
    if (iters) *iters = (int)mg->h_s[sf::S_ITERS];
    if (relres) *relres = rel;
    if (!(rel <= reltol)) throw Error(SF_ERR_NOT_CONVERGED, "multigrid CG reached its iteration cap");
  });
}

}  // extern "C"
