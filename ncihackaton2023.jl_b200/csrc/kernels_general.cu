// General element kernel: one element per group of max(SB,SQ)^2 threads.
//
// This is the per-cell action Arrays.evaluate! of SumFactorizationMap
// (src/SumFactorizationMaps.jl:78-89) together with the gather/assemble of
// LazyMatrix mul! (src/LazyMatrices.jl:52-61). The arithmetic is the same
// y_e = sum_r B_r^T G B_r x_e. The reference loops over D redundant
// components (src/SumFactorizationKernels.jl:40-65,105-130). Here the
// interpolation is shared between the gradient components instead:
//   forward  x: A1 = A x, B1 = B x            (SB*SB lines)
//            y: AA = A A1, AB = B A1, BA = A B1 (SQ*SB lines)
//            z: ux = A BA, uy = A AB, uz = B AA (SQ*SQ lines, registers)
//   metric   v = G(q) u, with G = wq djq jq^T jq (src/SumFactorizationKernels.jl:174-216)
//   backward the transposes in reverse order.
// Every pass gives each thread one full 1D line, read from shared memory into
// registers. The thread computes all outputs of the line, so every value
// loaded is reused SQ (or SB) times. The 1D matrices are passed in the kernel's
// __grid_constant__ parameters (staged in shared memory for FP64 at high order,
// see kStageMats). The scatter-add uses atomics into a y that was zeroed before
// the launch. Dirichlet dofs (id < 0) read as zero and are skipped.
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "sf_internal.cuh"

namespace sf {
namespace {

// Even-odd tables of one R x C operator M with M[R-1-r][C-1-c] = sign M[r][c]
// (A and A^T: sign +1; B and B^T: sign -1). Row r < HR holds the pairs
// (E[r][i], O[r][i]) for i < HC, with E[r][i] = (M[r][i] + M[r][C-1-i]) / 2 and
// O[r][i] = (M[r][i] - M[r][C-1-i]) / 2, then (M[r][HC], 0) when C is odd, so
// that one 2-wide shared load fetches a pair. Row length W is even.
template <int R, int C>
struct EOT {
  static constexpr int HR = (R + 1) / 2, HC = C / 2, MC = C % 2, W = 2 * HC + 2 * MC;
  static constexpr int N = HR * W;
};
template <int SB, int SQ>
struct EOTables {  // offsets of the tables of A, B (SQ x SB) and A^T, B^T (SB x SQ)
  static constexpr int NA = EOT<SQ, SB>::N, NT = EOT<SB, SQ>::N;
  static constexpr int OFF[4] = {0, NA, 2 * NA, 2 * NA + NT};
  static constexpr int TOTAL = 2 * NA + 2 * NT;
};

template <int SB, int SQ, typename T>
struct GenParams {
  T A[SQ * SB];  // [qp][basis]
  T B[SQ * SB];
  T eo[EOTables<SB, SQ>::TOTAL];  // even-odd tables (used when A and B are symmetric)
  double w1[SQ];
  double G0[6];
  const T* x;
  T* y;
  const int32_t* ids;   // CSR tensor-ordered ids or null (structured)
  const int32_t* t2l;     // cell-local mode: tensor position -> local dof k
  long long ncells;
  int nx, ny, nz;
  int mode;             // 0 = assembled apply, 1 = cell-local evaluate, 2 = diagonal
  int geom;             // GEOM_SEPARABLE / GEOM_TABLE
  const double* gtab;
  long long gstride;
  const float* gtab32;  // FP32 copy of gtab (read by the FP32 kernel)
  long long gstride32;
  const double* kappa;
  const double* wdet;
  long long wdet_stride;
};

template <int SB, int SQ>
struct Shape {
  static constexpr int SM = SB > SQ ? SB : SQ;
  static constexpr int NL = SM * SM;                    // threads per element
  static constexpr int S0 = SB * SB * SB;                // X / Y
  static constexpr int S1 = SB * SB * SQ;                // each of A1, B1
  static constexpr int S2 = SB * SQ * SQ;                // each of AA, AB, BA
  static constexpr int EPB = (256 / NL) > 0 ? (256 / NL) : 1;  // elements per block
  static constexpr int THREADS = EPB * NL;
  static constexpr int SM3 = SM * SM * SM;
  static constexpr int SL = 3 * SM3;  // words per element of k_general (three padded slots)
  static constexpr int MINB = 2;      // CTAs per SM asked of the register allocator
};

// Global free index of tensor position `pos` of cell `c` on the structured mesh, or -1.
__device__ __forceinline__ long long structured_index(long long c, int pos, int SB, int nx, int ny,
                                                      int nz) {
  const int p = SB - 1;
  const int cx = (int)(c % nx);
  const long long r = c / nx;
  const int cy = (int)(r % ny);
  const int cz = (int)(r / ny);
  const int i = pos % SB, j = (pos / SB) % SB, k = pos / (SB * SB);
  const int gx = cx * p + i, gy = cy * p + j, gz = cz * p + k;
  const int Nx = nx * p, Ny = ny * p, Nz = nz * p;
  if (gx <= 0 || gx >= Nx || gy <= 0 || gy >= Ny || gz <= 0 || gz >= Nz) return -1;
  return (long long)(gx - 1) + (long long)(Nx - 1) * ((long long)(gy - 1) + (long long)(Ny - 1) * (gz - 1));
}

// The same index with the cell's coordinates worked out once (structured_index
// recomputes them from c on every call): cell_origin gives the grid point of the
// cell's first node, cell_dof the free index of its tensor position (i, j, k).
struct CellOrigin {
  int gx, gy, gz, Nx, Ny, Nz;
};
__device__ __forceinline__ CellOrigin cell_origin(long long c, int p, int nx, int ny, int nz) {
  const int cx = (int)(c % nx);
  const long long r = c / nx;
  const int cy = (int)(r % ny);
  const int cz = (int)(r / ny);
  return CellOrigin{cx * p, cy * p, cz * p, nx * p, ny * p, nz * p};
}
__device__ __forceinline__ long long cell_dof(const CellOrigin& o, int i, int j, int k) {
  const int gx = o.gx + i, gy = o.gy + j, gz = o.gz + k;
  if (gx <= 0 || gx >= o.Nx || gy <= 0 || gy >= o.Ny || gz <= 0 || gz >= o.Nz) return -1;
  return (long long)(gx - 1) +
         (long long)(o.Nx - 1) * ((long long)(gy - 1) + (long long)(o.Ny - 1) * (gz - 1));
}

template <typename T>
__device__ __forceinline__ void atomic_add(T* a, T v) { atomicAdd(a, v); }

// FP64 FMAs cannot take a 64-bit operand from the constant bank, so the FP64
// 1D matrices are staged once per CTA in shared memory and read with
// broadcast loads; keeping 2*SQ*SB doubles in registers would cost up to 162
// registers per thread at Q8. FP32 reads them straight from the kernel
// parameters below SQ*SB = 64.
template <typename T, int SB, int SQ>
constexpr bool kStageMats = sizeof(T) == 8 ? SQ * SB >= 16 : SQ * SB >= 64;
#define MA(i) (kStageMats<T, SB, SQ> ? sMat[(i)] : P.A[(i)])
#define MB(i) (kStageMats<T, SB, SQ> ? sMat[SQ * SB + (i)] : P.B[(i)])

template <int SB, int SQ, typename T>
__device__ __forceinline__ void stage_mats(const GenParams<SB, SQ, T>& P, T* sMat) {
  if constexpr (kStageMats<T, SB, SQ>) {
    for (int i = threadIdx.x; i < SQ * SB; i += blockDim.x) {
      sMat[i] = P.A[i];
      sMat[SQ * SB + i] = P.B[i];
    }
  }
}

// Element kernel. Shared memory per element is three slots U0, U1, U2 of
// SM^3 words each, indexed (c3 * SM + c2) * SM + c1 with c1 fastest. Every
// pass gives a thread whole 1D lines, and the line's inputs and outputs sit at
// the same slot positions (the padding to SM makes that true for SB != SQ),
// so each pass works in place on positions no other thread touches:
//   gather      U0 = X
//   forward x   lines (j,k):   U1 = A1 = A X,  U2 = B1 = B X
//   forward y   lines (qi,k):  U1 = AA = A A1, U0 = AB = B A1, U2 = BA = A B1
//   z           lines (qi,qj): u = (A BA, A AB, B AA) in place, one component at a
//               time; v = G(q) u point by point; the transposes back, again one
//               component at a time (the same thread, so no barrier in between)
//   backward y  lines (qi,k):  U1 = A1 = A^T AA + B^T AB,  U2 = B1 = A^T BA
//   backward x  lines (j,k):   U0 = Y = A^T A1 + B^T B1
// A thread holds at most 2 lines (18 values at Q8) in registers, which keeps
// several CTAs resident per SM to hide the latency of the per-point metric.
// Shared copy of the even-odd tables (read with broadcast loads).
template <int SB, int SQ, typename T>
__device__ __forceinline__ void stage_eo(const GenParams<SB, SQ, T>& P, T* sEO) {
  for (int i = threadIdx.x; i < EOTables<SB, SQ>::TOTAL; i += blockDim.x) sEO[i] = P.eo[i];
}

// Even-odd table entries read from the kernel parameters (FP32: an FMA takes a
// constant-bank operand; deformed Q8 0.537 -> 0.464 ms) or from the shared copy
// (FP64: the parameter reads measured slower, 0.723 -> 0.835 ms at Q8).
template <typename T>
constexpr bool kEOParams = sizeof(T) == 4;

// out(r, v) for r < R receives (M u)[r], M one of A, B (OP 0, 1; R = SQ, C = SB) or
// A^T, B^T (OP 2, 3; R = SB, C = SQ). EO: through the even-odd tables in sEO
// (about half the FMAs and matrix loads); otherwise the full matrices.
template <int OP, bool EO, int SB, int SQ, typename T, int R, int C, typename Out>
__device__ __forceinline__ void contract(const T* sMat, const T* sEO, const GenParams<SB, SQ, T>& P,
                                         const T (&u)[C], const Out& out) {
  if constexpr (EO) {
    using E = EOT<R, C>;
    using V2 = typename std::conditional<sizeof(T) == 8, double2, float2>::type;
    const V2* tab = reinterpret_cast<const V2*>(sEO + EOTables<SB, SQ>::OFF[OP]);
    constexpr bool anti = OP == 1 || OP == 3;
    T ue[E::HC > 0 ? E::HC : 1], uo[E::HC > 0 ? E::HC : 1];
#pragma unroll
    for (int i = 0; i < E::HC; ++i) {
      ue[i] = u[i] + u[C - 1 - i];
      uo[i] = u[i] - u[C - 1 - i];
    }
#pragma unroll
    for (int r = 0; r < E::HR; ++r) {
      const V2* t = tab + r * (E::W / 2);
      const T* pt = P.eo + EOTables<SB, SQ>::OFF[OP] + r * E::W;
      constexpr bool kParam = kEOParams<T>;
      T e = E::MC ? (kParam ? pt[2 * E::HC] : (T)t[E::HC].x) * u[E::HC] : T(0);
      T o = T(0);
#pragma unroll
      for (int i = 0; i < E::HC; ++i) {
        const T ex = kParam ? pt[2 * i] : (T)t[i].x;
        const T ox = kParam ? pt[2 * i + 1] : (T)t[i].y;
        e = fma(ex, ue[i], e);
        o = fma(ox, uo[i], o);
      }
      out(r, e + o);
      if (R - 1 - r != r) out(R - 1 - r, anti ? o - e : e - o);
    }
  } else {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      T acc = T(0);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int ix = OP < 2 ? r * SB + c : c * SB + r;
        acc = fma((OP == 0 || OP == 2) ? MA(ix) : MB(ix), u[c], acc);
      }
      out(r, acc);
    }
  }
}

// Four CTAs per SM are asked of the register allocator (at most 64 registers at 256
// threads): the kernel waits on its metric and gather loads, and a fourth CTA hides more of
// that than the registers cost. Measured against three CTAs (deformed Q8 32^3; Q4 64^3 table
// gather): FP32 0.444 -> 0.378 ms and 0.565 -> 0.433 ms, FP64 0.723 -> 0.712 ms and
// 0.948 -> 0.912 ms (no spills at Q8 FP64, 24 bytes at Q8 FP32). FP32 elements of 9 or more
// points per axis ask for five (deformed Q8 FP32 0.362 -> 0.341 ms with 80 bytes of spills; at
// Q4 five were 1 % slower).
template <typename T, int SM>
constexpr int kMinbApply = sizeof(T) == 4 && SM >= 9 ? 5 : 4;
template <int SB, int SQ, typename T, bool EO>
__global__ void __launch_bounds__(Shape<SB, SQ>::THREADS, kMinbApply<T, Shape<SB, SQ>::SM>)
k_general(const __grid_constant__ GenParams<SB, SQ, T> P) {
  using S = Shape<SB, SQ>;
  constexpr int SM = S::SM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int el = threadIdx.x / S::NL;
  const int l = threadIdx.x % S::NL;
  const long long cell = (long long)blockIdx.x * S::EPB + el;
  const bool valid = cell < P.ncells;
  // One thread per element asks for the element's row of the metric table in L2: it
  // arrives while the gather and the forward passes run, and the metric stage's loads
  // then hit L2. The row starts on a 16-byte boundary (6 SQ^3 doubles, or the padded
  // FP32 row); the size is rounded down to 16 bytes, so it stays inside the row.
  if (P.geom == GEOM_TABLE && valid && l == 0) {
    const void* row = sizeof(T) == 4 ? static_cast<const void*>(P.gtab32 + cell * P.gstride32)
                                     : static_cast<const void*>(P.gtab + cell * P.gstride);
    constexpr unsigned kRowBytes = (unsigned)(6 * SQ * SQ * SQ * sizeof(T)) & ~15u;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(row), "r"(kRowBytes)
                 : "memory");
  }

  T* U0 = reinterpret_cast<T*>(smem_raw) + (size_t)el * S::SL;
  T* U1 = U0 + S::SM3;
  T* U2 = U1 + S::SM3;
  __shared__ T sMat[(!EO && kStageMats<T, SB, SQ>) ? 2 * SQ * SB : 1];
  __shared__ __align__(16) T sEO[EO ? EOTables<SB, SQ>::TOTAL : 2];
  if constexpr (EO) stage_eo<SB, SQ, T>(P, sEO);
  else stage_mats<SB, SQ, T>(P, sMat);  // visible after the first __syncthreads below
  auto at = [](int c3, int c2, int c1) { return (c3 * SM + c2) * SM + c1; };
  // u[c] = io[c * stride] (c < N); keeps the compiler from overlapping consecutive
  // line passes, which would hold several lines in registers at once
  auto load = [](const T* io, int stride, auto& u) {
    asm volatile("" ::: "memory");
    constexpr int N = sizeof(u) / sizeof(T);
#pragma unroll
    for (int c = 0; c < N; ++c) u[c] = io[c * stride];
  };

  // ---------------- gather ----------------
  // structured gather only (the table and cell-local modes have no mesh sizes)
  const CellOrigin org = (valid && !P.ids && P.mode != 1)
                             ? cell_origin(cell, SB - 1, P.nx, P.ny, P.nz)
                             : CellOrigin{0, 0, 0, 0, 0, 0};
  for (int pos = l; pos < S::S0; pos += S::NL) {
    const int i = pos % SB, j = (pos / SB) % SB, k = pos / (SB * SB);
    T v = T(0);
    if (valid) {
      if (P.mode == 1) {
        // cell-local: x_cells[cell][k] with k the local dof of tensor position pos
        v = P.x[cell * S::S0 + P.t2l[pos]];
      } else if (P.ids) {
        const int id = P.ids[cell * S::S0 + pos];
        if (id >= 0) v = P.x[id];
      } else {
        const long long id = cell_dof(org, i, j, k);
        if (id >= 0) v = P.x[id];
      }
    }
    U0[at(k, j, i)] = v;
  }
  __syncthreads();

  // ---------------- forward x: lines (j,k): A1 = A X, B1 = B X ----------------
  if (l < SB * SB) {
    const int j = l % SB, k = l / SB;
    T u[SB];
    load(U0 + at(k, j, 0), 1, u);
    T* a1 = U1 + at(k, j, 0);
    T* b1 = U2 + at(k, j, 0);
    contract<0, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { a1[r] = v; });
    contract<1, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { b1[r] = v; });
  }
  __syncthreads();

  // ---------- forward y: lines (qi,k): AA = A A1, AB = B A1, BA = A B1 ----------
  if (l < SQ * SB) {
    const int qi = l % SQ, k = l / SQ;
    T* l0 = U0 + at(k, 0, qi);
    T* l1 = U1 + at(k, 0, qi);
    T* l2 = U2 + at(k, 0, qi);
    {
      T u[SB];
      load(l1, SM, u);
      contract<0, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { l1[r * SM] = v; });
      contract<1, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { l0[r * SM] = v; });
    }
    T u[SB];
    load(l2, SM, u);
    contract<0, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { l2[r * SM] = v; });
  }
  __syncthreads();

  // ------------- z: forward, metric, backward; lines (qi,qj) -------------
  if (l < SQ * SQ) {
    const int qi = l % SQ, qj = l / SQ;
    constexpr int ZS = SM * SM;
    T* zx = U2 + at(0, qj, qi);  // BA -> ux -> vx -> back
    T* zy = U0 + at(0, qj, qi);  // AB -> uy -> vy -> back
    T* zz = U1 + at(0, qj, qi);  // AA -> uz -> vz -> back
    {
      T u[SB];
      load(zx, ZS, u);
      contract<0, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { zx[r * ZS] = v; });
    }
    {
      T u[SB];
      load(zy, ZS, u);
      contract<0, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { zy[r * ZS] = v; });
    }
    {
      T u[SB];
      load(zz, ZS, u);
      contract<1, EO, SB, SQ, T, SQ, SB>(sMat, sEO, P, u, [&](int r, T v) { zz[r * ZS] = v; });
    }
    // metric v = G u in the kernel's type: the FP64 kernel reads the FP64 table, the
    // FP32 kernel its FP32 copy (half the bytes of the largest stream)
    const long long gc = valid ? cell : 0;
    const double* gt = P.geom == GEOM_SEPARABLE || sizeof(T) == 4 ? nullptr : P.gtab + gc * P.gstride;
    const float* gt32 = P.geom == GEOM_SEPARABLE || sizeof(T) == 8 ? nullptr
                                                                   : P.gtab32 + gc * P.gstride32;
#pragma unroll 3
    for (int qk = 0; qk < SQ; ++qk) {
      const int q = qi + SQ * (qj + SQ * qk);
      T g[6];
      asm volatile("" ::: "memory");
      if (P.geom == GEOM_SEPARABLE) {
        const double s = P.w1[qi] * P.w1[qj] * P.w1[qk];
#pragma unroll
        for (int c = 0; c < 6; ++c) g[c] = (T)(s * P.G0[c]);
      } else if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int c = 0; c < 6; ++c) g[c] = __ldg(gt32 + c * SQ * SQ * SQ + q);
      } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) g[c] = __ldg(gt + c * SQ * SQ * SQ + q);
      }
      if (P.kappa) {
        const T kq = valid ? (T)P.kappa[cell * (SQ * SQ * SQ) + q] : T(0);
#pragma unroll
        for (int c = 0; c < 6; ++c) g[c] *= kq;
      }
      const T dx = zx[qk * ZS], dy = zy[qk * ZS], dz = zz[qk * ZS];
      zx[qk * ZS] = g[0] * dx + g[3] * dy + g[4] * dz;
      zy[qk * ZS] = g[3] * dx + g[1] * dy + g[5] * dz;
      zz[qk * ZS] = g[4] * dx + g[5] * dy + g[2] * dz;
    }
    {
      T u[SQ];
      load(zx, ZS, u);
      contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { zx[r * ZS] = v; });
    }
    {
      T u[SQ];
      load(zy, ZS, u);
      contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { zy[r * ZS] = v; });
    }
    {
      T u[SQ];
      load(zz, ZS, u);
      contract<3, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { zz[r * ZS] = v; });
    }
  }
  __syncthreads();

  // ------- backward y: lines (qi,k): A1 = A^T AA + B^T AB, B1 = A^T BA -------
  if (l < SQ * SB) {
    const int qi = l % SQ, k = l / SQ;
    T* l0 = U0 + at(k, 0, qi);
    T* l1 = U1 + at(k, 0, qi);
    T* l2 = U2 + at(k, 0, qi);
    {
      T u[SQ];
      load(l1, SM, u);
      contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { l1[r * SM] = v; });
    }
    {
      T u[SQ];
      load(l0, SM, u);
      contract<3, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { l1[r * SM] += v; });
    }
    T u[SQ];
    load(l2, SM, u);
    contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { l2[r * SM] = v; });
  }
  __syncthreads();

  // ---------------- backward x: lines (j,k): Y = A^T A1 + B^T B1 in U0 ----------------
  if (l < SB * SB) {
    const int j = l % SB, k = l / SB;
    T* y0 = U0 + at(k, j, 0);
    {
      T u[SQ];
      load(U1 + at(k, j, 0), 1, u);
      contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { y0[r] = v; });
    }
    T u[SQ];
    load(U2 + at(k, j, 0), 1, u);
    contract<3, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { y0[r] += v; });
  }
  __syncthreads();

  // ---------------- scatter ----------------
  if (!valid) return;
  for (int pos = l; pos < S::S0; pos += S::NL) {
    const int i = pos % SB, j = (pos / SB) % SB, k = pos / (SB * SB);
    const T v = U0[at(k, j, i)];
    if (P.mode == 1) {
      P.y[cell * S::S0 + P.t2l[pos]] = v;
    } else if (P.ids) {
      const int id = P.ids[cell * S::S0 + pos];
      if (id >= 0) atomic_add(P.y + id, v);
    } else {
      const long long id = cell_dof(org, i, j, k);
      if (id >= 0) atomic_add(P.y + id, v);
    }
  }
}

// Right-hand side of the linear form v -> integral of f v (profiling/drivers.jl:20):
// b_e = (A^T (x) A^T (x) A^T) (w |det J| f) per cell, the scalar interpolation of
// src/SumFactorizationKernels.jl:15-38 transposed, then assembled with atomics.
// P.x holds f at the points ([cell][SQ^3]); one slot of SM^3 words per element,
// the same in-place line passes as k_general.
template <int SB, int SQ, bool EO>
__global__ void __launch_bounds__(Shape<SB, SQ>::THREADS, Shape<SB, SQ>::MINB)
k_rhs(const __grid_constant__ GenParams<SB, SQ, double> P) {
  using S = Shape<SB, SQ>;
  using T = double;
  constexpr int SM = S::SM, NQ = SQ * SQ * SQ;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int el = threadIdx.x / S::NL;
  const int l = threadIdx.x % S::NL;
  const long long cell = (long long)blockIdx.x * S::EPB + el;
  const bool valid = cell < P.ncells;
  T* U = reinterpret_cast<T*>(smem_raw) + (size_t)el * S::SM3;
  __shared__ T sMat[(!EO && kStageMats<T, SB, SQ>) ? 2 * SQ * SB : 1];
  __shared__ __align__(16) T sEO[EO ? EOTables<SB, SQ>::TOTAL : 2];
  if constexpr (EO) stage_eo<SB, SQ, T>(P, sEO);
  else stage_mats<SB, SQ, T>(P, sMat);
  auto at = [](int c3, int c2, int c1) { return (c3 * SM + c2) * SM + c1; };
  auto load = [](const T* io, int stride, auto& u) {
    asm volatile("" ::: "memory");
    constexpr int N = sizeof(u) / sizeof(T);
#pragma unroll
    for (int c = 0; c < N; ++c) u[c] = io[c * stride];
  };
  // weighted point values
  const double* wd = P.wdet + (valid ? cell : 0) * P.wdet_stride;
  for (int q = l; q < NQ; q += S::NL) {
    const int qi = q % SQ, qj = (q / SQ) % SQ, qk = q / (SQ * SQ);
    U[at(qk, qj, qi)] = valid ? P.x[cell * NQ + q] * wd[q] : 0.0;
  }
  __syncthreads();
  if (l < SQ * SQ) {  // z: lines (qi, qj)
    const int qi = l % SQ, qj = l / SQ;
    T* z = U + at(0, qj, qi);
    T u[SQ];
    load(z, SM * SM, u);
    contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { z[r * SM * SM] = v; });
  }
  __syncthreads();
  if (l < SQ * SB) {  // y: lines (qi, k)
    const int qi = l % SQ, k = l / SQ;
    T* yl = U + at(k, 0, qi);
    T u[SQ];
    load(yl, SM, u);
    contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { yl[r * SM] = v; });
  }
  __syncthreads();
  if (l < SB * SB) {  // x: lines (j, k)
    const int j = l % SB, k = l / SB;
    T* xl = U + at(k, j, 0);
    T u[SQ];
    load(xl, 1, u);
    contract<2, EO, SB, SQ, T, SB, SQ>(sMat, sEO, P, u, [&](int r, T v) { xl[r] = v; });
  }
  __syncthreads();
  if (!valid) return;
  const CellOrigin org =
      P.ids ? CellOrigin{0, 0, 0, 0, 0, 0} : cell_origin(cell, SB - 1, P.nx, P.ny, P.nz);
  for (int pos = l; pos < S::S0; pos += S::NL) {
    const int i = pos % SB, j = (pos / SB) % SB, k = pos / (SB * SB);
    const long long id = P.ids ? (long long)P.ids[cell * S::S0 + pos] : cell_dof(org, i, j, k);
    if (id >= 0) atomicAdd(P.y + id, U[at(k, j, i)]);
  }
}

// Diagonal of the assembled operator: for each cell and tensor position a,
//   diag_e[a] = sum_q kappa(q) sum_{r,s} G_rs(q) dphi_a/dxi_r(q) dphi_a/dxi_s(q).
// The 3D gradient is a product of 1D values, so for each of the six symmetric
// pairs (r, s) the product of two gradients is, direction by direction, one of
// W0 = A*A, W1 = A*B, W2 = B*B (elementwise, [q][a]), and
//   diag_e[a1 a2 a3] += c_rs sum_{q1 q2 q3} H_rs(q) W(q1,a1) W'(q2,a2) W''(q3,a3)
// with H_rs = kappa G_rs and c_rs = 1 (r = s) or 2: three 1D contractions per pair
// (sum factorization), about SB SQ^3 + SB^2 SQ^2 + SB^3 SQ multiply-adds each
// instead of SB^3 SQ^3. One element per max(SB,SQ)^2 threads, as in k_general;
// per element H, the two partial contractions and the diagonal sit in shared
// memory. Assembled with atomics (Jacobi needs diag(A)).
template <int SB, int SQ>
struct DiagShape {
  static constexpr int NQ = SQ * SQ * SQ;
  static constexpr int WE = NQ + SB * SQ * SQ + SB * SB * SQ + SB * SB * SB;  // words per element
};

template <int SB, int SQ, typename T>
__global__ void __launch_bounds__(Shape<SB, SQ>::THREADS)
k_general_diag(const __grid_constant__ GenParams<SB, SQ, T> P) {
  using S = Shape<SB, SQ>;
  using DS = DiagShape<SB, SQ>;
  constexpr int NQ = DS::NQ, S0 = SB * SB * SB;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int el = threadIdx.x / S::NL;
  const int l = threadIdx.x % S::NL;
  const long long cell = (long long)blockIdx.x * S::EPB + el;
  const bool valid = cell < P.ncells;
  double* H = reinterpret_cast<double*>(smem_raw) + (size_t)el * DS::WE;  // [q3][q2][q1]
  double* T1 = H + NQ;                // [q3][q2][a1]
  double* T2 = T1 + SB * SQ * SQ;     // [q3][a2][a1]
  double* D = T2 + SB * SB * SQ;      // [a3][a2][a1]
  __shared__ double W[3][SQ * SB];    // A*A, A*B, B*B, [q][a]
  for (int i = threadIdx.x; i < SQ * SB; i += S::THREADS) {
    const double a = (double)P.A[i], b = (double)P.B[i];
    W[0][i] = a * a;
    W[1][i] = a * b;
    W[2][i] = b * b;
  }
  for (int i = l; i < S0; i += S::NL) D[i] = 0.0;
  const double* gt = P.gtab + (valid ? cell : 0) * P.gstride;
#pragma unroll 1
  for (int k = 0; k < 6; ++k) {  // G components xx, yy, zz, xy, xz, yz
    const int r = k < 3 ? k : (k == 5 ? 1 : 0);
    const int sp = k < 3 ? k : (k == 3 ? 1 : 2);
    const double cf = k < 3 ? 1.0 : 2.0;
    __syncthreads();  // W written; the last pass of the previous pair has read H
    for (int q = l; q < NQ; q += S::NL) {
      double g = 0.0;
      if (valid) {
        if (P.geom == GEOM_SEPARABLE) {
          const int qi = q % SQ, qj = (q / SQ) % SQ, qk = q / (SQ * SQ);
          g = P.w1[qi] * P.w1[qj] * P.w1[qk] * P.G0[k];
        } else {
          g = gt[k * NQ + q];
        }
        if (P.kappa) g *= P.kappa[cell * NQ + q];
      }
      H[q] = cf * g;
    }
    __syncthreads();
    const double* W1 = W[(r == 0) + (sp == 0)];
    const double* W2 = W[(r == 1) + (sp == 1)];
    const double* W3 = W[(r == 2) + (sp == 2)];
    if (l < SQ * SQ) {  // q1 -> a1 on lines (q2, q3)
      double in[SQ];
#pragma unroll
      for (int q1 = 0; q1 < SQ; ++q1) in[q1] = H[l * SQ + q1];
#pragma unroll
      for (int a1 = 0; a1 < SB; ++a1) {
        double acc = 0.0;
#pragma unroll
        for (int q1 = 0; q1 < SQ; ++q1) acc = fma(W1[q1 * SB + a1], in[q1], acc);
        T1[l * SB + a1] = acc;
      }
    }
    __syncthreads();
    if (l < SB * SQ) {  // q2 -> a2 on lines (a1, q3)
      const int a1 = l % SB, q3 = l / SB;
      double in[SQ];
#pragma unroll
      for (int q2 = 0; q2 < SQ; ++q2) in[q2] = T1[(q3 * SQ + q2) * SB + a1];
#pragma unroll
      for (int a2 = 0; a2 < SB; ++a2) {
        double acc = 0.0;
#pragma unroll
        for (int q2 = 0; q2 < SQ; ++q2) acc = fma(W2[q2 * SB + a2], in[q2], acc);
        T2[(q3 * SB + a2) * SB + a1] = acc;
      }
    }
    __syncthreads();
    if (l < SB * SB) {  // q3 -> a3 on lines (a1, a2), added into the diagonal
      double in[SQ];
#pragma unroll
      for (int q3 = 0; q3 < SQ; ++q3) in[q3] = T2[q3 * SB * SB + l];
#pragma unroll
      for (int a3 = 0; a3 < SB; ++a3) {
        double acc = 0.0;
#pragma unroll
        for (int q3 = 0; q3 < SQ; ++q3) acc = fma(W3[q3 * SB + a3], in[q3], acc);
        D[a3 * SB * SB + l] += acc;
      }
    }
  }
  __syncthreads();
  if (!valid) return;
  for (int pos = l; pos < S0; pos += S::NL) {
    long long id;
    if (P.ids) id = P.ids[cell * S0 + pos];
    else id = structured_index(cell, pos, SB, P.nx, P.ny, P.nz);
    if (id >= 0) atomicAdd(P.y + id, (T)D[pos]);
  }
}

// ---------------------------------------------------------------------------
// Vector-Jacobian product of y = A(kappa) x with respect to kappa:
//   kappa_bar[c][q] = (grad ybar)_q^T G_q (grad x)_q
// with G = wq djq jq^T jq (without kappa). This is the derivative of ybar^T A(kappa) x
// with respect to kappa_q, the per-point factor of the reference's apply_weights
// (src/SumFactorizationKernels.jl:174-216). The gradients at the points are
// recomputed by sum factorization for both vectors, one element per
// max(SB,SQ)^2 threads, and never stored in global memory. Nothing is scattered.
// ---------------------------------------------------------------------------
template <int SB, int SQ>
struct VjpShape {
  using S = Shape<SB, SQ>;
  static constexpr int SE = 2 * (S::S0 + 2 * S::S1 + 3 * S::S2);  // x and ybar buffers
  static constexpr int EPB = (128 / S::NL) > 0 ? (128 / S::NL) : 1;
  static constexpr int THREADS = EPB * S::NL;
};

// forward passes x/y of the element kernel: X -> (A1, B1) -> (AA, AB, BA)
template <int SB, int SQ, typename T>
__device__ __forceinline__ void forward_xy(const GenParams<SB, SQ, T>& P, const T* sMat, int l,
                                           const T* X, T* A1, T* B1, T* AA, T* AB, T* BA) {
  if (l < SB * SB) {
    T in[SB];
#pragma unroll
    for (int i = 0; i < SB; ++i) in[i] = X[l * SB + i];
#pragma unroll
    for (int qi = 0; qi < SQ; ++qi) {
      T a = T(0), b = T(0);
#pragma unroll
      for (int i = 0; i < SB; ++i) {
        a = fma(MA(qi * SB + i), in[i], a);
        b = fma(MB(qi * SB + i), in[i], b);
      }
      A1[l * SQ + qi] = a;
      B1[l * SQ + qi] = b;
    }
  }
  __syncthreads();
  if (l < SQ * SB) {
    const int qi = l % SQ, k = l / SQ;
    T a1[SB], b1[SB];
#pragma unroll
    for (int j = 0; j < SB; ++j) {
      a1[j] = A1[(k * SB + j) * SQ + qi];
      b1[j] = B1[(k * SB + j) * SQ + qi];
    }
#pragma unroll
    for (int qj = 0; qj < SQ; ++qj) {
      T aa = T(0), ab = T(0), ba = T(0);
#pragma unroll
      for (int j = 0; j < SB; ++j) {
        aa = fma(MA(qj * SB + j), a1[j], aa);
        ab = fma(MB(qj * SB + j), a1[j], ab);
        ba = fma(MA(qj * SB + j), b1[j], ba);
      }
      const int o = (k * SQ + qj) * SQ + qi;
      AA[o] = aa;
      AB[o] = ab;
      BA[o] = ba;
    }
  }
}

template <int SB, int SQ, typename T>
__global__ void __launch_bounds__(VjpShape<SB, SQ>::THREADS)
k_kappa_vjp(const __grid_constant__ GenParams<SB, SQ, T> P, const T* __restrict__ ybar,
            double* __restrict__ kbar) {
  using S = Shape<SB, SQ>;
  using V = VjpShape<SB, SQ>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int el = threadIdx.x / S::NL;
  const int l = threadIdx.x % S::NL;
  const long long cell = (long long)blockIdx.x * V::EPB + el;
  const bool valid = cell < P.ncells;
  T* base = reinterpret_cast<T*>(smem_raw) + (size_t)el * V::SE;
  T* buf[2][6];
#pragma unroll
  for (int v = 0; v < 2; ++v) {
    T* b = base + v * (V::SE / 2);
    buf[v][0] = b;                        // X
    buf[v][1] = b + S::S0;                // A1
    buf[v][2] = buf[v][1] + S::S1;        // B1
    buf[v][3] = buf[v][2] + S::S1;        // AA
    buf[v][4] = buf[v][3] + S::S2;        // AB
    buf[v][5] = buf[v][4] + S::S2;        // BA
  }
  __shared__ T sMat[kStageMats<T, SB, SQ> ? 2 * SQ * SB : 1];
  stage_mats<SB, SQ, T>(P, sMat);  // visible after the first __syncthreads below
  // gather x and ybar
  for (int pos = l; pos < S::S0; pos += S::NL) {
    T vx = T(0), vy = T(0);
    if (valid) {
      long long id;
      if (P.ids) id = P.ids[cell * S::S0 + pos];
      else id = structured_index(cell, pos, SB, P.nx, P.ny, P.nz);
      if (id >= 0) {
        vx = P.x[id];
        vy = ybar[id];
      }
    }
    buf[0][0][pos] = vx;
    buf[1][0][pos] = vy;
  }
  __syncthreads();
  forward_xy<SB, SQ, T>(P, sMat, l, buf[0][0], buf[0][1], buf[0][2], buf[0][3], buf[0][4],
                        buf[0][5]);
  forward_xy<SB, SQ, T>(P, sMat, l, buf[1][0], buf[1][1], buf[1][2], buf[1][3], buf[1][4],
                        buf[1][5]);
  __syncthreads();
  if (l < SQ * SQ && valid) {
    const int qi = l % SQ, qj = l / SQ;
    T c[2][3][SB];  // [vector][BA, AB, AA][k]
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int k = 0; k < SB; ++k) {
        const int o = (k * SQ + qj) * SQ + qi;
        c[v][0][k] = buf[v][5][o];
        c[v][1][k] = buf[v][4][o];
        c[v][2][k] = buf[v][3][o];
      }
#pragma unroll
    for (int qk = 0; qk < SQ; ++qk) {
      double g[2][3];
#pragma unroll
      for (int v = 0; v < 2; ++v) {
        T gx = T(0), gy = T(0), gz = T(0);
#pragma unroll
        for (int k = 0; k < SB; ++k) {
          gx = fma(MA(qk * SB + k), c[v][0][k], gx);
          gy = fma(MA(qk * SB + k), c[v][1][k], gy);
          gz = fma(MB(qk * SB + k), c[v][2][k], gz);
        }
        g[v][0] = (double)gx;
        g[v][1] = (double)gy;
        g[v][2] = (double)gz;
      }
      const int q = qi + SQ * (qj + SQ * qk);
      double G[6];
      if (P.geom == GEOM_SEPARABLE) {
        const double s = P.w1[qi] * P.w1[qj] * P.w1[qk];
#pragma unroll
        for (int m = 0; m < 6; ++m) G[m] = s * P.G0[m];
      } else {
        const double* gt = P.gtab + cell * P.gstride;
#pragma unroll
        for (int m = 0; m < 6; ++m) G[m] = gt[m * SQ * SQ * SQ + q];
      }
      const double* u = g[0];
      const double* w = g[1];
      const double gu0 = G[0] * u[0] + G[3] * u[1] + G[4] * u[2];
      const double gu1 = G[3] * u[0] + G[1] * u[1] + G[5] * u[2];
      const double gu2 = G[4] * u[0] + G[5] * u[1] + G[2] * u[2];
      kbar[cell * (SQ * SQ * SQ) + q] = w[0] * gu0 + w[1] * gu1 + w[2] * gu2;
    }
  }
}

// True when A[SQ-1-q][SB-1-i] = A[q][i] and B[SQ-1-q][SB-1-i] = -B[q][i] (nodes and
// quadrature points symmetric about the segment's midpoint, which holds for
// equispaced Lagrange nodes with Gauss points): the even-odd kernel applies.
bool centro_symmetric(const double* A, const double* B, int SB, int SQ) {
  double amax = 0.0, bmax = 0.0;
  for (int i = 0; i < SB * SQ; ++i) {
    amax = std::fmax(amax, std::fabs(A[i]));
    bmax = std::fmax(bmax, std::fabs(B[i]));
  }
  for (int q = 0; q < SQ; ++q)
    for (int i = 0; i < SB; ++i) {
      const int m = (SQ - 1 - q) * SB + (SB - 1 - i);
      if (std::fabs(A[m] - A[q * SB + i]) > 1e-13 * amax) return false;
      if (std::fabs(B[m] + B[q * SB + i]) > 1e-13 * bmax) return false;
    }
  return true;
}

template <int SB, int SQ, typename T>
GenParams<SB, SQ, T> make_params(const double* A, const double* B, const Geometry& geom) {
  GenParams<SB, SQ, T> P{};
  for (int i = 0; i < SQ * SB; ++i) {
    P.A[i] = (T)A[i];
    P.B[i] = (T)B[i];
  }
  // even-odd tables of A, B, A^T, B^T (see EOT)
  auto fill = [&](int op, int R, int C, auto m) {
    const int HR = (R + 1) / 2, HC = C / 2, MC = C % 2, W = 2 * HC + 2 * MC;
    T* t = P.eo + EOTables<SB, SQ>::OFF[op];
    for (int r = 0; r < HR; ++r) {
      for (int i = 0; i < HC; ++i) {
        t[r * W + 2 * i] = (T)(0.5 * (m(r, i) + m(r, C - 1 - i)));
        t[r * W + 2 * i + 1] = (T)(0.5 * (m(r, i) - m(r, C - 1 - i)));
      }
      if (MC) {
        t[r * W + 2 * HC] = (T)m(r, HC);
        t[r * W + 2 * HC + 1] = T(0);
      }
    }
  };
  fill(0, SQ, SB, [&](int r, int c) { return A[r * SB + c]; });
  fill(1, SQ, SB, [&](int r, int c) { return B[r * SB + c]; });
  fill(2, SB, SQ, [&](int r, int c) { return A[c * SB + r]; });
  fill(3, SB, SQ, [&](int r, int c) { return B[c * SB + r]; });
  for (int i = 0; i < SQ; ++i) P.w1[i] = geom.w1[i];
  for (int c = 0; c < 6; ++c) P.G0[c] = geom.G0[c];
  P.geom = geom.kind;
  P.gtab = geom.table;
  P.gstride = geom.table_stride;
  P.gtab32 = geom.table32;
  P.gstride32 = geom.table32_stride;
  P.kappa = geom.kappa;
  P.wdet = geom.wdet;
  P.wdet_stride = geom.wdet_stride;
  return P;
}

template <int SB, int SQ, typename T>
void run_general(int mode, const double* A, const double* B, const Cells& cells,
                 long long ncells, const int32_t* t2l, const Geometry& geom, const void* x,
                 void* y, cudaStream_t stream) {
  using S = Shape<SB, SQ>;
  auto P = make_params<SB, SQ, T>(A, B, geom);
  P.x = static_cast<const T*>(x);
  P.y = static_cast<T*>(y);
  P.ids = cells.ids;
  P.t2l = t2l;
  P.ncells = ncells;
  P.nx = cells.nx;
  P.ny = cells.ny;
  P.nz = cells.nz;
  P.mode = mode;
  if (ncells == 0) return;
  SF_REQUIRE(sizeof(T) == 8 || mode == 2 || geom.kind != GEOM_TABLE || geom.table32, SF_ERR_STATE,
             "internal: no FP32 copy of the geometry table");
  if (mode == 2) {
    const size_t smem = (size_t)S::EPB * DiagShape<SB, SQ>::WE * sizeof(double);
    const long long blocks = (ncells + S::EPB - 1) / S::EPB;
    SF_REQUIRE(blocks < (1LL << 31), SF_ERR_ARG, "too many cells for one launch");
    SF_CUDA_CHECK(cudaFuncSetAttribute(k_general_diag<SB, SQ, T>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_general_diag<SB, SQ, T><<<(unsigned)blocks, S::THREADS, smem, stream>>>(P);
    SF_CUDA_CHECK(cudaGetLastError());
    return;
  }
  const size_t smem = (size_t)S::EPB * S::SL * sizeof(T);
  const long long blocks = (ncells + S::EPB - 1) / S::EPB;
  SF_REQUIRE(blocks < (1LL << 31), SF_ERR_ARG, "too many cells for one launch");
  auto kern = centro_symmetric(A, B, SB, SQ) ? k_general<SB, SQ, T, true>
                                             : k_general<SB, SQ, T, false>;
  SF_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)blocks, S::THREADS, smem, stream>>>(P);
  SF_CUDA_CHECK(cudaGetLastError());
}

template <int SB, int SQ>
void run_rhs(const double* A, const double* B, const Cells& cells, const Geometry& geom,
             const double* fq, double* b, cudaStream_t stream) {
  using S = Shape<SB, SQ>;
  auto P = make_params<SB, SQ, double>(A, B, geom);
  P.x = fq;
  P.y = b;
  P.ids = cells.ids;
  P.ncells = cells.ncells;
  P.nx = cells.nx;
  P.ny = cells.ny;
  P.nz = cells.nz;
  if (cells.ncells == 0) return;
  SF_REQUIRE(geom.wdet, SF_ERR_STATE, "no point weights: call sf_set_cell_quantities first");
  const size_t smem = (size_t)S::EPB * S::SM3 * sizeof(double);
  const long long blocks = (cells.ncells + S::EPB - 1) / S::EPB;
  SF_REQUIRE(blocks < (1LL << 31), SF_ERR_ARG, "too many cells for one launch");
  auto kern = centro_symmetric(A, B, SB, SQ) ? k_rhs<SB, SQ, true> : k_rhs<SB, SQ, false>;
  SF_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)blocks, S::THREADS, smem, stream>>>(P);
  SF_CUDA_CHECK(cudaGetLastError());
}

using RhsFn = void (*)(const double*, const double*, const Cells&, const Geometry&, const double*,
                       double*, cudaStream_t);

RhsFn select_rhs(int SB, int SQ) {
#define SF_CASE(sb, sq) \
  if (SB == sb && SQ == sq) return &run_rhs<sb, sq>;
#define SF_ROW(sb) SF_CASE(sb, sb - 1) SF_CASE(sb, sb) SF_CASE(sb, sb + 1) SF_CASE(sb, sb + 2)
  SF_ROW(2) SF_ROW(3) SF_ROW(4) SF_ROW(5) SF_ROW(6) SF_ROW(7) SF_ROW(8)
  SF_CASE(9, 8) SF_CASE(9, 9) SF_CASE(9, 10)
  SF_CASE(10, 9) SF_CASE(10, 10)
#undef SF_ROW
#undef SF_CASE
  return nullptr;
}

using RunFn = void (*)(int, const double*, const double*, const Cells&, long long, const int32_t*,
                       const Geometry&, const void*, void*, cudaStream_t);

// Instantiated (SB, SQ) pairs: SB = 2..10, SQ in SB-1..SB+2 (1..10).
template <typename T>
RunFn select(int SB, int SQ) {
#define SF_CASE(sb, sq) \
  if (SB == sb && SQ == sq) return &run_general<sb, sq, T>;
#define SF_ROW(sb) SF_CASE(sb, sb - 1) SF_CASE(sb, sb) SF_CASE(sb, sb + 1) SF_CASE(sb, sb + 2)
  SF_ROW(2) SF_ROW(3) SF_ROW(4) SF_ROW(5) SF_ROW(6) SF_ROW(7) SF_ROW(8)
  SF_CASE(9, 8) SF_CASE(9, 9) SF_CASE(9, 10)
  SF_CASE(10, 9) SF_CASE(10, 10)
#undef SF_ROW
#undef SF_CASE
  return nullptr;
}

RunFn select_dtype(int dtype, int SB, int SQ) {
  RunFn f = nullptr;
  if (dtype == SF_F64) f = select<double>(SB, SQ);
  else if (dtype == SF_F32) f = select<float>(SB, SQ);
  else throw Error(SF_ERR_ARG, "dtype must be SF_F64 or SF_F32");
  if (!f)
    throw Error(SF_ERR_UNSUPPORTED, "no general kernel instantiated for SB=" + std::to_string(SB) +
                                        " SQ=" + std::to_string(SQ));
  return f;
}

template <int SB, int SQ, typename T>
void run_vjp(const double* A, const double* B, const Cells& cells, const Geometry& geom,
             const void* x, const void* ybar, double* kbar, cudaStream_t stream) {
  using V = VjpShape<SB, SQ>;
  auto P = make_params<SB, SQ, T>(A, B, geom);
  P.x = static_cast<const T*>(x);
  P.ids = cells.ids;
  P.ncells = cells.ncells;
  P.nx = cells.nx;
  P.ny = cells.ny;
  P.nz = cells.nz;
  if (cells.ncells == 0) return;
  const size_t smem = (size_t)V::EPB * V::SE * sizeof(T);
  SF_CUDA_CHECK(cudaFuncSetAttribute(k_kappa_vjp<SB, SQ, T>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const long long blocks = (cells.ncells + V::EPB - 1) / V::EPB;
  SF_REQUIRE(blocks < (1LL << 31), SF_ERR_ARG, "too many cells for one launch");
  k_kappa_vjp<SB, SQ, T><<<(unsigned)blocks, V::THREADS, smem, stream>>>(
      P, static_cast<const T*>(ybar), kbar);
  SF_CUDA_CHECK(cudaGetLastError());
}

using VjpFn = void (*)(const double*, const double*, const Cells&, const Geometry&, const void*,
                       const void*, double*, cudaStream_t);

template <typename T>
VjpFn select_vjp(int SB, int SQ) {
#define SF_CASE(sb, sq) \
  if (SB == sb && SQ == sq) return &run_vjp<sb, sq, T>;
#define SF_ROW(sb) SF_CASE(sb, sb - 1) SF_CASE(sb, sb) SF_CASE(sb, sb + 1) SF_CASE(sb, sb + 2)
  SF_ROW(2) SF_ROW(3) SF_ROW(4) SF_ROW(5) SF_ROW(6) SF_ROW(7) SF_ROW(8)
  SF_CASE(9, 8) SF_CASE(9, 9) SF_CASE(9, 10)
  SF_CASE(10, 9) SF_CASE(10, 10)
#undef SF_ROW
#undef SF_CASE
  return nullptr;
}

}  // namespace

void launch_kappa_vjp(int dtype, int SB, int SQ, const double* A, const double* B,
                      const Cells& cells, const Geometry& geom, const void* x, const void* ybar,
                      double* kbar, cudaStream_t stream) {
  VjpFn f = nullptr;
  if (dtype == SF_F64) f = select_vjp<double>(SB, SQ);
  else if (dtype == SF_F32) f = select_vjp<float>(SB, SQ);
  else throw Error(SF_ERR_ARG, "dtype must be SF_F64 or SF_F32");
  if (!f) throw Error(SF_ERR_UNSUPPORTED, "no adjoint kernel for this SB/SQ");
  f(A, B, cells, geom, x, ybar, kbar, stream);
}

__global__ void k_table32(const double* __restrict__ src, long long total, int per,
                          long long dst_stride, float* __restrict__ dst) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / per;
    dst[c * dst_stride + (i - c * per)] = (float)src[i];
  }
}

void convert_table32(const double* src, long long ncopy, int per, long long dst_stride, float* dst,
                     cudaStream_t stream) {
  const long long total = ncopy * per;
  if (total == 0) return;
  const long long blocks = std::min<long long>((total + 255) / 256, 148LL * 16);
  k_table32<<<(unsigned)blocks, 256, 0, stream>>>(src, total, per, dst_stride, dst);
  SF_CUDA_CHECK(cudaGetLastError());
}

void launch_general_apply(int dtype, int SB, int SQ, const double* A, const double* B,
                          const Cells& cells, const Geometry& geom, const void* x, void* y,
                          cudaStream_t stream) {
  select_dtype(dtype, SB, SQ)(0, A, B, cells, cells.ncells, nullptr, geom, x, y, stream);
}

void launch_general_diag(int dtype, int SB, int SQ, const double* A, const double* B,
                         const Cells& cells, const Geometry& geom, void* d, cudaStream_t stream) {
  select_dtype(dtype, SB, SQ)(2, A, B, cells, cells.ncells, nullptr, geom, nullptr, d, stream);
}

void launch_general_rhs(int SB, int SQ, const double* A, const double* B, const Cells& cells,
                        const Geometry& geom, const double* fq, double* b, cudaStream_t stream) {
  RhsFn f = select_rhs(SB, SQ);
  if (!f)
    throw Error(SF_ERR_UNSUPPORTED, "no right-hand-side kernel for SB=" + std::to_string(SB) +
                                        " SQ=" + std::to_string(SQ));
  f(A, B, cells, geom, fq, b, stream);
}

void launch_general_evaluate(int dtype, int SB, int SQ, const double* A, const double* B,
                             long long ncells, const int32_t* t2l, const Geometry& geom,
                             const void* x_cells, void* y_cells, cudaStream_t stream) {
  Cells none;
  select_dtype(dtype, SB, SQ)(1, A, B, none, ncells, t2l, geom, x_cells, y_cells, stream);
}

}  // namespace sf
