// Tiled Cartesian kernels: constant-coefficient, axis-aligned affine cells on
// a structured mesh. This is the fast path of LazyMatrix mul!
// (src/LazyMatrices.jl:52-61) for the Cartesian meshes that every
// reference driver builds (profiling/drivers.jl:7-10).
//
// Algebra. On such a cell the metric is G(q) = w_q * diag(cx, cy, cz), with w_q
// the product of 1D weights (the structured_mesh_opt case of the reference's
// flop model, src/Utils.jl:33-72). Then the element operator
// sum_r B_r^T G B_r of src/SumFactorizationKernels.jl:40-216 equals, exactly,
//     cx K(x) M(y) M(z) + cy M(x) K(y) M(z) + cz M(x) M(y) K(z),
// where M = A0^T W A0 and K = B0^T W B0 are the 1D element matrices with the
// quadrature already summed. Assembled over a line of cells the structure
// stays, with M and K assembled along the line:
//     t1 = M_z x,  t2 = (cz/cy) K_z x,                       (z pass)
//     a = (cx/cy) M_y t1,  s = K_y t1 + M_y t2,              (y pass)
//     y = cy (K_x a + M_x s).                                (x pass)
// This is the same operator up to rounding; the parity tests hold it to 1e-12.
//
// Even-odd form. With equispaced nodes in ascending order and a symmetric
// Gauss rule, M and K are symmetric and centro-symmetric
// (M[P-i][P-j] = M[i][j]). One cell's 1D product y = M u then splits into an
// even part (ceil(S/2) square) acting on u_j + u_{P-j} and an odd part
// (floor(S/2) square) acting on u_j - u_{P-j}, and both parts are symmetric.
// For P = 4 this takes 21 FP64 operations instead of 25, and 2 x 9 unique
// constants hold both operators. FP64 FMAs cannot take their operand from the
// constant bank, so those 18 constants live in registers for the whole kernel.
//
// Work decomposition. A CTA owns a box of OUTPUT dofs covering EX x EY x EZ
// cells: the points (e0 p, (e0+E) p] in each direction. Nothing is scattered,
// so no atomics and no zeroing of y are needed, and the result is
// deterministic. The z pass reads x straight from global memory into
// registers, one z-line per thread, including a one-cell halo in x and y;
// Dirichlet and out-of-mesh points read as zero. t1/t2 go to shared memory.
// The y and x passes run one thread per line in shared memory, streaming cell
// by cell and carrying the vertex shared by neighbouring cells. The output box
// is written back coalesced.
#include "sf_cartesian.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace sf {
namespace {

template <int P>
struct EO {
  static constexpr int S = P + 1;
  static constexpr int H = S / 2;           // mirrored pairs (j, P-j)
  static constexpr bool MID = (S % 2) == 1; // a middle node j = H
  static constexpr int NE = H + (MID ? 1 : 0);
  static constexpr int NO = H;
  static constexpr int UE = NE * (NE + 1) / 2;  // unique entries (upper triangle)
  static constexpr int UO = NO * (NO + 1) / 2;
};

__host__ __device__ constexpr int tri(int i, int j, int n) {
  // packed upper-triangular index of the symmetric pair (i, j), 0 <= i, j < n
  return i <= j ? i * n - i * (i - 1) / 2 + (j - i) : j * n - j * (j - 1) / 2 + (i - j);
}

// A Chebyshev smoothing step fused into the store phase of an apply of z (the
// kernel's input x): with az = (A z) at an owned point,
//   d = c2 dinv (r - az) (mode 1) or c1 d + c2 dinv (r - az) (mode 2),  z_out = z + d.
// z_out must not be z (other tiles still read z's halo).
template <typename T>
struct ChebEpi {
  const T* r;
  const T* dinv;
  T* d;
  T* z_out;
  T c1, c2;
  int mode;  // 0: a plain apply
};

template <int P, typename T>
struct CartParams {
  T Me[EO<P>::UE], Mo[EO<P>::UO];  // even / odd parts of M
  T Ke[EO<P>::UE], Ko[EO<P>::UO];  // even / odd parts of K
  T rz, rx, cy;                    // cz/cy, cx/cy, cy
  const T* x;
  T* y;
  int nfx, nfy, nfz;  // free grid (inputs are read for z in [zlo, nfz))
  int zlo, nfz_out;   // lowest input z (-1 on a slab: the halo plane below); outputs z < nfz_out
  int ntx, nty, ntz;  // tiles
  int tile0;          // first tile of the launch (CTA b applies tile tile0 + b)
  double* dot;  // non-null: dot[tile] = sum of x*y over the tile's outputs
  const int32_t* num;  // numbered kernel: the vectors' index of each lexicographic free point
  ChebEpi<T> cheb;     // CHEB kernel: the fused Chebyshev step
};

// FP64 sum over the CTA, valid in thread 0 (adds warps in a fixed order).
template <int NT>
__device__ __forceinline__ double cta_sum(double v) {
  __shared__ double red[NT / 32];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) t += red[w];
  }
  return t;
}

// Even/odd parts of one operator, held in registers (symmetric entries share one register).
template <int P, typename T>
struct EOMat {
  using S = EO<P>;
  T e[S::NE][S::NE];
  T o[S::NO > 0 ? S::NO : 1][S::NO > 0 ? S::NO : 1];
  __device__ __forceinline__ void load(const T* ue, const T* uo) {
#pragma unroll
    for (int i = 0; i < S::NE; ++i)
#pragma unroll
      for (int j = i; j < S::NE; ++j) {
        const T v = ue[tri(i, j, S::NE)];
        e[i][j] = v;
        e[j][i] = v;
      }
#pragma unroll
    for (int i = 0; i < S::NO; ++i)
#pragma unroll
      for (int j = i; j < S::NO; ++j) {
        const T v = uo[tri(i, j, S::NO)];
        o[i][j] = v;
        o[j][i] = v;
      }
  }
};

template <int P, typename T>
struct Split {  // u_j + u_{P-j} (and the middle node) / u_j - u_{P-j}
  T e[EO<P>::NE];
  T o[EO<P>::NO > 0 ? EO<P>::NO : 1];
};

template <int P, typename T>
__device__ __forceinline__ Split<P, T> split(const T (&u)[P + 1]) {
  using S = EO<P>;
  Split<P, T> s;
#pragma unroll
  for (int j = 0; j < S::H; ++j) {
    s.e[j] = u[j] + u[P - j];
    s.o[j] = u[j] - u[P - j];
  }
  if constexpr (S::MID) s.e[S::H] = u[S::H];
  return s;
}

// (ye, yo) += (E e, O o)
template <int P, typename T>
__device__ __forceinline__ void mac(const EOMat<P, T>& A, const Split<P, T>& s, T (&ye)[EO<P>::NE],
                                   T (&yo)[EO<P>::NO > 0 ? EO<P>::NO : 1]) {
  using S = EO<P>;
#pragma unroll
  for (int i = 0; i < S::NE; ++i)
#pragma unroll
    for (int j = 0; j < S::NE; ++j) ye[i] = fma(A.e[i][j], s.e[j], ye[i]);
#pragma unroll
  for (int i = 0; i < S::NO; ++i)
#pragma unroll
    for (int j = 0; j < S::NO; ++j) yo[i] = fma(A.o[i][j], s.o[j], yo[i]);
}

// row 0 only: E[0] . e + O[0] . o
template <int P, typename T>
__device__ __forceinline__ T mac_row0(const EOMat<P, T>& A, const Split<P, T>& s, T acc) {
  using S = EO<P>;
#pragma unroll
  for (int j = 0; j < S::NE; ++j) acc = fma(A.e[0][j], s.e[j], acc);
#pragma unroll
  for (int j = 0; j < S::NO; ++j) acc = fma(A.o[0][j], s.o[j], acc);
  return acc;
}

template <int P, typename T>
struct Acc {  // even/odd accumulators of one output line
  T e[EO<P>::NE];
  T o[EO<P>::NO > 0 ? EO<P>::NO : 1];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int i = 0; i < EO<P>::NE; ++i) e[i] = T(0);
#pragma unroll
    for (int i = 0; i < EO<P>::NO; ++i) o[i] = T(0);
  }
  // value at local node l
  __device__ __forceinline__ T at(int l) const {
    using S = EO<P>;
    if (S::MID && l == S::H) return e[S::H];
    if (l < S::H) return e[l] + o[l];
    return e[P - l] - o[P - l];
  }
};

template <int P, int EX, int EY, int EZ, typename T>
struct Tile {
  static constexpr int BX = (EX + 1) * P + 1, BY = (EY + 1) * P + 1, BZ = (EZ + 1) * P + 1;
  static constexpr int OX = EX * P, OY = EY * P, OZ = EZ * P;
  // Plane stride padded so that PLANE = BX (mod M), M = words per bank sweep (16
  // doubles / 32 floats). The y pass gives consecutive lanes consecutive x, and a
  // request that wraps from one z-plane into the next then maps onto the banks as
  // if the rows were contiguous, so it has no bank conflicts.
  static constexpr int M = sizeof(T) == 8 ? 16 : 32;
  // Rows inside a plane have an odd pitch RX: the x pass gives consecutive threads
  // consecutive rows, and an even pitch (BX = 16 at p = 3 or 5 with small tiles)
  // would put their accesses on the same banks.
  static constexpr int RX = BX | 1;
  static constexpr int PAD = ((BX - RX * BY) % M + M) % M;
  static constexpr int PLANE = RX * BY + PAD;
  static constexpr int TS = PLANE * OZ;  // each of t1 (-> a -> y) and t2 (-> s)
  static constexpr int WORDS = 2 * TS;
};

// Generic streaming pass over a line of E+1 cells held in shared memory.
// NIN input lines (stride `st`), NOUT output lines written in place over the
// inputs at index (o-1)*st for the owned points o = 1..E*P. `body` forms the
// even/odd accumulators of every output from the split inputs; `row0` forms
// only the node-0 values (last cell).
template <int P, int E, int NIN, int NOUT, typename T, typename Body, typename Row0, typename Fin>
__device__ __forceinline__ void smem_line(T* const (&ln)[2], int st, const Body& body,
                                          const Row0& row0, const Fin& fin) {
  T u[NIN][P + 1];
  T un[NIN][P];  // next cell's nodes 1..P, loaded while the current cell computes
  T carry[NOUT];
#pragma unroll
  for (int j = 0; j < NOUT; ++j) carry[j] = T(0);
#pragma unroll
  for (int i = 0; i < NIN; ++i)
#pragma unroll
    for (int l = 0; l <= P; ++l) u[i][l] = ln[i][l * st];
#pragma unroll(sizeof(T) == 8 ? E : 1)  // FP64: unrolled, no register shuffles between cells
  for (int k = 0; k < E; ++k) {
    // prefetch: cell k+1 reads (k+1)P+1..(k+1)P+P, above every index cell k writes
#pragma unroll
    for (int i = 0; i < NIN; ++i)
#pragma unroll
      for (int l = 1; l <= P; ++l) un[i][l - 1] = ln[i][((k + 1) * P + l) * st];
    Split<P, T> s[NIN];
#pragma unroll
    for (int i = 0; i < NIN; ++i) s[i] = split<P, T>(u[i]);
    Acc<P, T> acc[NOUT];
#pragma unroll
    for (int j = 0; j < NOUT; ++j) acc[j].zero();
    body(s, acc);
#pragma unroll
    for (int j = 0; j < NOUT; ++j) {
      if (k > 0) ln[j][(k * P - 1) * st] = fin(j, acc[j].at(0) + carry[j]);
#pragma unroll
      for (int l = 1; l < P; ++l) ln[j][(k * P + l - 1) * st] = fin(j, acc[j].at(l));
      carry[j] = acc[j].at(P);
    }
#pragma unroll
    for (int i = 0; i < NIN; ++i) {
      u[i][0] = u[i][P];
#pragma unroll
      for (int l = 1; l <= P; ++l) u[i][l] = un[i][l - 1];
    }
  }
  // last cell: node 0 only (the end point E*P); its inputs are already in u
  Split<P, T> s[NIN];
#pragma unroll
  for (int i = 0; i < NIN; ++i) s[i] = split<P, T>(u[i]);
  T r[NOUT];
  row0(s, r);
#pragma unroll
  for (int j = 0; j < NOUT; ++j) ln[j][(E * P - 1) * st] = fin(j, r[j] + carry[j]);
}

// The three line passes of one tile. load_col(l, c) fills c with input z-column
// l of the tile's input box (x = l % BX, y = l / BX; points 0 .. BZ-1 along z).
// On return T1 holds the tile's outputs (plane stride PLANE, row pitch RX) and
// every thread has passed a barrier after the last pass. PAIR: when the box has
// between NT and 2 NT columns, a thread loads both of its columns before it
// computes either.
template <int P, int EX, int EY, int EZ, int NT, bool ISO, bool PAIR, typename T, typename Load>
__device__ __forceinline__ void tile_passes(T* T1, T* T2, const EOMat<P, T>& Mm,
                                            const EOMat<P, T>& Km, T rz, T rx, T cy,
                                            const Load& load_col) {
  using G = Tile<P, EX, EY, EZ, T>;
  // ---- z pass: one z-line per thread, inputs from load_col ----
  auto z_line = [&](int l, const T (&c)[G::BZ]) {
    const int sl = G::RX == G::BX ? l : (l % G::BX) + G::RX * (l / G::BX);  // in-plane offset
    T cm = T(0), ck = T(0);
#pragma unroll
    for (int k = 0; k < EZ; ++k) {
      T u[P + 1];
#pragma unroll
      for (int m = 0; m <= P; ++m) u[m] = c[k * P + m];
      const Split<P, T> s = split<P, T>(u);
      Acc<P, T> am, ak;
      am.zero();
      ak.zero();
      mac<P, T>(Mm, s, am.e, am.o);
      mac<P, T>(Km, s, ak.e, ak.o);
      if (k > 0) {
        T1[(k * P - 1) * G::PLANE + sl] = am.at(0) + cm;
        const T v = ak.at(0) + ck;
        T2[(k * P - 1) * G::PLANE + sl] = ISO ? v : v * rz;
      }
#pragma unroll
      for (int m = 1; m < P; ++m) {
        T1[(k * P + m - 1) * G::PLANE + sl] = am.at(m);
        const T v = ak.at(m);
        T2[(k * P + m - 1) * G::PLANE + sl] = ISO ? v : v * rz;
      }
      cm = am.at(P);
      ck = ak.at(P);
    }
    T u[P + 1];
#pragma unroll
    for (int m = 0; m <= P; ++m) u[m] = c[EZ * P + m];
    const Split<P, T> s = split<P, T>(u);
    T1[(EZ * P - 1) * G::PLANE + sl] = mac_row0<P, T>(Mm, s, cm);
    const T v = mac_row0<P, T>(Km, s, ck);
    T2[(EZ * P - 1) * G::PLANE + sl] = ISO ? v : v * rz;
  };
  constexpr int ZL = G::BX * G::BY;
  if constexpr (PAIR && ZL > NT && ZL <= 2 * NT) {
    // two z-lines per thread: both columns' loads are in flight before either computes
    const int l0 = threadIdx.x, l1 = threadIdx.x + NT;
    T c0[G::BZ], c1[G::BZ];
    load_col(l0, c0);
    if (l1 < ZL) load_col(l1, c1);
    z_line(l0, c0);
    if (l1 < ZL) z_line(l1, c1);
  } else {
    for (int l = threadIdx.x; l < ZL; l += NT) {
      T c[G::BZ];
      load_col(l, c);
      z_line(l, c);
    }
  }
  __syncthreads();

  // ---- y pass: lines (x, zo): a = rx M t1 -> T1, s = K t1 + M t2 -> T2 ----
  for (int l = threadIdx.x; l < G::BX * G::OZ; l += NT) {
    const int x = l % G::BX, zo = l / G::BX;
    T* const ln[2] = {T1 + zo * G::PLANE + x, T2 + zo * G::PLANE + x};
    smem_line<P, EY, 2, 2, T>(
        ln, G::RX,
        [&](const Split<P, T>(&s)[2], Acc<P, T>(&acc)[2]) {
          mac<P, T>(Mm, s[0], acc[0].e, acc[0].o);
          mac<P, T>(Km, s[0], acc[1].e, acc[1].o);
          mac<P, T>(Mm, s[1], acc[1].e, acc[1].o);
        },
        [&](const Split<P, T>(&s)[2], T(&r)[2]) {
          r[0] = mac_row0<P, T>(Mm, s[0], T(0));
          r[1] = mac_row0<P, T>(Mm, s[1], mac_row0<P, T>(Km, s[0], T(0)));
        },
        [&](int j, T v) { return (ISO || j == 1) ? v : v * rx; });
  }
  __syncthreads();

  // ---- x pass: lines (yo, zo): y = cy (K a + M s) -> T1 ----
  for (int l = threadIdx.x; l < G::OY * G::OZ; l += NT) {
    const int yo = l % G::OY, zo = l / G::OY;
    T* const ln[2] = {T1 + zo * G::PLANE + yo * G::RX, T2 + zo * G::PLANE + yo * G::RX};
    smem_line<P, EX, 2, 1, T>(
        ln, 1,
        [&](const Split<P, T>(&s)[2], Acc<P, T>(&acc)[1]) {
          mac<P, T>(Km, s[0], acc[0].e, acc[0].o);
          mac<P, T>(Mm, s[1], acc[0].e, acc[0].o);
        },
        [&](const Split<P, T>(&s)[2], T(&r)[1]) {
          r[0] = mac_row0<P, T>(Mm, s[1], mac_row0<P, T>(Km, s[0], T(0)));
        },
        [&](int, T v) { return v * cy; });
  }
  __syncthreads();
}

// One output tile: cells [tx*EX, (tx+1)*EX) x [ty*EY, ...) x [tz*EZ, ...) of a free grid
// nfx x nfy x nfz. Inputs outside the free grid read as zero, except that the
// z range read is [zlo, nfz) (zlo = -1: a slab's halo plane below it); outputs
// are written for z < nfz_out. T1/T2: shared buffers of Tile::TS words each. Ends with the
// outputs stored; the caller synchronises before reusing T1/T2. With `dot`
// non-null, *dot receives the FP64 sum of x*y over the tile's outputs (the
// (p, A p) term of CG), summed in a fixed order. With PS non-null the z pass
// keeps the x values of the owned points in PS (OX*OY*OZ shared words,
// [zo][yo][xo]) for that sum, so they are not read from global memory a second
// time; without it they are re-read. NUM: x and y are in another numbering of
// the free points, num[i] being the index of lexicographic point i; x is read
// as x[num[i]] and y written as y[num[i]] (no (x, y) sum then).
template <int P, int EX, int EY, int EZ, int NT, bool ISO, typename T, bool NUM = false,
          bool CHEB = false>
__device__ __forceinline__ void cart_tile(T* T1, T* T2, const EOMat<P, T>& Mm,
                                          const EOMat<P, T>& Km, const T* __restrict__ X,
                                          T* __restrict__ Y, int nfx, int nfy, int nfz, int zlo,
                                          int nfz_out, int tx,
                                          int ty, int tz, T rz, T rx, T cy,
                                          double* dot = nullptr, T* PS = nullptr,
                                          const int32_t* __restrict__ num = nullptr,
                                          const ChebEpi<T>* cheb = nullptr) {
  using G = Tile<P, EX, EY, EZ, T>;
  // free coordinate of the first input point (grid point e0*p has free index e0*p - 1)
  const int fx0 = tx * EX * P - 1, fy0 = ty * EY * P - 1, fz0 = tz * EZ * P - 1;
  const long long pz = (long long)nfx * nfy;

  // a tile whose whole input box lies inside the free grid needs no bounds checks
  const bool interior = fx0 >= 0 && fy0 >= 0 && fz0 >= zlo && fx0 + G::BX <= nfx &&
                        fy0 + G::BY <= nfy && fz0 + G::BZ <= nfz;

  auto load_col = [&](int l, T (&c)[G::BZ]) {
    const int x = l % G::BX, y = l / G::BX;
    const int fx = fx0 + x, fy = fy0 + y;
    if constexpr (NUM) {
      const bool inxy = (unsigned)fx < (unsigned)nfx && (unsigned)fy < (unsigned)nfy;
      const long long ci = (long long)fx + (long long)nfx * fy;
      int32_t k[G::BZ];
#pragma unroll
      for (int z = 0; z < G::BZ; ++z) {
        const int fz = fz0 + z;
        const bool in = interior || (inxy && (unsigned)(fz - zlo) < (unsigned)(nfz - zlo));
        k[z] = in ? __ldg(num + ci + fz * pz) : -1;
      }
#pragma unroll
      for (int z = 0; z < G::BZ; ++z) c[z] = k[z] >= 0 ? __ldg(X + k[z]) : T(0);
    } else if (interior) {
      const T* col = X + (long long)fx + (long long)nfx * fy + fz0 * pz;
#pragma unroll
      for (int z = 0; z < G::BZ; ++z) c[z] = __ldg(col + z * pz);
    } else {
      const bool inxy = (unsigned)fx < (unsigned)nfx && (unsigned)fy < (unsigned)nfy;
      const T* col = X + (long long)fx + (long long)nfx * fy;
#pragma unroll
      for (int z = 0; z < G::BZ; ++z) {
        const int fz = fz0 + z;
        c[z] = (inxy && (unsigned)(fz - zlo) < (unsigned)(nfz - zlo)) ? __ldg(col + fz * pz) : T(0);
      }
    }
    if (PS && x >= 1 && x <= G::OX && y >= 1 && y <= G::OY) {
#pragma unroll
      for (int z = 1; z <= G::OZ; ++z) PS[((z - 1) * G::OY + (y - 1)) * G::OX + (x - 1)] = c[z];
    }
  };
  tile_passes<P, EX, EY, EZ, NT, ISO, true, T>(T1, T2, Mm, Km, rz, rx, cy, load_col);

  // ---- store the owned outputs (free coords start at e0*p) ----
  const int ox0 = fx0 + 1, oy0 = fy0 + 1, oz0 = fz0 + 1;
  const bool full = ox0 + G::OX <= nfx && oy0 + G::OY <= nfy && oz0 + G::OZ <= nfz_out;
  const long long base = (long long)ox0 + (long long)nfx * (oy0 + (long long)nfy * oz0);
  T* ybase = Y + base;
  constexpr int NOUT = G::OX * G::OY * G::OZ;
  auto out_index = [&](int i, long long& o, int& t1) {  // false outside the free grid
    const int xo = i % G::OX;
    const int r = i / G::OX;
    const int yo = r % G::OY;
    const int zo = r / G::OY;
    o = xo + (long long)nfx * (yo + (long long)nfy * zo);
    t1 = zo * G::PLANE + yo * G::RX + xo;
    return full || (ox0 + xo < nfx && oy0 + yo < nfy && oz0 + zo < nfz_out);
  };
  if constexpr (CHEB) {  // the Chebyshev step: all loads of a thread first, then the stores
    constexpr int PER = (NOUT + NT - 1) / NT;
    constexpr int CH = PER < 4 ? PER : 4;
    const ChebEpi<T>& E = *cheb;
#pragma unroll
    for (int k0 = 0; k0 < PER; k0 += CH) {
      T rv[CH], dv[CH], zv[CH], av[CH];
      long long gv[CH];
      bool ok[CH];
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        const int i = threadIdx.x + (k0 + j) * NT;
        long long o;
        int t1;
        ok[j] = k0 + j < PER && i < NOUT && out_index(i, o, t1);
        gv[j] = base + (ok[j] ? o : 0);
        rv[j] = ok[j] ? __ldg(E.r + gv[j]) - T1[t1] : T(0);
        av[j] = ok[j] ? __ldg(E.dinv + gv[j]) : T(0);
        dv[j] = ok[j] && E.mode == 2 ? E.d[gv[j]] : T(0);
        zv[j] = ok[j] ? __ldg(X + gv[j]) : T(0);
      }
#pragma unroll
      for (int j = 0; j < CH; ++j) {
        if (!ok[j]) continue;
        const T v = fma(E.c1, dv[j], E.c2 * av[j] * rv[j]);
        E.d[gv[j]] = v;
        E.z_out[gv[j]] = zv[j] + v;
      }
    }
    return;
  }
  if (!dot) {
    for (int i = threadIdx.x; i < NOUT; i += NT) {
      long long o;
      int t1;
      if (out_index(i, o, t1)) {
        if constexpr (NUM) Y[__ldg(num + base + o)] = T1[t1];
        else ybase[o] = T1[t1];
      }
    }
    return;
  }
  // with the (x, y) sum: every x value of this thread is requested before any is used
  constexpr int PER = (NOUT + NT - 1) / NT;
  T xv[PER];
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int i = threadIdx.x + k * NT;
    long long o;
    int t1;
    // PS was written before the passes' barriers
    xv[k] = (i < NOUT && out_index(i, o, t1)) ? (PS ? PS[i] : __ldg(X + base + o)) : T(0);
  }
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < PER; ++k) {
    const int i = threadIdx.x + k * NT;
    long long o;
    int t1;
    if (i < NOUT && out_index(i, o, t1)) {
      const T v = T1[t1];
      ybase[o] = v;
      acc = fma((double)xv[k], (double)v, acc);
    }
  }
  const double t = cta_sum<NT>(acc);  // the same branch in every thread of the CTA
  if (threadIdx.x == 0) *dot = t;
}


// ---------------------------------------------------------------------------
// 2D (quadrilateral Q_p) tiled apply on an nx x ny Cartesian mesh:
//   y = cx Kx(x)My + cy Mx(x)Ky  (K along the first factor's axis),
// the 2D form of the Kronecker identity above (the domain of the reference's
// own 2D GPU kernels, src/GPUKernels.jl). A CTA owns EX x EY cells and
// recomputes a one-cell halo; nothing is scattered.
//   pass 1: y-line segments of CY cells straight from global memory into
//           registers: t1 = My x -> T1, t2 = Ky x -> T2 (owned rows, all columns);
//   pass 2: x-line segments of CX cells: every thread first loads its t1, t2
//           segment into registers, then (after a barrier) writes
//           cx Kx t1 + cy Mx t2 over its own owned points of T1;
//   store:  the owned box of T1 back to global memory, coalesced.
// ---------------------------------------------------------------------------
template <int P, typename T>
struct CartParams2 {
  T Me[EO<P>::UE], Mo[EO<P>::UO];
  T Ke[EO<P>::UE], Ko[EO<P>::UO];
  T cx, cy;
  const T* x;
  T* y;
  int nfx, nfy;  // free grid
  int ntx, nty;  // tiles
};

template <int P, int EX, int EY>
struct Tile2 {
  static constexpr int BX = (EX + 1) * P + 1, BY = (EY + 1) * P + 1;
  static constexpr int OX = EX * P, OY = EY * P;
  static constexpr int PX = BX | 1;  // odd pitch: threads on different rows hit different banks
  static constexpr int TS = OY * PX;
  static constexpr int WORDS = 2 * TS;
};

// One segment of E cells of a line in registers (c[0 .. E*P+P]): out(o, M c, K c) for the
// segment's outputs o = 0 .. E*P-1 (line points 1 .. E*P).
template <int P, int E, typename T, typename Out>
__device__ __forceinline__ void seg_mk(const EOMat<P, T>& Mm, const EOMat<P, T>& Km,
                                       const T (&c)[E * P + P + 1], const Out& out) {
  T cm = T(0), ck = T(0);
#pragma unroll
  for (int k = 0; k < E; ++k) {
    T u[P + 1];
#pragma unroll
    for (int m = 0; m <= P; ++m) u[m] = c[k * P + m];
    const Split<P, T> s = split<P, T>(u);
    Acc<P, T> am, ak;
    am.zero();
    ak.zero();
    mac<P, T>(Mm, s, am.e, am.o);
    mac<P, T>(Km, s, ak.e, ak.o);
    if (k > 0) out(k * P - 1, am.at(0) + cm, ak.at(0) + ck);
#pragma unroll
    for (int m = 1; m < P; ++m) out(k * P + m - 1, am.at(m), ak.at(m));
    cm = am.at(P);
    ck = ak.at(P);
  }
  T u[P + 1];
#pragma unroll
  for (int m = 0; m <= P; ++m) u[m] = c[E * P + m];
  const Split<P, T> s = split<P, T>(u);
  out(E * P - 1, mac_row0<P, T>(Mm, s, cm), mac_row0<P, T>(Km, s, ck));
}

// out(o, K a + M b) over a segment of E cells held in registers.
template <int P, int E, typename T, typename Out>
__device__ __forceinline__ void seg_kamb(const EOMat<P, T>& Km, const EOMat<P, T>& Mm,
                                         const T (&a)[E * P + P + 1], const T (&b)[E * P + P + 1],
                                         const Out& out) {
  T carry = T(0);
#pragma unroll
  for (int k = 0; k < E; ++k) {
    T ua[P + 1], ub[P + 1];
#pragma unroll
    for (int m = 0; m <= P; ++m) {
      ua[m] = a[k * P + m];
      ub[m] = b[k * P + m];
    }
    const Split<P, T> sa = split<P, T>(ua), sb = split<P, T>(ub);
    Acc<P, T> acc;
    acc.zero();
    mac<P, T>(Km, sa, acc.e, acc.o);
    mac<P, T>(Mm, sb, acc.e, acc.o);
    if (k > 0) out(k * P - 1, acc.at(0) + carry);
#pragma unroll
    for (int m = 1; m < P; ++m) out(k * P + m - 1, acc.at(m));
    carry = acc.at(P);
  }
  T ua[P + 1], ub[P + 1];
#pragma unroll
  for (int m = 0; m <= P; ++m) {
    ua[m] = a[E * P + m];
    ub[m] = b[E * P + m];
  }
  const Split<P, T> sa = split<P, T>(ua), sb = split<P, T>(ub);
  out(E * P - 1, mac_row0<P, T>(Mm, sb, mac_row0<P, T>(Km, sa, carry)));
}

template <int P, int EX, int EY, int CX, int CY, int NT, bool ISO, typename T, int MINB>
__global__ void __launch_bounds__(NT, MINB)
k_cartesian2d(const __grid_constant__ CartParams2<P, T> Q) {
  using G = Tile2<P, EX, EY>;
  constexpr int SY = EY / CY, NY = CY * P + P + 1;
  constexpr int SX = EX / CX, NX = CX * P + P + 1;
  static_assert(EY % CY == 0 && EX % CX == 0, "segments must divide the tile");
  static_assert(G::OY * SX <= NT, "pass 2 holds one segment per thread");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* T1 = reinterpret_cast<T*>(smem_raw);
  T* T2 = T1 + G::TS;
  EOMat<P, T> Mm, Km;
  Mm.load(Q.Me, Q.Mo);
  Km.load(Q.Ke, Q.Ko);
  const int tx = (int)blockIdx.x % Q.ntx, ty = (int)blockIdx.x / Q.ntx;
  const int fx0 = tx * EX * P - 1, fy0 = ty * EY * P - 1;

  // pass 1: y segments (column x, cells sy*CY ..), inputs from global memory; a tile
  // whose input box lies inside the free grid needs no bounds checks
  const bool interior = fx0 >= 0 && fy0 >= 0 && fx0 + G::BX <= Q.nfx && fy0 + G::BY <= Q.nfy;
  for (int w = threadIdx.x; w < G::BX * SY; w += NT) {
    const int x = w % G::BX, sy = w / G::BX;
    const int fx = fx0 + x, fyb = fy0 + sy * CY * P;
    T c[NY];
    if (interior) {
      const T* col = Q.x + fx + (long long)Q.nfx * fyb;
#pragma unroll
      for (int i = 0; i < NY; ++i) c[i] = __ldg(col + (long long)Q.nfx * i);
    } else {
      const bool inx = (unsigned)fx < (unsigned)Q.nfx;
#pragma unroll
      for (int i = 0; i < NY; ++i) {
        const int fy = fyb + i;
        c[i] = (inx && (unsigned)fy < (unsigned)Q.nfy) ? __ldg(Q.x + fx + (long long)Q.nfx * fy)
                                                       : T(0);
      }
    }
    seg_mk<P, CY, T>(Mm, Km, c, [&](int o, T m, T k) {
      const int yo = sy * CY * P + o;
      T1[yo * G::PX + x] = m;
      T2[yo * G::PX + x] = k;
    });
  }
  __syncthreads();

  // pass 2: x segments (row yo, cells sx*CX ..): load, barrier, write in place
  const int w = threadIdx.x;
  const bool active = w < G::OY * SX;
  const int yo = w % G::OY, sx = w / G::OY;
  T a[NX], b[NX];
  if (active) {
    const T* r1 = T1 + yo * G::PX + sx * CX * P;
    const T* r2 = T2 + yo * G::PX + sx * CX * P;
#pragma unroll
    for (int i = 0; i < NX; ++i) {
      a[i] = ISO ? r1[i] : r1[i] * Q.cx;
      b[i] = ISO ? r2[i] : r2[i] * Q.cy;
    }
  }
  __syncthreads();
  if (active) {
    T* o1 = T1 + yo * G::PX + sx * CX * P;
    seg_kamb<P, CX, T>(Km, Mm, a, b, [&](int o, T v) { o1[o] = ISO ? v * Q.cx : v; });
  }
  __syncthreads();

  // store the owned box (free coordinates start at e0 * p)
  const int ox0 = fx0 + 1, oy0 = fy0 + 1;
  const bool full = ox0 + G::OX <= Q.nfx && oy0 + G::OY <= Q.nfy;
  T* ybase = Q.y + (long long)ox0 + (long long)Q.nfx * oy0;
  for (int i = threadIdx.x; i < G::OX * G::OY; i += NT) {
    const int xo = i % G::OX, yr = i / G::OX;
    if (full || (ox0 + xo < Q.nfx && oy0 + yr < Q.nfy))
      ybase[xo + (long long)Q.nfx * yr] = T1[yr * G::PX + xo];
  }
}

// The fused (x, y) sum takes x of the owned points from a shared-memory copy for
// FP32 only. Measured at Q4 64^3 in the CG loop: FP32 0.242 -> 0.233-0.239 ms per
// iteration (runs differ by about 2 %), FP64 0.360 -> 0.372 ms (its re-reads mostly
// hit L2, and the copy's stores lengthen the z pass).
template <typename T>
constexpr bool kStashDot = sizeof(T) == 4;

template <int P, int EX, int EY, int EZ, int NT, bool ISO, typename T, int MINB, bool NUM = false,
          bool CHEB = false>
__global__ void __launch_bounds__(NT, MINB)
k_cartesian(const __grid_constant__ CartParams<P, T> Q) {
  using G = Tile<P, EX, EY, EZ, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* T1 = reinterpret_cast<T*>(smem_raw);  // t1 -> a -> y   [OZ][BY][BX]
  T* T2 = T1 + G::TS;                        // t2 -> s        [OZ][BY][BX]
  EOMat<P, T> Mm, Km;
  Mm.load(Q.Me, Q.Mo);
  Km.load(Q.Ke, Q.Ko);
  const int tile = Q.tile0 + (int)blockIdx.x;
  cart_tile<P, EX, EY, EZ, NT, ISO, T, NUM, CHEB>(
      T1, T2, Mm, Km, Q.x, Q.y, Q.nfx, Q.nfy, Q.nfz, Q.zlo, Q.nfz_out, tile % Q.ntx,
      (tile / Q.ntx) % Q.nty, tile / (Q.ntx * Q.nty), Q.rz, Q.rx, Q.cy,
      Q.dot ? Q.dot + tile : nullptr, Q.dot && kStashDot<T> ? T2 + G::TS : nullptr, Q.num,
      &Q.cheb);
}

// diag(A) on the free points written by an apply (full mesh or slab). On a
// Cartesian mesh A = cx Kx(x)My(x)Mz + cy Mx(x)Ky(x)Mz + cz Mx(x)My(x)Kz with the 1D
// operators assembled along each axis, so diag(A) is the same sum of products
// of the assembled 1D diagonals: K[l][l] at a cell-interior node l, and
// K[0][0] + K[p][p] at a vertex (every free vertex lies between two cells).
struct DiagParams {
  double Kd[kMaxSB], Md[kMaxSB];
  double c[3];
  double* d;  // first written point
  int p, nfx, nfy, nfz_out;
  int D;      // 2: d = cx dK(x) dM(y) + cy dM(x) dK(y) over nfx x nfy points
};

__global__ void k_cartesian_diag(const __grid_constant__ DiagParams Q) {
  const long long n = (long long)Q.nfx * Q.nfy * Q.nfz_out;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int gx = (int)(i % Q.nfx) + 1;
    const long long r = i / Q.nfx;
    const int gy = (int)(r % Q.nfy) + 1;
    const int gz = (int)(r / Q.nfy) + 1;  // grid level, modulo p (a slab starts on a vertex)
    auto d1 = [&](const double* D, int g) {
      const int l = g % Q.p;
      return l == 0 ? D[0] + D[Q.p] : D[l];
    };
    if (Q.D == 2)
      Q.d[i] = Q.c[0] * d1(Q.Kd, gx) * d1(Q.Md, gy) + Q.c[1] * d1(Q.Md, gx) * d1(Q.Kd, gy);
    else
      Q.d[i] = Q.c[0] * d1(Q.Kd, gx) * d1(Q.Md, gy) * d1(Q.Md, gz) +
               Q.c[1] * d1(Q.Md, gx) * d1(Q.Kd, gy) * d1(Q.Md, gz) +
               Q.c[2] * d1(Q.Md, gx) * d1(Q.Md, gy) * d1(Q.Kd, gz);
  }
}

template <int P, typename T>
void fill_eo(const double* M, double scale, T* ue, T* uo) {
  using S = EO<P>;
  auto m = [&](int i, int j) { return scale * M[i * (P + 1) + j]; };
  for (int i = 0; i < S::NE; ++i)
    for (int j = i; j < S::NE; ++j) {
      double v;
      if (i < S::H && j < S::H) v = 0.5 * (m(i, j) + m(i, P - j));
      else v = m(i, j);  // a middle row or column
      ue[tri(i, j, S::NE)] = (T)v;
    }
  for (int i = 0; i < S::NO; ++i)
    for (int j = i; j < S::NO; ++j) uo[tri(i, j, S::NO)] = (T)(0.5 * (m(i, j) - m(i, P - j)));
}

// ---------------------------------------------------------------------------
// Batched form: one persistent kernel applies many problems of the same order
// (and the same 1D operators). The work items are (problem, right-hand side,
// tile), numbered problem by problem. Every CTA takes the next item from a
// global counter with one atomicAdd, until the items run out. No CTA ever waits
// for another. The counter is zeroed before each launch.
// ---------------------------------------------------------------------------
template <typename T>
struct BatchProblem {
  const T* x;
  T* y;
  long long ldx, ldy;   // elements between consecutive right-hand sides
  long long first;      // index of the problem's first work item
  int nfx, nfy, nfz;    // free grid
  int ntx, nty, ntz;    // tiles
  T rz, rx, cy;
};

template <int P, typename T>
struct BatchParams {
  T Me[EO<P>::UE], Mo[EO<P>::UO];
  T Ke[EO<P>::UE], Ko[EO<P>::UO];
  const BatchProblem<T>* probs;
  int nprob;
  long long total;  // work items
  unsigned long long* counter;
};

template <int P, int EX, int EY, int EZ, int NT, bool ISO, typename T, int MINB>
__global__ void __launch_bounds__(NT, MINB)
k_cartesian_batch(const __grid_constant__ BatchParams<P, T> Q) {
  using G = Tile<P, EX, EY, EZ, T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ long long s_item;
  T* T1 = reinterpret_cast<T*>(smem_raw);
  T* T2 = T1 + G::TS;
  EOMat<P, T> Mm, Km;
  Mm.load(Q.Me, Q.Mo);
  Km.load(Q.Ke, Q.Ko);
  for (;;) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(Q.counter, 1ull);
    __syncthreads();
    const long long item = s_item;
    if (item >= Q.total) break;  // the same value in every thread of the CTA
    int lo = 0, hi = Q.nprob - 1;  // last problem whose first item <= item
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (Q.probs[mid].first <= item) lo = mid;
      else hi = mid - 1;
    }
    const BatchProblem<T> pb = Q.probs[lo];
    const long long tiles = (long long)pb.ntx * pb.nty * pb.ntz;
    const long long local = item - pb.first;
    const long long rhs = local / tiles;
    const int tile = (int)(local - rhs * tiles);
    cart_tile<P, EX, EY, EZ, NT, ISO, T>(T1, T2, Mm, Km, pb.x + rhs * pb.ldx, pb.y + rhs * pb.ldy,
                                         pb.nfx, pb.nfy, pb.nfz, 0, pb.nfz, tile % pb.ntx,
                                         (tile / pb.ntx) % pb.nty, tile / (pb.ntx * pb.nty),
                                         pb.rz, pb.rx, pb.cy);
    __syncthreads();  // T1/T2 and s_item are reused by the next item
  }
}

template <int P, typename T, int EX, int EY, int EZ, int NT, int MINB>
void run_batch(const CartesianPlan& proto, const void* d_probs, int nprob, long long total,
               unsigned long long* counter, bool iso, cudaStream_t st) {
  using G = Tile<P, EX, EY, EZ, T>;
  BatchParams<P, T> Q{};
  fill_eo<P, T>(proto.M, 1.0, Q.Me, Q.Mo);
  fill_eo<P, T>(proto.K, 1.0, Q.Ke, Q.Ko);
  Q.probs = static_cast<const BatchProblem<T>*>(d_probs);
  Q.nprob = nprob;
  Q.total = total;
  Q.counter = counter;
  if (total == 0 || nprob == 0) return;
  const size_t smem = (size_t)G::WORDS * sizeof(T);
  auto kern = iso ? k_cartesian_batch<P, EX, EY, EZ, NT, true, T, MINB>
                  : k_cartesian_batch<P, EX, EY, EZ, NT, false, T, MINB>;
  SF_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int dev = 0, sms = 0, per_sm = 0;
  SF_CUDA_CHECK(cudaGetDevice(&dev));
  SF_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  SF_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  long long grid = (long long)sms * (per_sm > 0 ? per_sm : 1);
  if (grid > total) grid = total;
  kern<<<(unsigned)grid, NT, smem, st>>>(Q);
  SF_CUDA_CHECK(cudaGetLastError());
}

// One launch of the tile configuration (EX, EY, EZ cells, NT threads, MINB CTAs per SM).
// NUM: x and y in the numbering fuse.num (the numbered kernel).
template <int P, typename T, int EX, int EY, int EZ, int NT, int MINB, bool NUM = false>
void run_tile(const CartesianPlan& plan, const void* x, void* y, const CartFuse& fuse,
              cudaStream_t st) {
  using G = Tile<P, EX, EY, EZ, T>;
  CartParams<P, T> Q{};
  fill_eo<P, T>(plan.M, 1.0, Q.Me, Q.Mo);
  fill_eo<P, T>(plan.K, 1.0, Q.Ke, Q.Ko);
  const double cx = plan.c[0], cy = plan.c[1], cz = plan.c[2];
  Q.rz = (T)(cz / cy);
  Q.rx = (T)(cx / cy);
  Q.cy = (T)cy;
  const bool iso = (cx == cy) && (cz == cy);
  Q.x = static_cast<const T*>(x);
  Q.y = static_cast<T*>(y);
  Q.nfx = plan.nx * P - 1;
  Q.nfy = plan.ny * P - 1;
  Q.nfz = plan.nz * P - 1;
  Q.zlo = 0;
  Q.nfz_out = Q.nfz;
  if (plan.slab) {  // planes of levels z0 p .. (z1 + 1) p; outputs on levels z0 p + 1 ..
    const long long pz = (long long)Q.nfx * Q.nfy;
    Q.x += pz;
    Q.y += pz;
    Q.nfz = (plan.nz + 1) * P;
    Q.zlo = -1;
    Q.nfz_out = plan.nz * P - (plan.slab_top ? 1 : 0);
  }
  Q.ntx = (plan.nx + EX - 1) / EX;
  Q.nty = (plan.ny + EY - 1) / EY;
  Q.ntz = (plan.nz + EZ - 1) / EZ;
  Q.dot = fuse.dot;
  Q.num = fuse.num;
  SF_REQUIRE(NUM == (fuse.num != nullptr), SF_ERR_STATE, "numbered kernel without a numbering");
  SF_REQUIRE(!NUM || (!fuse.dot && !plan.slab && fuse.tz1 < 0), SF_ERR_UNSUPPORTED,
             "a numbered apply has no fused dot, slab or tile-row range");
  long long tiles = (long long)Q.ntx * Q.nty * Q.ntz;
  SF_REQUIRE(tiles < (1LL << 31), SF_ERR_ARG, "too many tiles");
  if (fuse.tz1 >= 0) {  // tile rows [tz0, tz1) only
    SF_REQUIRE(fuse.tz0 >= 0 && fuse.tz0 < fuse.tz1 && fuse.tz1 <= Q.ntz, SF_ERR_ARG,
               "tile-row range out of bounds");
    Q.tile0 = fuse.tz0 * Q.ntx * Q.nty;
    tiles = (long long)(fuse.tz1 - fuse.tz0) * Q.ntx * Q.nty;
  }
  // with the dot (FP32): the owned x values of the tile after T1, T2
  const size_t smem =
      ((size_t)G::WORDS + (fuse.dot && kStashDot<T> ? (size_t)G::OX * G::OY * G::OZ : 0)) *
      sizeof(T);
  if (fuse.cheb.mode) {  // an apply with the Chebyshev step in its store phase (FP32)
    SF_REQUIRE(!fuse.dot && fuse.tz1 < 0 && !plan.slab, SF_ERR_UNSUPPORTED,
               "the Chebyshev store phase takes a whole mesh without a fused dot or row range");
    if constexpr (sizeof(T) == 4 && !NUM) {
      SF_REQUIRE(fuse.cheb.z_out != x, SF_ERR_ARG, "the Chebyshev step writes z elsewhere");
      Q.cheb = ChebEpi<T>{static_cast<const T*>(fuse.cheb.r), static_cast<const T*>(fuse.cheb.dinv),
                          static_cast<T*>(fuse.cheb.d), static_cast<T*>(fuse.cheb.z_out),
                          (T)fuse.cheb.c1, (T)fuse.cheb.c2, fuse.cheb.mode};
      auto kc = iso ? k_cartesian<P, EX, EY, EZ, NT, true, T, MINB, false, true>
                    : k_cartesian<P, EX, EY, EZ, NT, false, T, MINB, false, true>;
      SF_CUDA_CHECK(cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      kc<<<(unsigned)tiles, NT, smem, st>>>(Q);
      SF_CUDA_CHECK(cudaGetLastError());
      return;
    } else {
      throw Error(SF_ERR_UNSUPPORTED, "the Chebyshev store phase is FP32 only");
    }
  }
  auto kern = iso ? k_cartesian<P, EX, EY, EZ, NT, true, T, MINB, NUM>
                  : k_cartesian<P, EX, EY, EZ, NT, false, T, MINB, NUM>;
  SF_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)tiles, NT, smem, st>>>(Q);
  SF_CUDA_CHECK(cudaGetLastError());
}

// One launch of the 2D tile configuration (EX x EY cells, x/y segments of CX/CY cells).
template <int P, typename T, int EX, int EY, int CX, int CY, int NT, int MINB>
void run_tile2(const CartesianPlan& plan, const void* x, void* y, const CartFuse& fuse,
               cudaStream_t st) {
  using G = Tile2<P, EX, EY>;
  SF_REQUIRE(!fuse.dot && fuse.tz1 < 0, SF_ERR_UNSUPPORTED,
             "the 2D apply has no fused dot or tile-row range");
  CartParams2<P, T> Q{};
  fill_eo<P, T>(plan.M, 1.0, Q.Me, Q.Mo);
  fill_eo<P, T>(plan.K, 1.0, Q.Ke, Q.Ko);
  const double cx = plan.c[0], cy = plan.c[1];
  const bool iso = cx == cy;
  Q.cx = (T)cx;
  Q.cy = (T)cy;
  Q.x = static_cast<const T*>(x);
  Q.y = static_cast<T*>(y);
  Q.nfx = plan.nx * P - 1;
  Q.nfy = plan.ny * P - 1;
  Q.ntx = (plan.nx + EX - 1) / EX;
  Q.nty = (plan.ny + EY - 1) / EY;
  const long long tiles = (long long)Q.ntx * Q.nty;
  SF_REQUIRE(tiles < (1LL << 31), SF_ERR_ARG, "too many tiles");
  const size_t smem = (size_t)G::WORDS * sizeof(T);
  auto kern = iso ? k_cartesian2d<P, EX, EY, CX, CY, NT, true, T, MINB>
                  : k_cartesian2d<P, EX, EY, CX, CY, NT, false, T, MINB>;
  SF_CUDA_CHECK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  kern<<<(unsigned)tiles, NT, smem, st>>>(Q);
  SF_CUDA_CHECK(cudaGetLastError());
}

using RunFn = void (*)(const CartesianPlan&, const void*, void*, const CartFuse&, cudaStream_t);
using BatchFn = void (*)(const CartesianPlan&, const void*, int, long long, unsigned long long*,
                         bool, cudaStream_t);
struct Candidate {
  RunFn run;
  BatchFn batch;
  int ex, ey, ez;
  const char* name;
};
#define SF_TILE(P_, T_, EX_, EY_, EZ_, NT_, MINB_)                                          \
  {&run_tile<P_, T_, EX_, EY_, EZ_, NT_, MINB_>, &run_batch<P_, T_, EX_, EY_, EZ_, NT_, MINB_>, \
   EX_, EY_, EZ_, #EX_ "x" #EY_ "x" #EZ_ " cells, " #NT_ " thr, " #MINB_ "/SM"}

// Candidate tile shapes per (P, dtype); the first is the default. Shared
// memory per CTA is 2 * PLANE * EZ*P words. The autotuner times them all on
// the operator's own mesh.
template <int P, typename T>
struct Cands;
// Low and high orders: tiles chosen so that the three passes (BX*BY columns, BX*OZ
// and OY*OZ lines) keep most of the threads busy.
template <> struct Cands<1, double> { static constexpr Candidate c[] = {SF_TILE(1, double, 8, 8, 4, 256, 2),
                                                                      SF_TILE(1, double, 8, 16, 16, 256, 2),
                                                                      SF_TILE(1, double, 16, 16, 16, 256, 2)}; };
template <> struct Cands<2, double> { static constexpr Candidate c[] = {SF_TILE(2, double, 4, 4, 4, 256, 2),
                                                                      SF_TILE(2, double, 8, 4, 2, 256, 2),
                                                                      SF_TILE(2, double, 8, 8, 8, 256, 2),
                                                                      SF_TILE(2, double, 4, 8, 8, 256, 2)}; };
template <> struct Cands<3, double> { static constexpr Candidate c[] = {SF_TILE(3, double, 4, 4, 2, 256, 2),
                                                                      SF_TILE(3, double, 4, 4, 3, 256, 2),
                                                                      SF_TILE(3, double, 4, 6, 4, 256, 2),
                                                                      SF_TILE(3, double, 4, 4, 6, 256, 2)}; };
template <> struct Cands<4, double> { static constexpr Candidate c[] = {SF_TILE(4, double, 4, 4, 2, 256, 3),
                                                                      SF_TILE(4, double, 4, 4, 2, 256, 2),
                                                                      SF_TILE(4, double, 4, 4, 3, 256, 2),
                                                                      SF_TILE(4, double, 4, 4, 4, 256, 2),
                                                                      SF_TILE(4, double, 4, 4, 2, 224, 3),
                                                                      SF_TILE(4, double, 4, 4, 3, 320, 2),
                                                                      SF_TILE(4, double, 4, 4, 1, 128, 6),
                                                                      SF_TILE(4, double, 8, 4, 2, 256, 2)}; };
// Q5 2x2x3 at three CTAs per SM and Q6 2x2x2 at two were the fastest FP64 shapes on 20^3 and
// 36^3 (Q5: 0.0168 / 0.0664 ms) and on 16^3 (Q6: 0.0168 ms; 2x3x2 on 30^3, 0.0739 ms).
template <> struct Cands<5, double> { static constexpr Candidate c[] = {SF_TILE(5, double, 2, 2, 3, 256, 3),
                                                                      SF_TILE(5, double, 2, 2, 2, 256, 2),
                                                                      SF_TILE(5, double, 2, 3, 3, 256, 2),
                                                                      SF_TILE(5, double, 2, 4, 2, 256, 2)}; };
template <> struct Cands<6, double> { static constexpr Candidate c[] = {SF_TILE(6, double, 2, 2, 2, 256, 2),
                                                                      SF_TILE(6, double, 2, 3, 2, 256, 2)}; };
template <> struct Cands<7, double> { static constexpr Candidate c[] = {SF_TILE(7, double, 2, 2, 1, 256, 1),
                                                                      SF_TILE(7, double, 2, 2, 2, 256, 1)}; };
template <> struct Cands<8, double> { static constexpr Candidate c[] = {SF_TILE(8, double, 2, 2, 1, 256, 1),
                                                                      SF_TILE(8, double, 2, 2, 2, 256, 1)}; };
template <> struct Cands<1, float> { static constexpr Candidate c[] = {SF_TILE(1, float, 8, 8, 4, 256, 2),
                                                                     SF_TILE(1, float, 8, 16, 16, 256, 3),
                                                                     SF_TILE(1, float, 16, 16, 16, 256, 2)}; };
template <> struct Cands<2, float> { static constexpr Candidate c[] = {SF_TILE(2, float, 4, 4, 4, 256, 2),
                                                                     SF_TILE(2, float, 8, 8, 8, 256, 2),
                                                                     SF_TILE(2, float, 4, 8, 8, 256, 3)}; };
template <> struct Cands<3, float> { static constexpr Candidate c[] = {SF_TILE(3, float, 4, 4, 4, 256, 2),
                                                                     SF_TILE(3, float, 4, 4, 2, 256, 3),
                                                                     SF_TILE(3, float, 4, 6, 4, 256, 2),
                                                                     SF_TILE(3, float, 4, 4, 6, 256, 2)}; };
template <> struct Cands<4, float> { static constexpr Candidate c[] = {SF_TILE(4, float, 4, 4, 2, 256, 3),
                                                                     SF_TILE(4, float, 4, 4, 3, 256, 3),
                                                                     SF_TILE(4, float, 4, 4, 4, 256, 3),
                                                                     SF_TILE(4, float, 4, 4, 3, 256, 4)}; };
template <> struct Cands<5, float> { static constexpr Candidate c[] = {SF_TILE(5, float, 2, 2, 2, 256, 2),
                                                                     SF_TILE(5, float, 2, 3, 3, 256, 2),
                                                                     SF_TILE(5, float, 2, 4, 2, 256, 2)}; };
template <> struct Cands<6, float> { static constexpr Candidate c[] = {SF_TILE(6, float, 2, 2, 2, 256, 2),
                                                                     SF_TILE(6, float, 2, 3, 2, 256, 2)}; };
template <> struct Cands<7, float> { static constexpr Candidate c[] = {SF_TILE(7, float, 2, 2, 2, 256, 2),
                                                                     SF_TILE(7, float, 2, 2, 1, 256, 2)}; };
template <> struct Cands<8, float> { static constexpr Candidate c[] = {SF_TILE(8, float, 2, 2, 1, 256, 2),
                                                                     SF_TILE(8, float, 2, 2, 2, 256, 1)}; };
#undef SF_TILE

// 2D candidates: tiles of about 64 x 64 points; pass 2 gives every thread one x segment.
#define SF_TILE2(P_, T_, EX_, EY_, CX_, CY_, NT_, MINB_)                                  \
  {&run_tile2<P_, T_, EX_, EY_, CX_, CY_, NT_, MINB_>, nullptr, EX_, EY_, 0,             \
   #EX_ "x" #EY_ " cells, segments " #CX_ "/" #CY_ ", " #NT_ " thr, " #MINB_ "/SM"}
template <int P, typename T>
struct Cands2;
#define SF_C2(P_, ...)                                                                     \
  template <> struct Cands2<P_, double> { static constexpr Candidate c[] = {__VA_ARGS__}; };
#define SF_T2D(P_, EX_, EY_, CX_, CY_, NT_, MINB_) SF_TILE2(P_, double, EX_, EY_, CX_, CY_, NT_, MINB_)
#define SF_T2F(P_, EX_, EY_, CX_, CY_, NT_, MINB_) SF_TILE2(P_, float, EX_, EY_, CX_, CY_, NT_, MINB_)
SF_C2(1, SF_T2D(1, 64, 64, 16, 16, 256, 2))
SF_C2(2, SF_T2D(2, 32, 32, 8, 8, 256, 2))
SF_C2(3, SF_T2D(3, 20, 20, 5, 5, 256, 2))
SF_C2(4, SF_T2D(4, 16, 16, 4, 4, 256, 2), SF_T2D(4, 16, 16, 2, 4, 512, 1),
      SF_T2D(4, 16, 16, 4, 4, 288, 2), SF_T2D(4, 16, 15, 4, 5, 256, 2),
      SF_T2D(4, 20, 12, 5, 4, 256, 2))
SF_C2(5, SF_T2D(5, 12, 12, 3, 3, 256, 2))
SF_C2(6, SF_T2D(6, 10, 8, 2, 2, 256, 2))
SF_C2(7, SF_T2D(7, 8, 8, 2, 2, 256, 2))
SF_C2(8, SF_T2D(8, 8, 8, 2, 2, 256, 2))
#undef SF_C2
#define SF_C2(P_, ...)                                                                     \
  template <> struct Cands2<P_, float> { static constexpr Candidate c[] = {__VA_ARGS__}; };
SF_C2(1, SF_T2F(1, 64, 64, 16, 16, 256, 2))
SF_C2(2, SF_T2F(2, 32, 32, 8, 8, 256, 2))
SF_C2(3, SF_T2F(3, 20, 20, 5, 5, 256, 2))
SF_C2(4, SF_T2F(4, 16, 16, 4, 4, 256, 2), SF_T2F(4, 16, 16, 2, 4, 512, 1),
      SF_T2F(4, 16, 16, 4, 4, 288, 3), SF_T2F(4, 16, 15, 4, 5, 256, 3),
      SF_T2F(4, 20, 12, 5, 4, 256, 3))
SF_C2(5, SF_T2F(5, 12, 12, 3, 3, 256, 2))
SF_C2(6, SF_T2F(6, 10, 8, 2, 2, 256, 2))
SF_C2(7, SF_T2F(7, 8, 8, 2, 2, 256, 2))
SF_C2(8, SF_T2F(8, 8, 8, 2, 2, 256, 2))
#undef SF_C2
#undef SF_T2D
#undef SF_T2F
#undef SF_TILE2

// The numbered kernel: one tile shape per order and dtype (the autotuner's usual choice
// on large meshes), which keeps its instantiations few.
template <int P, typename T>
struct NumTile;
#define SF_NUMT(P_, T_, EX_, EY_, EZ_, NT_, MINB_)                           \
  template <> struct NumTile<P_, T_> {                                      \
    static constexpr RunFn run = &run_tile<P_, T_, EX_, EY_, EZ_, NT_, MINB_, true>; \
  };
SF_NUMT(1, double, 8, 8, 4, 256, 2) SF_NUMT(1, float, 8, 8, 4, 256, 2)
SF_NUMT(2, double, 4, 4, 4, 256, 2) SF_NUMT(2, float, 4, 4, 4, 256, 2)
SF_NUMT(3, double, 4, 4, 2, 256, 2) SF_NUMT(3, float, 4, 4, 4, 256, 2)
SF_NUMT(4, double, 4, 4, 3, 256, 2) SF_NUMT(4, float, 4, 4, 3, 256, 4)
SF_NUMT(5, double, 2, 2, 2, 256, 2) SF_NUMT(5, float, 2, 2, 2, 256, 2)
SF_NUMT(6, double, 2, 2, 2, 256, 1) SF_NUMT(6, float, 2, 2, 2, 256, 2)
SF_NUMT(7, double, 2, 2, 1, 256, 1) SF_NUMT(7, float, 2, 2, 2, 256, 2)
SF_NUMT(8, double, 2, 2, 1, 256, 1) SF_NUMT(8, float, 2, 2, 1, 256, 2)
#undef SF_NUMT

template <typename T>
RunFn numbered_run(int SB) {
  switch (SB - 1) {
#define SF_CASE(P_) \
  case P_: return NumTile<P_, T>::run;
    SF_CASE(1) SF_CASE(2) SF_CASE(3) SF_CASE(4) SF_CASE(5) SF_CASE(6) SF_CASE(7) SF_CASE(8)
#undef SF_CASE
    default: throw Error(SF_ERR_UNSUPPORTED, "no tiled Cartesian kernel for this order");
  }
}

template <typename T, int P>
int cand_count() { return (int)(sizeof(Cands<P, T>::c) / sizeof(Candidate)); }

template <typename T, int P>
int cand2_count() { return (int)(sizeof(Cands2<P, T>::c) / sizeof(Candidate)); }

template <typename T>
const Candidate& candidate(int D, int SB, int k) {
  if (D == 2) {
    switch (SB - 1) {
#define SF_CASE(P_) \
  case P_: return Cands2<P_, T>::c[k < cand2_count<T, P_>() ? k : 0];
      SF_CASE(1) SF_CASE(2) SF_CASE(3) SF_CASE(4) SF_CASE(5) SF_CASE(6) SF_CASE(7) SF_CASE(8)
#undef SF_CASE
      default: throw Error(SF_ERR_UNSUPPORTED, "no 2D tiled Cartesian kernel for this order");
    }
  }
  switch (SB - 1) {
#define SF_CASE(P_) \
  case P_: return Cands<P_, T>::c[k < cand_count<T, P_>() ? k : 0];
    SF_CASE(1) SF_CASE(2) SF_CASE(3) SF_CASE(4) SF_CASE(5) SF_CASE(6) SF_CASE(7) SF_CASE(8)
#undef SF_CASE
    default: throw Error(SF_ERR_UNSUPPORTED, "no tiled Cartesian kernel for this order");
  }
}

template <typename T>
int candidates_for(int D, int SB) {
  switch (SB - 1) {
#define SF_CASE(P_) \
  case P_: return D == 2 ? cand2_count<T, P_>() : cand_count<T, P_>();
    SF_CASE(1) SF_CASE(2) SF_CASE(3) SF_CASE(4) SF_CASE(5) SF_CASE(6) SF_CASE(7) SF_CASE(8)
#undef SF_CASE
    default: return 0;
  }
}

int candidate_count(int D, int SB, int dtype) {
  return dtype == SF_F64 ? candidates_for<double>(D, SB) : candidates_for<float>(D, SB);
}

const Candidate& pick(const CartesianPlan& plan, int dtype, int k) {
  return dtype == SF_F64 ? candidate<double>(plan.D, plan.SB, k)
                         : candidate<float>(plan.D, plan.SB, k);
}

}  // namespace

bool cartesian_prepare(CartesianPlan& plan, int SB, int SQ, const double* A, const double* B,
                       const double* w1, const double* G0, int nx, int ny, int nz, int D) {
  plan.ready = false;
  if (SB < 2 || SB > 9) return false;
  if (!(G0[0] > 0 && G0[1] > 0 && (D == 2 || G0[2] > 0))) return false;
  plan.D = D;
  plan.SB = SB;
  plan.SQ = SQ;
  plan.nx = nx;
  plan.ny = ny;
  plan.nz = nz;
  // M = A^T W A, K = B^T W B (1D, kernel order = lexicographic along the segment)
  double mmax = 0.0, kmax = 0.0;
  for (int l = 0; l < SB; ++l)
    for (int m = 0; m < SB; ++m) {
      double mm = 0.0, kk = 0.0;
      for (int q = 0; q < SQ; ++q) {
        mm += w1[q] * A[q * SB + l] * A[q * SB + m];
        kk += w1[q] * B[q * SB + l] * B[q * SB + m];
      }
      plan.M[l * SB + m] = mm;
      plan.K[l * SB + m] = kk;
      mmax = std::fmax(mmax, std::fabs(mm));
      kmax = std::fmax(kmax, std::fabs(kk));
    }
  // the even-odd form needs symmetric, centro-symmetric M and K
  const int P = SB - 1;
  for (int l = 0; l < SB; ++l)
    for (int m = 0; m < SB; ++m) {
      const double* Ms = plan.M;
      const double* Ks = plan.K;
      if (std::fabs(Ms[l * SB + m] - Ms[m * SB + l]) > 1e-13 * mmax ||
          std::fabs(Ms[l * SB + m] - Ms[(P - l) * SB + (P - m)]) > 1e-13 * mmax ||
          std::fabs(Ks[l * SB + m] - Ks[m * SB + l]) > 1e-13 * kmax ||
          std::fabs(Ks[l * SB + m] - Ks[(P - l) * SB + (P - m)]) > 1e-13 * kmax)
        return false;
    }
  plan.c[0] = G0[0];
  plan.c[1] = G0[1];
  plan.c[2] = G0[2];
  plan.ready = true;
  return true;
}

bool cartesian_supported(const CartesianPlan& plan, int dtype) {
  return plan.ready && (dtype == SF_F64 || dtype == SF_F32) && plan.SB >= 2 && plan.SB <= 9;
}

int cartesian_launches(const CartesianPlan& plan) { return 1; }

static int dtype_slot(int dtype) {
  if (dtype == SF_F64) return 0;
  if (dtype == SF_F32) return 1;
  throw Error(SF_ERR_ARG, "dtype must be SF_F64 or SF_F32");
}

int cartesian_candidates(const CartesianPlan& plan, int dtype) {
  dtype_slot(dtype);
  return candidate_count(plan.D, plan.SB, dtype);
}

const char* cartesian_candidate_name(const CartesianPlan& plan, int dtype, int k) {
  dtype_slot(dtype);
  return pick(plan, dtype, k).name;
}

void cartesian_apply_candidate(const CartesianPlan& plan, int dtype, int k, const void* x, void* y,
                               cudaStream_t stream) {
  SF_REQUIRE(plan.ready, SF_ERR_STATE, "Cartesian plan not prepared");
  dtype_slot(dtype);
  pick(plan, dtype, k).run(plan, x, y, CartFuse{}, stream);
}

void cartesian_apply(const CartesianPlan& plan, int dtype, const void* x, void* y,
                     cudaStream_t stream, const CartFuse& fuse) {
  SF_REQUIRE(plan.ready, SF_ERR_STATE, "Cartesian plan not prepared");
  if (fuse.num) {  // the numbered kernel has its own tile shape
    SF_REQUIRE(plan.D == 3, SF_ERR_UNSUPPORTED, "the numbered kernel is 3D");
    (dtype_slot(dtype) == 0 ? numbered_run<double>(plan.SB) : numbered_run<float>(plan.SB))(
        plan, x, y, fuse, stream);
    return;
  }
  pick(plan, dtype, plan.choice[dtype_slot(dtype)]).run(plan, x, y, fuse, stream);
}

void cartesian_diag(const CartesianPlan& plan, double* d, cudaStream_t stream) {
  SF_REQUIRE(plan.ready, SF_ERR_STATE, "Cartesian plan not prepared");
  DiagParams Q{};
  const int SB = plan.SB, P = SB - 1;
  for (int l = 0; l < SB; ++l) {
    Q.Kd[l] = plan.K[l * SB + l];
    Q.Md[l] = plan.M[l * SB + l];
  }
  for (int k = 0; k < 3; ++k) Q.c[k] = plan.c[k];
  Q.p = P;
  Q.nfx = plan.nx * P - 1;
  Q.nfy = plan.ny * P - 1;
  Q.nfz_out = plan.slab ? plan.nz * P - (plan.slab_top ? 1 : 0) : plan.nz * P - 1;
  Q.D = plan.D;
  if (plan.D == 2) Q.nfz_out = 1;
  Q.d = d + (plan.slab ? (long long)Q.nfx * Q.nfy : 0);
  const long long n = (long long)Q.nfx * Q.nfy * Q.nfz_out;
  if (n <= 0) return;
  const long long blocks = std::min<long long>((n + 255) / 256, 148LL * 16);
  k_cartesian_diag<<<(unsigned)blocks, 256, 0, stream>>>(Q);
  SF_CUDA_CHECK(cudaGetLastError());
}

int cartesian_tile_ez(const CartesianPlan& plan, int dtype) {
  return pick(plan, dtype, plan.choice[dtype_slot(dtype)]).ez;
}

long long cartesian_tiles(const CartesianPlan& plan, int dtype) {
  const Candidate& c = pick(plan, dtype, plan.choice[dtype_slot(dtype)]);
  return (long long)((plan.nx + c.ex - 1) / c.ex) * ((plan.ny + c.ey - 1) / c.ey) *
         ((plan.nz + c.ez - 1) / c.ez);
}

void cartesian_release(CartesianPlan& plan) { plan.ready = false; }

size_t cartesian_batch_desc_bytes(int dtype) {
  return dtype_slot(dtype) == 0 ? sizeof(BatchProblem<double>) : sizeof(BatchProblem<float>);
}

namespace {
template <typename T>
long long batch_desc(const CartesianPlan& plan, const Candidate& c, const void* x, void* y,
                     long long ldx, long long ldy, int nrhs, long long first, void* out) {
  BatchProblem<T> d{};
  const int P = plan.SB - 1;
  d.x = static_cast<const T*>(x);
  d.y = static_cast<T*>(y);
  d.ldx = ldx;
  d.ldy = ldy;
  d.first = first;
  d.nfx = plan.nx * P - 1;
  d.nfy = plan.ny * P - 1;
  d.nfz = plan.nz * P - 1;
  d.ntx = (plan.nx + c.ex - 1) / c.ex;
  d.nty = (plan.ny + c.ey - 1) / c.ey;
  d.ntz = (plan.nz + c.ez - 1) / c.ez;
  d.rz = (T)(plan.c[2] / plan.c[1]);
  d.rx = (T)(plan.c[0] / plan.c[1]);
  d.cy = (T)plan.c[1];
  std::memcpy(out, &d, sizeof(d));
  return (long long)d.ntx * d.nty * d.ntz * nrhs;
}
}  // namespace

long long cartesian_batch_desc(const CartesianPlan& plan, int dtype, int cand, const void* x,
                               void* y, long long ldx, long long ldy, int nrhs, long long first,
                               void* out) {
  const Candidate& c = pick(plan, dtype, cand);
  return dtype_slot(dtype) == 0 ? batch_desc<double>(plan, c, x, y, ldx, ldy, nrhs, first, out)
                                : batch_desc<float>(plan, c, x, y, ldx, ldy, nrhs, first, out);
}

void cartesian_batch_launch(const CartesianPlan& proto, int dtype, int cand, const void* d_desc,
                            int nprob, long long total, unsigned long long* d_counter, bool iso,
                            cudaStream_t st) {
  SF_REQUIRE(proto.ready, SF_ERR_STATE, "Cartesian plan not prepared");
  pick(proto, dtype, cand).batch(proto, d_desc, nprob, total, d_counter, iso, st);
}

}  // namespace sf
