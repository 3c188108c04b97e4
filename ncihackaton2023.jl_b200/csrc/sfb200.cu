// C ABI of the sum-factorized Laplacian operator (include/sfb200.h).
//
// The handle mirrors the pair SumFactorizationMap + LazyMatrix of the
// reference (src/SumFactorizationMaps.jl:2-10, src/LazyMatrices.jl:1-50).
// It owns the device copies of the 1D basis, the cell-to-dof table and the
// geometric factors. The x and y vectors are borrowed from the caller.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "sf_cg.cuh"
#include "sf_internal.cuh"
#include "sf_cartesian.cuh"

using sf::Error;

struct sf_op {
  int D = 3, SB = 0, SQ = 0, p = 0;
  std::vector<double> A_user, B_user;  // [q][j], caller's 1D order
  std::vector<int> jt_user;            // [k][d]: 0-based 1D index of local dof k along d
  std::vector<int> perm;               // caller 1D index -> kernel 1D index
  std::vector<double> A, B;            // [q][j], kernel 1D order
  sf::Cells cells;
  long long n_free = 0;
  int32_t* d_ids = nullptr;
  int32_t* d_t2l = nullptr;
  sf::Geometry geom;
  double* d_gtab = nullptr;
  float* d_gtab32 = nullptr;  // FP32 copy of d_gtab (the FP32 element kernel's metric)
  double* d_wdet = nullptr;  // w |det J| at the points (right-hand side)
  double* d_kappa = nullptr;
  long long cq_cells = -1;  // -1 = unset, 0 = fill (one cell for all)
  bool cartesian_ok = false;
  sf::CartesianPlan cart;   // tiled Cartesian kernel set-up
  // z-slab of a structured mesh (sf_set_structured_slab): cells [slab_z0, slab_z1) of mesh_nz
  bool slab = false;
  int slab_z0 = 0, slab_z1 = 0, mesh_nz = 0;
  long long plane = 0;       // free points per z level
  double* d_dinv = nullptr;  // 1 / diag(A) on the owned points (distributed CG)
  // sf_set_structured_numbering: the caller's free id of each lexicographic free point.
  // Vector entry points then permute into lexicographic order and back around the work.
  int32_t* d_numbering = nullptr;
  int32_t* d_numbering_inv = nullptr;  // its inverse: lexicographic index of each caller id
  // A numbered apply on the tiled kernel reads and writes through the numbering inside
  // the kernel when the numbering keeps neighbours near (numbering_local), else it permutes
  // into lexicographic order and back. numbered_fused: -1 that choice, 0 / 1 forced.
  bool numbering_local = false;
  int numbered_fused = -1;
  void* d_lex = nullptr;     // two lexicographic vectors (8 bytes per entry) for that
  bool lex_inside = false;   // set while the work runs on lexicographic vectors
  // workspaces
  double* d_diag = nullptr;  // FP64 diag(A), cached
  double* d_jtab = nullptr;  // inverse Jacobi diagonal per position in a cell (Cartesian), cached
  bool jacobi_table = true;  // CG vector kernels read D^-1 from d_jtab where it exists
  void* d_ws = nullptr;
  size_t ws_bytes = 0;
  double* d_hx = nullptr;    // sf_mul_host staging
  double* d_hy = nullptr;
  long long h_n = 0;         // their length
  cudaStream_t pipe[3] = {nullptr, nullptr, nullptr};  // sf_mul_host: copy in, apply, copy out
  std::vector<cudaEvent_t> pipe_ev;
  double* h_scalar = nullptr;  // pinned
  double* h_report = nullptr;  // mapped pinned: CG progress reports written by the device
  double* d_report = nullptr;  // its device address
  double mixed_inner_reltol = 1e-1;
  int host_groups = 8;  // sf_mul_host: groups of tile rows copied in, applied and copied out
  int last_outer = 0, last_inner = 0;
  double last_relres = 0.0;
  std::string err;
};

namespace {

int fail(sf_op* op, int status, const std::string& msg) {
  if (op) op->err = msg;
  return status;
}

template <typename F>
int guarded(sf_op* op, F&& f) {
  try {
    f();
    if (op) op->err.clear();
    return SF_OK;
  } catch (const Error& e) {
    return fail(op, e.status, e.what());
  } catch (const std::bad_alloc&) {
    return fail(op, SF_ERR_ARG, "host allocation failed");
  } catch (const std::exception& e) {
    return fail(op, SF_ERR_ARG, e.what());
  }
}

// Rethrows the failure of a nested entry-point call on the same handle.
void check_status(int status, const sf_op* op) {
  if (status != SF_OK) throw Error(status, op->err);
}

void dfree(void* p) {
  if (p) cudaFree(p);
}

template <typename T>
T* dalloc(size_t n) {
  void* p = nullptr;
  SF_CUDA_CHECK(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
  return static_cast<T*>(p);
}

size_t dsize(int dtype) {
  if (dtype == SF_F64) return 8;
  if (dtype == SF_F32) return 4;
  throw Error(SF_ERR_ARG, "dtype must be SF_F64 or SF_F32");
}

// Kernel-order tensor position of local dof k.
int tensor_pos(const sf_op* op, int k) {
  int pos = 0, stride = 1;
  for (int d = 0; d < op->D; ++d) {
    pos += op->perm[op->jt_user[k * op->D + d]] * stride;
    stride *= op->SB;
  }
  return pos;
}

void rebuild_kernel_basis(sf_op* op) {
  const int SB = op->SB, SQ = op->SQ;
  op->A.assign(SQ * SB, 0.0);
  op->B.assign(SQ * SB, 0.0);
  for (int q = 0; q < SQ; ++q)
    for (int j = 0; j < SB; ++j) {
      op->A[q * SB + op->perm[j]] = op->A_user[q * SB + j];
      op->B[q * SB + op->perm[j]] = op->B_user[q * SB + j];
    }
  int nloc = 1;
  for (int d = 0; d < op->D; ++d) nloc *= SB;
  std::vector<int32_t> t2l(nloc, -1);
  for (int k = 0; k < nloc; ++k) t2l[tensor_pos(op, k)] = k;
  for (int v : t2l)
    SF_REQUIRE(v >= 0, SF_ERR_ARG, "dof_map is not a permutation of the tensor indices");
  dfree(op->d_t2l);
  op->d_t2l = nullptr;
  op->d_t2l = dalloc<int32_t>(nloc);
  SF_CUDA_CHECK(cudaMemcpy(op->d_t2l, t2l.data(), nloc * sizeof(int32_t), cudaMemcpyHostToDevice));
}

void require_ready(const sf_op* op) {
  SF_REQUIRE(op, SF_ERR_ARG, "null handle");
  SF_REQUIRE(op->cells.mesh != sf::MESH_NONE, SF_ERR_STATE,
             "no mesh: call sf_set_cells or sf_set_structured first");
  SF_REQUIRE(op->geom.kind != sf::GEOM_NONE, SF_ERR_STATE,
             "no geometry: call sf_set_cell_quantities first");
  SF_REQUIRE(op->cq_cells == 0 || op->cq_cells == op->cells.ncells, SF_ERR_STATE,
             "cell quantities were given for a different number of cells");
}

void update_cartesian(sf_op* op) {
  op->cartesian_ok = false;
  if (op->cells.mesh != sf::MESH_STRUCTURED || op->geom.kind != sf::GEOM_SEPARABLE ||
      op->geom.kappa != nullptr)
    return;
  const double* G = op->geom.G0;
  const double scale = std::max({std::fabs(G[0]), std::fabs(G[1]), std::fabs(G[2])});
  if (std::fabs(G[3]) > 1e-14 * scale || std::fabs(G[4]) > 1e-14 * scale ||
      std::fabs(G[5]) > 1e-14 * scale)
    return;
  op->cartesian_ok = sf::cartesian_prepare(op->cart, op->SB, op->SQ, op->A.data(), op->B.data(),
                                           op->geom.w1, G, op->cells.nx, op->cells.ny,
                                           op->cells.nz, op->D);
  op->cart.slab = op->slab;
  op->cart.slab_top = op->slab && op->slab_z1 == op->mesh_nz;
}

// A numbered operator whose caller passes vectors in its own numbering.
bool numbered(const sf_op* op) { return op->d_numbering && !op->lex_inside; }

// Lexicographic vector k (0 or 1) of a numbered operator, n_free entries of up to 8 bytes.
void* lex_vec(sf_op* op, int k) {
  const size_t vb = (op->n_free * sizeof(double) + 255) & ~size_t(255);
  if (!op->d_lex) SF_CUDA_CHECK(cudaMalloc(&op->d_lex, 2 * vb));
  return static_cast<char*>(op->d_lex) + k * vb;
}

// While alive, vector entry points take lexicographic vectors.
struct LexScope {
  sf_op* op;
  bool prev;
  explicit LexScope(sf_op* o) : op(o), prev(o->lex_inside) { o->lex_inside = true; }
  ~LexScope() { op->lex_inside = prev; }
};

void drop_numbering(sf_op* op) {
  dfree(op->d_numbering);
  op->d_numbering = nullptr;
  dfree(op->d_numbering_inv);
  op->d_numbering_inv = nullptr;
  dfree(op->d_lex);
  op->d_lex = nullptr;
}

void require_own_numbering(const sf_op* op, const char* what) {
  SF_REQUIRE(!op->d_numbering, SF_ERR_UNSUPPORTED,
             std::string(what) + " does not take an operator with a dof numbering "
                                 "(sf_set_structured_numbering)");
}

void apply_impl(sf_op* op, int dtype, const void* x, void* y, cudaStream_t st) {
  require_ready(op);
  const size_t es = dsize(dtype);
  if (op->n_free == 0) return;
  SF_REQUIRE(x && y, SF_ERR_ARG, "null x or y");
  SF_REQUIRE(x != y, SF_ERR_ARG, "x and y must not alias");
  const bool fused = op->numbered_fused == 1 || (op->numbered_fused < 0 && op->numbering_local);
  if (numbered(op) && fused && op->cartesian_ok && sf::cartesian_supported(op->cart, dtype) &&
      op->D == 3 && !op->slab) {  // the tiled kernel reads and writes through the numbering
    sf::CartFuse fuse;
    fuse.num = op->d_numbering;
    sf::cartesian_apply(op->cart, dtype, x, y, st, fuse);
    return;
  }
  if (numbered(op)) {  // into lexicographic order, apply, back
    void* xl = lex_vec(op, 0);
    void* yl = lex_vec(op, 1);
    sf::permute_gather(dtype, x, op->d_numbering, xl, op->n_free, st);
    {
      LexScope lex(op);
      apply_impl(op, dtype, xl, yl, st);
    }
    sf::permute_gather(dtype, yl, op->d_numbering_inv, y, op->n_free, st);
    return;
  }
  if (op->cartesian_ok && sf::cartesian_supported(op->cart, dtype)) {
    sf::cartesian_apply(op->cart, dtype, x, y, st);
    return;
  }
  SF_REQUIRE(!op->slab, SF_ERR_UNSUPPORTED,
             "a slab operator needs the tiled Cartesian kernel (axis-aligned affine cells, "
             "constant coefficient)");
  SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED,
             "D = 2 runs on the tiled Cartesian kernel only (axis-aligned affine cells, "
             "constant coefficient)");
  SF_CUDA_CHECK(cudaMemsetAsync(y, 0, op->n_free * es, st));
  sf::launch_general_apply(dtype, op->SB, op->SQ, op->A.data(), op->B.data(), op->cells, op->geom,
                           x, y, st);
}

// diag(A) into d (n_free FP64, zeroed first): the Kronecker form on Cartesian
// operators, the element kernel otherwise.
void compute_diag(sf_op* op, double* d, cudaStream_t st) {
  SF_CUDA_CHECK(cudaMemsetAsync(d, 0, op->n_free * sizeof(double), st));
  if (op->cartesian_ok) {
    sf::cartesian_diag(op->cart, d, st);
    return;
  }
  SF_REQUIRE(!op->slab, SF_ERR_UNSUPPORTED, "a slab operator needs the tiled Cartesian kernel");
  SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED, "D = 2 runs on the tiled Cartesian kernel only");
  sf::launch_general_diag(SF_F64, op->SB, op->SQ, op->A.data(), op->B.data(), op->cells, op->geom,
                          d, st);
}

void ensure_diag(sf_op* op, cudaStream_t st) {
  if (op->d_diag) return;
  op->d_diag = dalloc<double>(op->n_free);
  compute_diag(op, op->d_diag, st);
}

// The points a slab operator owns: the planes after the lower halo plane, up to
// the upper halo (the top plane left out when it is the Dirichlet boundary).
long long owned_offset(const sf_op* op) { return op->slab ? op->plane : 0; }
long long owned_count(const sf_op* op) {
  if (!op->slab) return op->n_free;
  const long long planes = (long long)(op->slab_z1 - op->slab_z0) * op->p -
                           (op->slab_z1 == op->mesh_nz ? 1 : 0);
  return planes * op->plane;
}

bool host_pinned(const void* p) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // pageable memory on older runtimes reports an error; clear it
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// sf_mul_host on the tiled Cartesian kernel with pinned host buffers: the z-levels
// are copied in, applied and copied out in groups of tile rows on three streams,
// so the two PCIe directions and the apply overlap. Group g can run once the levels
// its tiles read (up to one cell above its last row) are on the device, and its
// owned levels go back as soon as it is done. Returns false when it does not apply.
bool mul_host_pipelined(sf_op* op, const double* x, double* y) {
  if (!(op->cartesian_ok && sf::cartesian_supported(op->cart, SF_F64)) || op->slab || op->D != 3 ||
      op->d_numbering)
    return false;
  if (!host_pinned(x) || !host_pinned(y)) return false;
  const int P = op->p, nz = op->cells.nz;
  const int ez = sf::cartesian_tile_ez(op->cart, SF_F64);
  const int ntz = (nz + ez - 1) / ez;
  const int groups = std::min(op->host_groups, ntz);
  if (groups < 2) return false;
  const long long plane = op->plane, nfz = (long long)nz * P - 1;
  for (cudaStream_t& q : op->pipe)
    if (!q) SF_CUDA_CHECK(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
  while ((int)op->pipe_ev.size() < 2 * groups) {
    cudaEvent_t e;
    SF_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    op->pipe_ev.push_back(e);
  }
  cudaStream_t s_in = op->pipe[0], s_cmp = op->pipe[1], s_out = op->pipe[2];
  long long copied = 0;  // planes [0, copied) of x are on their way to the device
  for (int g = 0; g < groups; ++g) {
    const int r0 = (int)((long long)ntz * g / groups), r1 = (int)((long long)ntz * (g + 1) / groups);
    const long long need = std::min(nfz, (long long)(r1 * ez + 1) * P);  // input planes read
    if (need > copied) {
      SF_CUDA_CHECK(cudaMemcpyAsync(op->d_hx + copied * plane, x + copied * plane,
                                    (size_t)((need - copied) * plane) * sizeof(double),
                                    cudaMemcpyHostToDevice, s_in));
      copied = need;
    }
    SF_CUDA_CHECK(cudaEventRecord(op->pipe_ev[2 * g], s_in));
    SF_CUDA_CHECK(cudaStreamWaitEvent(s_cmp, op->pipe_ev[2 * g], 0));
    sf::CartFuse rows;
    rows.tz0 = r0;
    rows.tz1 = r1;
    sf::cartesian_apply(op->cart, SF_F64, op->d_hx, op->d_hy, s_cmp, rows);
    SF_CUDA_CHECK(cudaEventRecord(op->pipe_ev[2 * g + 1], s_cmp));
    SF_CUDA_CHECK(cudaStreamWaitEvent(s_out, op->pipe_ev[2 * g + 1], 0));
    const long long o0 = (long long)r0 * ez * P, o1 = std::min(nfz, (long long)r1 * ez * P);
    if (o1 > o0)
      SF_CUDA_CHECK(cudaMemcpyAsync(y + o0 * plane, op->d_hy + o0 * plane,
                                    (size_t)((o1 - o0) * plane) * sizeof(double),
                                    cudaMemcpyDeviceToHost, s_out));
  }
  SF_CUDA_CHECK(cudaStreamSynchronize(s_out));
  SF_CUDA_CHECK(cudaStreamSynchronize(s_cmp));
  SF_CUDA_CHECK(cudaStreamSynchronize(s_in));
  return true;
}

// 1 / diag(A) on the owned points (zero elsewhere), cached.
const double* ensure_dinv(sf_op* op, cudaStream_t st) {
  if (op->d_dinv) return op->d_dinv;
  ensure_diag(op, st);
  op->d_dinv = dalloc<double>(op->n_free);
  SF_CUDA_CHECK(cudaMemsetAsync(op->d_dinv, 0, op->n_free * sizeof(double), st));
  const long long off = owned_offset(op);
  sf::vec_invert<double>(op->d_diag + off, op->d_dinv + off, owned_count(op), st);
  return op->d_dinv;
}

void invalidate_caches(sf_op* op) {
  dfree(op->d_diag);
  op->d_diag = nullptr;
  dfree(op->d_jtab);
  op->d_jtab = nullptr;
  dfree(op->d_dinv);
  op->d_dinv = nullptr;
}

void* workspace(sf_op* op, size_t bytes) {
  if (op->ws_bytes < bytes) {
    dfree(op->d_ws);
    op->d_ws = nullptr;
    op->ws_bytes = 0;
    SF_CUDA_CHECK(cudaMalloc(&op->d_ws, bytes));
    op->ws_bytes = bytes;
  }
  return op->d_ws;
}

double read_scalar(sf_op* op, const double* d_s, int slot, cudaStream_t st) {
  if (!op->h_scalar) SF_CUDA_CHECK(cudaMallocHost(&op->h_scalar, 8 * sizeof(double)));
  SF_CUDA_CHECK(cudaMemcpyAsync(op->h_scalar, d_s + slot, sizeof(double), cudaMemcpyDeviceToHost, st));
  SF_CUDA_CHECK(cudaStreamSynchronize(st));
  return op->h_scalar[0];
}

size_t align256(size_t b) { return (b + 255) & ~size_t(255); }

// The host reads the CG progress reports kCgLag iterations behind the last
// queued iteration, so the device always has work queued and no iteration
// waits on the host. The device writes each report into mapped host memory
// (no copy or event in the stream).
constexpr int kCgLag = 2;
constexpr int kStateWords = sf::CG_TOL2 - sf::CG_RR + 1;  // RR, BB, DONE, ITERS, TOL2

// Clears the report buffer (allocated on first use); call with nothing of an
// earlier solve in flight.
void reset_reports(sf_op* op) {
  if (!op->h_report) {
    SF_CUDA_CHECK(cudaHostAlloc(&op->h_report, 8 * sizeof(double), cudaHostAllocMapped));
    void* d = nullptr;
    SF_CUDA_CHECK(cudaHostGetDevicePointer(&d, op->h_report, 0));
    op->d_report = static_cast<double*>(d);
  }
  for (int k = 0; k < 8; ++k) op->h_report[k] = 0.0;
}

struct Report {
  double rr, done, iters;
};

// Waits for report number k (or a later one) and returns it. Gives up with an
// error if the stream ends or fails without it, or after kReportWaitSeconds.
constexpr double kReportWaitSeconds = 600.0;

Report wait_report(sf_op* op, int k, cudaStream_t st) {
  volatile const double* r = op->h_report;
  const auto t0 = std::chrono::steady_clock::now();
  for (unsigned spin = 1; r[3] < k; ++spin) {
    if ((spin & 255) == 0) {
      const cudaError_t e = cudaStreamQuery(st);
      if (e == cudaSuccess && r[3] < k)
        throw Error(SF_ERR_STATE, "CG progress report missing");
      if (e != cudaSuccess && e != cudaErrorNotReady) SF_CUDA_CHECK(e);
      if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() >
          kReportWaitSeconds)
        throw Error(SF_ERR_CUDA, "no CG progress from the device within the wait limit");
      std::this_thread::yield();
    }
  }
  std::atomic_thread_fence(std::memory_order_acquire);
  return Report{r[0], r[1], r[2]};
}

// Scalars RR.. now (synchronises the stream).
const double* read_state(sf_op* op, const double* s, cudaStream_t st) {
  if (!op->h_scalar) SF_CUDA_CHECK(cudaMallocHost(&op->h_scalar, 8 * sizeof(double)));
  SF_CUDA_CHECK(cudaMemcpyAsync(op->h_scalar, s + sf::CG_RR, kStateWords * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
  SF_CUDA_CHECK(cudaStreamSynchronize(st));
  return op->h_scalar;
}

constexpr int kRR = 0, kBB = sf::CG_BB - sf::CG_RR, kDone = sf::CG_DONE - sf::CG_RR,
              kIters = sf::CG_ITERS - sf::CG_RR;

// The 3D tiled kernel, whose store phase can also form the CG's (p, Ap) partial sums.
bool tiled(const sf_op* op, int dtype) {
  return op->cartesian_ok && op->D == 3 && sf::cartesian_supported(op->cart, dtype);
}

// Partial-sum entries the CG reductions of this operator need.
long long cg_partials(const sf_op* op) {
  long long n = 3LL * sf::kRedBlocks;
  for (int dt : {SF_F64, SF_F32})
    if (tiled(op, dt)) n = std::max(n, sf::cartesian_tiles(op->cart, dt));
  return n;
}

// q = A p and s[PQ] = (p, q). The apply itself always runs (after convergence
// its result is not used); the sum is skipped once s[DONE] != 0. The tiled
// kernel forms per-tile partial sums in its store phase.
template <typename T>
void apply_pq(sf_op* op, const T* p, T* q, double* partials, double* s, cudaStream_t st) {
  const int dtype = sizeof(T) == 8 ? SF_F64 : SF_F32;
  if (tiled(op, dtype)) {
    sf::CartFuse fuse;
    fuse.dot = partials;
    sf::cartesian_apply(op->cart, dtype, p, q, st, fuse);
    sf::dot_finish(partials, sf::cartesian_tiles(op->cart, dtype), s + sf::CG_PQ,
                   s + sf::CG_DONE, st);
  } else {
    apply_impl(op, dtype, p, q, st);
    sf::vec_dot<T>(p, q, op->n_free, partials, s + sf::CG_PQ, s, s + sf::CG_DONE, st);
  }
}

// D^-1 of a whole-mesh 3D Cartesian operator as a p^3 table (sf::JacobiTable), or
// p = 0 where there is none (the CG then reads a D^-1 vector). The table is the
// Kronecker-form diagonal of cartesian_diag, inverted, per position in a cell.
sf::JacobiTable jacobi_table(sf_op* op) {
  sf::JacobiTable J;
  if (!op->jacobi_table || op->slab || !tiled(op, SF_F64)) return J;
  const int P = op->SB - 1;
  if (!op->d_jtab) {
    const int SB = op->SB;
    const double* M = op->cart.M;
    const double* K = op->cart.K;
    auto d1 = [&](const double* D, int l) { return l == 0 ? D[0] + D[P * SB + P] : D[l * SB + l]; };
    std::vector<double> tab((size_t)P * P * P);
    for (int lz = 0; lz < P; ++lz)
      for (int ly = 0; ly < P; ++ly)
        for (int lx = 0; lx < P; ++lx) {
          const double d = op->cart.c[0] * d1(K, lx) * d1(M, ly) * d1(M, lz) +
                           op->cart.c[1] * d1(M, lx) * d1(K, ly) * d1(M, lz) +
                           op->cart.c[2] * d1(M, lx) * d1(M, ly) * d1(K, lz);
          tab[((size_t)lz * P + ly) * P + lx] = 1.0 / d;
        }
    op->d_jtab = dalloc<double>(tab.size());
    SF_CUDA_CHECK(cudaMemcpy(op->d_jtab, tab.data(), tab.size() * sizeof(double),
                             cudaMemcpyHostToDevice));
  }
  J.tab = op->d_jtab;
  J.p = P;
  J.nfx = op->cells.nx * P - 1;
  J.nfy = op->cells.ny * P - 1;
  return J;
}

// Plain or Jacobi FP64 CG. Returns iterations; sets relres.
int cg_f64(sf_op* op, bool jacobi, const double* b, double* x, double reltol, int maxiter,
           double* relres, cudaStream_t st) {
  const long long n = op->n_free;
  const size_t vb = align256(n * sizeof(double));
  const size_t sb = align256(sf::CG_NSLOTS * sizeof(double));
  const size_t pb = align256(cg_partials(op) * sizeof(double));
  char* ws = static_cast<char*>(workspace(op, 4 * vb + sb + pb));
  double* r = reinterpret_cast<double*>(ws);
  double* p = reinterpret_cast<double*>(ws + vb);
  double* q = reinterpret_cast<double*>(ws + 2 * vb);
  double* dinv = reinterpret_cast<double*>(ws + 3 * vb);
  double* s = reinterpret_cast<double*>(ws + 4 * vb);
  double* partials = reinterpret_cast<double*>(ws + 4 * vb + sb);
  if (jacobi) {
    ensure_diag(op, st);
    sf::vec_invert<double>(op->d_diag, dinv, n, st);
  }
  const double* Dv = jacobi ? dinv : nullptr;
  const sf::JacobiTable J = jacobi ? jacobi_table(op) : sf::JacobiTable{};
  sf::cg_reset(s, st);
  apply_impl(op, SF_F64, x, q, st);
  sf::cg_start<double>(b, q, Dv, r, p, n, partials, s, st);
  sf::cg_init(s, reltol * reltol, st);
  const double* h = read_state(op, s, st);
  const double bb = h[kBB];
  const double nb = std::sqrt(bb) > 0 ? std::sqrt(bb) : 1.0;
  double done = h[kDone];
  reset_reports(op);
  for (int it = 0; it < maxiter && done == 0.0;) {
    apply_pq<double>(op, p, q, partials, s, st);
    if (J.p > 0) {  // D^-1 from the table: two vector sweeps fewer
      sf::cg_update_table<double>(s, r, q, J, n, partials, st);
      sf::cg_direction_table<double>(s, x, p, r, J, n, op->d_report, st);
    } else {
      sf::cg_update<double>(s, r, q, Dv, n, partials, st);
      sf::cg_direction<double>(s, x, p, r, Dv, n, op->d_report, st);
    }
    ++it;
    if (it > kCgLag) done = wait_report(op, it - kCgLag, st).done;
  }
  h = read_state(op, s, st);
  SF_REQUIRE(h[kDone] != 3.0, SF_ERR_NONFINITE, "non-finite residual in CG");
  *relres = std::sqrt(h[kRR]) / nb;
  return (int)h[kIters];
}

// Mixed-precision Jacobi CG with reliable updates. The CG recurrence (p, q,
// r, the partial solution xs) runs in FP32 with the FP32 apply; dot products
// accumulate in FP64. Whenever the FP32 residual has dropped by the factor
// `mixed_inner_reltol` since the last update (or below the target), the
// partial solution is folded into the FP64 solution x, and the FP64 true
// residual b - A64 x replaces r. The search direction is kept, so the Krylov
// recurrence is not restarted. The stopping test uses the FP64 true residual
// only. The host reads the FP32 residual kCgLag iterations late, so an update
// comes up to kCgLag iterations after the drop that triggers it.
int cg_mixed(sf_op* op, const double* b, double* x, double reltol, int maxiter, double* relres,
             int* outer_out, cudaStream_t st) {
  const long long n = op->n_free;
  const size_t v8 = align256(n * sizeof(double));
  const size_t v4 = align256(n * sizeof(float));
  const size_t sb = align256(sf::CG_NSLOTS * sizeof(double));
  const size_t pb = align256(cg_partials(op) * sizeof(double));
  char* ws = static_cast<char*>(workspace(op, v8 + 5 * v4 + sb + pb));
  double* q64 = reinterpret_cast<double*>(ws);
  char* w4 = ws + v8;
  float* xs32 = reinterpret_cast<float*>(w4);
  float* r32 = reinterpret_cast<float*>(w4 + v4);
  float* p32 = reinterpret_cast<float*>(w4 + 2 * v4);
  float* q32 = reinterpret_cast<float*>(w4 + 3 * v4);
  float* dinv32 = reinterpret_cast<float*>(w4 + 4 * v4);
  double* s = reinterpret_cast<double*>(ws + v8 + 5 * v4);
  double* partials = reinterpret_cast<double*>(ws + v8 + 5 * v4 + sb);
  ensure_diag(op, st);
  sf::vec_invert<float>(op->d_diag, dinv32, n, st);
  sf::cg_reset(s, st);
  sf::vec_dot<double>(b, b, n, partials, s + sf::CG_BB, s, nullptr, st);
  // true residual of the initial guess; p = dinv r; the device never stops on its own
  apply_impl(op, SF_F64, x, q64, st);
  sf::mixed_residual(b, q64, dinv32, r32, xs32, p32, true, n, partials, s, st);
  sf::cg_init(s, -1.0, st);
  const double* h = read_state(op, s, st);
  const double bb = h[kBB];
  const double nb = std::sqrt(bb) > 0 ? std::sqrt(bb) : 1.0;
  const double tol2 = reltol * reltol * (bb > 0 ? bb : 1.0);
  const double delta2 = op->mixed_inner_reltol * op->mixed_inner_reltol;
  double rr64 = h[kRR];
  SF_REQUIRE(std::isfinite(rr64), SF_ERR_NONFINITE, "non-finite residual in mixed CG");
  double rr_ref = rr64;
  int it = 0, updates = 0, last_update = 0;
  bool dirty = false;  // xs32 holds a partial solution not yet folded into x
  reset_reports(op);
  while (rr64 > tol2 && it < maxiter) {
    apply_pq<float>(op, p32, q32, partials, s, st);
    // D^-1 from the FP32 vector: at 4 bytes per element the table's index arithmetic
    // costs more than the vector sweep it saves (measured)
    sf::cg_update<float>(s, r32, q32, dinv32, n, partials, st);
    sf::cg_direction<float>(s, xs32, p32, r32, dinv32, n, op->d_report, st);
    ++it;
    dirty = true;
    bool refine = it >= maxiter;
    if (it - kCgLag > last_update) {  // residuals from before the last update do not count
      const Report rep = wait_report(op, it - kCgLag, st);
      SF_REQUIRE(rep.done != 3.0, SF_ERR_NONFINITE, "non-finite residual in mixed CG");
      refine = refine || rep.rr <= delta2 * rr_ref || rep.rr <= tol2;
    }
    if (refine) {
      // reliable update: fold xs into x, replace r by the FP64 true residual
      sf::mixed_fold(x, xs32, n, st);
      apply_impl(op, SF_F64, x, q64, st);
      sf::mixed_residual(b, q64, dinv32, r32, xs32, p32, false, n, partials, s, st);
      sf::copy_scalar(s, sf::CG_RZ, sf::CG_RZ_NEW, st);
      rr64 = read_state(op, s, st)[kRR];
      SF_REQUIRE(std::isfinite(rr64), SF_ERR_NONFINITE, "non-finite residual in mixed CG");
      rr_ref = rr64;
      last_update = it;
      dirty = false;
      ++updates;
    }
  }
  if (dirty) sf::mixed_fold(x, xs32, n, st);
  *relres = std::sqrt(rr64) / nb;
  *outer_out = updates;
  return it;
}

// Fastest of nc candidates: run(k) is launched twice untimed, then timed over five launches.
template <typename F>
int fastest(int nc, cudaStream_t st, const F& run) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&] {
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  int best = 0;
  try {
    SF_CUDA_CHECK(cudaEventCreate(&e0));
    SF_CUDA_CHECK(cudaEventCreate(&e1));
    float best_ms = 0.f;
    for (int k = 0; k < nc; ++k) {
      for (int w = 0; w < 2; ++w) run(k);
      SF_CUDA_CHECK(cudaEventRecord(e0, st));
      for (int r = 0; r < 5; ++r) run(k);
      SF_CUDA_CHECK(cudaEventRecord(e1, st));
      SF_CUDA_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      SF_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      if (k == 0 || ms < best_ms) {
        best = k;
        best_ms = ms;
      }
    }
  } catch (...) {
    cleanup();
    throw;
  }
  cleanup();
  return best;
}

// Device buffers freed on scope exit.
struct Scratch {
  std::vector<void*> bufs;
  void* get(size_t bytes) {
    void* p = nullptr;
    SF_CUDA_CHECK(cudaMalloc(&p, bytes));
    bufs.push_back(p);
    return p;
  }
  ~Scratch() {
    for (void* p : bufs) cudaFree(p);
  }
};

}  // namespace

extern "C" {

int sf_version(void) { return 100; }

const char* sf_status_string(int status) {
  switch (status) {
    case SF_OK: return "ok";
    case SF_ERR_ARG: return "invalid argument";
    case SF_ERR_CUDA: return "CUDA error";
    case SF_ERR_STATE: return "handle not set up";
    case SF_ERR_UNSUPPORTED: return "unsupported";
    case SF_ERR_NOT_CONVERGED: return "not converged";
    case SF_ERR_NONFINITE: return "non-finite value";
    default: return "unknown status";
  }
}

int sf_create(sf_op** out, int D, int SB, int SQ, const double* A0, const double* B0,
              const int32_t* dof_map) {
  if (!out) return SF_ERR_ARG;
  *out = nullptr;
  if (D != 2 && D != 3) return SF_ERR_UNSUPPORTED;
  if (SB < 2 || SB > sf::kMaxSB || SQ < 1 || SQ > sf::kMaxSQ || !A0 || !B0 || !dof_map)
    return SF_ERR_ARG;
  sf_op* op = new (std::nothrow) sf_op();
  if (!op) return SF_ERR_ARG;
  op->D = D;
  op->SB = SB;
  op->SQ = SQ;
  op->p = SB - 1;
  op->A_user.resize(SQ * SB);
  op->B_user.resize(SQ * SB);
  for (int q = 0; q < SQ; ++q)
    for (int j = 0; j < SB; ++j) {
      op->A_user[q * SB + j] = A0[q + SQ * j];  // column-major in
      op->B_user[q * SB + j] = B0[q + SQ * j];
    }
  const int nloc = D == 2 ? SB * SB : SB * SB * SB;
  op->jt_user.resize(nloc * D);
  for (int k = 0; k < nloc; ++k)
    for (int d = 0; d < D; ++d) {
      const int v = dof_map[k + nloc * d] - 1;  // column-major, 1-based
      if (v < 0 || v >= SB) {
        delete op;
        return SF_ERR_ARG;
      }
      op->jt_user[k * D + d] = v;
    }
  op->perm.resize(SB);
  for (int j = 0; j < SB; ++j) op->perm[j] = j;
  int st = guarded(op, [&] { rebuild_kernel_basis(op); });
  if (st != SF_OK) {
    sf_destroy(op);
    return st;
  }
  *out = op;
  return SF_OK;
}

int sf_destroy(sf_op* op) {
  if (!op) return SF_OK;
  dfree(op->d_ids);
  dfree(op->d_t2l);
  dfree(op->d_gtab);
  dfree(op->d_gtab32);
  dfree(op->d_wdet);
  dfree(op->d_kappa);
  dfree(op->d_diag);
  dfree(op->d_jtab);
  dfree(op->d_dinv);
  drop_numbering(op);
  dfree(op->d_ws);
  dfree(op->d_hx);
  dfree(op->d_hy);
  if (op->h_scalar) cudaFreeHost(op->h_scalar);
  if (op->h_report) cudaFreeHost(op->h_report);
  for (cudaStream_t q : op->pipe)
    if (q) cudaStreamDestroy(q);
  for (cudaEvent_t e : op->pipe_ev) cudaEventDestroy(e);
  sf::cartesian_release(op->cart);
  delete op;
  return SF_OK;
}

const char* sf_last_error(const sf_op* op) { return op ? op->err.c_str() : "null handle"; }

int sf_get_dimensional_parameters(const sf_op* op, int* D, int* SB, int* SQ) {
  if (!op) return SF_ERR_ARG;
  if (D) *D = op->D;
  if (SB) *SB = op->SB;
  if (SQ) *SQ = op->SQ;
  return SF_OK;
}

int sf_set_cells(sf_op* op, int64_t ncells, const int32_t* ptrs, const int32_t* data,
                 int64_t n_free) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED,
               "D = 2 takes the structured Cartesian path (sf_set_structured) only");
    SF_REQUIRE(ncells >= 0 && n_free >= 0 && (ncells == 0 || (ptrs && data)), SF_ERR_ARG,
               "bad arguments to sf_set_cells");
    SF_REQUIRE(n_free < (1LL << 31), SF_ERR_ARG, "n_free must fit in int32");
    const int nloc = op->SB * op->SB * op->SB;
    for (int j = 0; j < op->SB; ++j) op->perm[j] = j;
    rebuild_kernel_basis(op);
    std::vector<int> tpos(nloc);
    for (int k = 0; k < nloc; ++k) tpos[k] = tensor_pos(op, k);
    std::vector<int32_t> ids((size_t)ncells * nloc);
    for (int64_t c = 0; c < ncells; ++c) {
      const int64_t b = (int64_t)ptrs[c] - 1, e = (int64_t)ptrs[c + 1] - 1;
      SF_REQUIRE(e - b == nloc, SF_ERR_ARG,
                 "cell " + std::to_string(c + 1) + " does not have SB^D dofs");
      for (int k = 0; k < nloc; ++k) {
        const int32_t id = data[b + k];
        SF_REQUIRE(id != 0 && id <= n_free, SF_ERR_ARG,
                   "dof id out of range in cell " + std::to_string(c + 1));
        ids[(size_t)c * nloc + tpos[k]] = id > 0 ? id - 1 : -1;
      }
    }
    dfree(op->d_ids);
    drop_numbering(op);
    op->d_ids = nullptr;
    op->d_ids = dalloc<int32_t>(ids.size());
    SF_CUDA_CHECK(cudaMemcpy(op->d_ids, ids.data(), ids.size() * sizeof(int32_t),
                             cudaMemcpyHostToDevice));
    op->cells = sf::Cells();
    op->cells.mesh = sf::MESH_CSR;
    op->cells.ncells = ncells;
    op->cells.ids = op->d_ids;
    op->cells.p = op->p;
    op->n_free = n_free;
    invalidate_caches(op);
    update_cartesian(op);
  });
}

int sf_set_structured(sf_op* op, int nx, int ny, int nz, const int32_t* node_order) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(nx > 0 && ny > 0 && (op->D == 2 ? nz == 0 : nz > 0) && node_order, SF_ERR_ARG,
               "bad arguments to sf_set_structured (nz = 0 for D = 2)");
    std::vector<int> seen(op->SB, 0);
    for (int j = 0; j < op->SB; ++j) {
      SF_REQUIRE(node_order[j] >= 0 && node_order[j] < op->SB && !seen[node_order[j]], SF_ERR_ARG,
                 "node_order must be a permutation of 0..p");
      seen[node_order[j]] = 1;
    }
    const long long p = op->p;
    const long long fx = nx * p - 1, fy = ny * p - 1, fz = op->D == 2 ? 1 : nz * p - 1;
    SF_REQUIRE(fx * fy * fz < (1LL << 31), SF_ERR_ARG, "mesh too large for int32 dof ids");
    for (int j = 0; j < op->SB; ++j) op->perm[j] = node_order[j];
    rebuild_kernel_basis(op);
    dfree(op->d_ids);
    op->d_ids = nullptr;
    drop_numbering(op);
    op->cells = sf::Cells();
    op->cells.mesh = sf::MESH_STRUCTURED;
    op->cells.ncells = (long long)nx * ny * (op->D == 2 ? 1 : nz);
    op->cells.nx = nx;
    op->cells.ny = ny;
    op->cells.nz = nz;
    op->cells.p = op->p;
    op->n_free = fx * fy * fz;
    op->slab = false;
    op->plane = fx * fy;
    invalidate_caches(op);
    update_cartesian(op);
  });
}

int sf_set_structured_slab(sf_op* op, int nx, int ny, int nz, int z0, int z1,
                           const int32_t* node_order) {
  if (!op) return SF_ERR_ARG;
  const int status = sf_set_structured(op, nx, ny, z1 > z0 ? z1 - z0 : 1, node_order);
  if (status != SF_OK) return status;
  return guarded(op, [&] {
    SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED, "slabs split a 3D mesh");
    SF_REQUIRE(nz > 0 && z0 >= 0 && z0 < z1 && z1 <= nz, SF_ERR_ARG,
               "slab cells [z0, z1) must lie in [0, nz) and be non-empty");
    const long long p = op->p;
    op->slab = true;
    op->slab_z0 = z0;
    op->slab_z1 = z1;
    op->mesh_nz = nz;
    op->n_free = op->plane * ((long long)(z1 - z0 + 1) * p + 1);
    SF_REQUIRE(op->n_free < (1LL << 31), SF_ERR_ARG, "slab too large for int32 dof ids");
    invalidate_caches(op);
    update_cartesian(op);
  });
}

int sf_set_structured_numbering(sf_op* op, int nx, int ny, int nz, const int32_t* node_order,
                                const int32_t* free_id) {
  if (!op) return SF_ERR_ARG;
  if (op->D != 3) return fail(op, SF_ERR_UNSUPPORTED, "sf_set_structured_numbering is 3D only");
  if (!free_id) return fail(op, SF_ERR_ARG, "null free_id");
  const int status = sf_set_structured(op, nx, ny, nz, node_order);
  if (status != SF_OK) return status;
  return guarded(op, [&] {
    const long long n = op->n_free;
    std::vector<char> seen((size_t)n, 0);
    for (long long i = 0; i < n; ++i) {
      const int32_t k = free_id[i];
      SF_REQUIRE(k >= 0 && k < n && !seen[(size_t)k], SF_ERR_ARG,
                 "free_id must be a permutation of 0 .. n_free-1 (entry " + std::to_string(i) + ")");
      seen[(size_t)k] = 1;
    }
    // back to the caller's numbering as a gather by the inverse: scattered reads cost
    // less than scattered partial-sector writes when the numbering has no locality
    std::vector<int32_t> inv((size_t)n);
    for (long long i = 0; i < n; ++i) inv[(size_t)free_id[i]] = (int32_t)i;
    // locality: the share of x-neighbours whose ids lie within 64 of each other. Reading
    // and writing through the numbering inside the tiled kernel pays when most do (a
    // cell-by-cell numbering: 0.8-1.0); a numbering without locality (random: about 0.01)
    // is cheaper to permute as a whole into lexicographic order and back
    const long long fx = (long long)nx * op->p - 1;
    long long near = 0, pairs = 0;
    for (long long i = 0; i + 1 < n; ++i) {
      if ((i + 1) % fx == 0) continue;
      ++pairs;
      if (std::llabs((long long)free_id[i + 1] - free_id[i]) <= 64) ++near;
    }
    op->numbering_local = pairs == 0 || 2 * near >= pairs;
    op->d_numbering = dalloc<int32_t>((size_t)n);
    op->d_numbering_inv = dalloc<int32_t>((size_t)n);
    SF_CUDA_CHECK(cudaMemcpy(op->d_numbering, free_id, (size_t)n * sizeof(int32_t),
                             cudaMemcpyHostToDevice));
    SF_CUDA_CHECK(cudaMemcpy(op->d_numbering_inv, inv.data(), (size_t)n * sizeof(int32_t),
                             cudaMemcpyHostToDevice));
  });
}

int sf_set_cell_quantities(sf_op* op, int fill, const double* wq, const double* jq,
                           const double* djq) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(wq && jq && djq, SF_ERR_ARG, "null cell quantity");
    SF_REQUIRE(fill || op->cells.mesh != sf::MESH_NONE, SF_ERR_STATE,
               "per-cell quantities need the mesh first (sf_set_cells / sf_set_structured)");
    const int SQ = op->SQ, D = op->D;
    const int nq = D == 2 ? SQ * SQ : SQ * SQ * SQ;
    const long long nc = fill ? 1 : op->cells.ncells;
    // G = wq*djq*jq^T jq at every point (src/SumFactorizationKernels.jl:174-216)
    std::vector<double> G((size_t)nc * 6 * nq);
    std::vector<double> H((size_t)nc * 6 * nq);  // djq*jq^T jq (without the weight)
    std::vector<double> WD((size_t)nc * nq);     // wq*djq (the right-hand side's weights)
    static const int rr[6] = {0, 1, 2, 0, 0, 1}, kk[6] = {0, 1, 2, 1, 2, 2};
    for (long long c = 0; c < nc; ++c)
      for (int q = 0; q < nq; ++q) {
        const double* J = jq + ((size_t)c * nq + q) * D * D;
        const double w = wq[(size_t)c * nq + q], dj = djq[(size_t)c * nq + q];
        WD[(size_t)c * nq + q] = w * dj;
        for (int m = 0; m < 6; ++m) {
          double acc = 0.0;  // in 2D the components with a z index stay zero
          if (rr[m] < D && kk[m] < D)
            for (int l = 0; l < D; ++l) acc += J[l + D * rr[m]] * J[l + D * kk[m]];
          H[((size_t)c * 6 + m) * nq + q] = dj * acc;
          G[((size_t)c * 6 + m) * nq + q] = w * dj * acc;
        }
      }
    // all cells equal?
    bool same = true;
    for (long long c = 1; c < nc && same; ++c)
      for (size_t i = 0; i < (size_t)6 * nq; ++i)
        if (G[(size_t)c * 6 * nq + i] != G[i]) {
          same = false;
          break;
        }
    // separable: H constant over points and wq a tensor product of 1D weights
    bool sep = same;
    double Hmax = 0.0;
    for (int m = 0; m < 6; ++m) Hmax = std::max(Hmax, std::fabs(H[(size_t)m * nq]));
    if (Hmax == 0.0) Hmax = 1.0;
    for (int m = 0; m < 6 && sep; ++m)
      for (int q = 1; q < nq; ++q)
        if (std::fabs(H[(size_t)m * nq + q] - H[(size_t)m * nq]) > 1e-13 * Hmax) {
          sep = false;
          break;
        }
    double w1[sf::kMaxSQ] = {0};
    if (sep) {
      const double w000 = wq[0];
      sep = w000 > 0;
      if (sep) {
        // wq = w1 (x) w1 (x) w1 (D = 3) or w1 (x) w1 (D = 2), with w1[0] = c0
        const double c0 = D == 2 ? std::sqrt(w000) : std::cbrt(w000);
        for (int i = 0; i < SQ; ++i) w1[i] = wq[i] / (D == 2 ? c0 : c0 * c0);
        for (int k = 0; k < (D == 2 ? 1 : SQ) && sep; ++k)
          for (int j = 0; j < SQ && sep; ++j)
            for (int i = 0; i < SQ; ++i) {
              const double t = w1[i] * w1[j] * (D == 2 ? 1.0 : w1[k]);
              if (std::fabs(t - wq[i + SQ * (j + SQ * k)]) > 1e-13 * std::fabs(t)) {
                sep = false;
                break;
              }
            }
      }
    }
    dfree(op->d_gtab);
    dfree(op->d_gtab32);
    op->d_gtab = nullptr;
    op->d_gtab32 = nullptr;
    sf::Geometry g;
    g.kappa = op->d_kappa;
    if (sep) {
      g.kind = sf::GEOM_SEPARABLE;
      for (int i = 0; i < SQ; ++i) g.w1[i] = w1[i];
      for (int m = 0; m < 6; ++m) g.G0[m] = H[(size_t)m * nq];
    } else {
      const long long ncopy = same ? 1 : nc;
      op->d_gtab = dalloc<double>((size_t)ncopy * 6 * nq);
      SF_CUDA_CHECK(cudaMemcpy(op->d_gtab, G.data(), (size_t)ncopy * 6 * nq * sizeof(double),
                               cudaMemcpyHostToDevice));
      g.kind = sf::GEOM_TABLE;
      g.table = op->d_gtab;
      g.table_stride = same ? 0 : 6LL * nq;
      // the FP32 copy, each cell's rows padded to 16 bytes
      const long long s32 = same ? 0 : (6LL * nq + 3) / 4 * 4;
      const long long n32 = same ? 6LL * nq : ncopy * s32;
      op->d_gtab32 = dalloc<float>((size_t)n32);
      SF_CUDA_CHECK(cudaMemset(op->d_gtab32, 0, (size_t)n32 * sizeof(float)));
      sf::convert_table32(op->d_gtab, ncopy, 6 * nq, same ? 0 : s32, op->d_gtab32, nullptr);
      SF_CUDA_CHECK(cudaDeviceSynchronize());
      g.table32 = op->d_gtab32;
      g.table32_stride = s32;
    }
    bool wsame = true;
    for (long long c = 1; c < nc && wsame; ++c)
      for (int q = 0; q < nq; ++q)
        if (WD[(size_t)c * nq + q] != WD[q]) {
          wsame = false;
          break;
        }
    dfree(op->d_wdet);
    op->d_wdet = nullptr;
    const long long nw = wsame ? 1 : nc;
    op->d_wdet = dalloc<double>((size_t)nw * nq);
    SF_CUDA_CHECK(cudaMemcpy(op->d_wdet, WD.data(), (size_t)nw * nq * sizeof(double),
                             cudaMemcpyHostToDevice));
    g.wdet = op->d_wdet;
    g.wdet_stride = wsame ? 0 : nq;
    op->geom = g;
    op->cq_cells = (fill || same) ? 0 : nc;
    invalidate_caches(op);
    update_cartesian(op);
  });
}

int sf_set_coefficient(sf_op* op, const double* kappa) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    dfree(op->d_kappa);
    op->d_kappa = nullptr;
    if (kappa) {
      SF_REQUIRE(op->cells.mesh != sf::MESH_NONE, SF_ERR_STATE, "set the mesh before kappa");
      const size_t n = (size_t)op->cells.ncells * op->SQ * op->SQ * op->SQ;
      op->d_kappa = dalloc<double>(n);
      SF_CUDA_CHECK(cudaMemcpy(op->d_kappa, kappa, n * sizeof(double), cudaMemcpyHostToDevice));
    }
    op->geom.kappa = op->d_kappa;
    invalidate_caches(op);
    update_cartesian(op);
  });
}

int sf_set_coefficient_device(sf_op* op, const double* kappa, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(kappa, SF_ERR_ARG, "null kappa (use sf_set_coefficient(op, NULL) to clear)");
    SF_REQUIRE(op->cells.mesh != sf::MESH_NONE, SF_ERR_STATE, "set the mesh before kappa");
    const size_t n = (size_t)op->cells.ncells * op->SQ * op->SQ * op->SQ;
    if (!op->d_kappa) op->d_kappa = dalloc<double>(n);
    SF_CUDA_CHECK(cudaMemcpyAsync(op->d_kappa, kappa, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                  static_cast<cudaStream_t>(stream)));
    op->geom.kappa = op->d_kappa;
    invalidate_caches(op);
    update_cartesian(op);
  });
}

int sf_kappa_vjp(sf_op* op, int dtype, const void* x, const void* ybar, double* kappa_bar,
                 void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(!op->slab, SF_ERR_UNSUPPORTED, "sf_kappa_vjp does not take slab operators");
    require_own_numbering(op, "sf_kappa_vjp");
    SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED, "sf_kappa_vjp is 3D only");
    SF_REQUIRE(x && ybar && kappa_bar, SF_ERR_ARG, "null x, ybar or kappa_bar");
    sf::launch_kappa_vjp(dtype, op->SB, op->SQ, op->A.data(), op->B.data(), op->cells, op->geom, x,
                         ybar, kappa_bar, static_cast<cudaStream_t>(stream));
  });
}

int sf_apply(sf_op* op, int dtype, const void* x, void* y, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] { apply_impl(op, dtype, x, y, static_cast<cudaStream_t>(stream)); });
}

int sf_apply_multi(sf_op* op, int dtype, int nrhs, const void* x, int64_t ldx, void* y,
                   int64_t ldy, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(nrhs >= 0 && ldx >= op->n_free && ldy >= op->n_free, SF_ERR_ARG,
               "bad nrhs / leading dimensions");
    const size_t es = dsize(dtype);
    for (int k = 0; k < nrhs; ++k)
      apply_impl(op, dtype, static_cast<const char*>(x) + (size_t)k * ldx * es,
                 static_cast<char*>(y) + (size_t)k * ldy * es, static_cast<cudaStream_t>(stream));
  });
}

int sf_mul_host(sf_op* op, const double* x, double* y) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(x && y, SF_ERR_ARG, "null x or y");
    const size_t bytes = op->n_free * sizeof(double);
    if (op->h_n != op->n_free) {
      dfree(op->d_hx);
      dfree(op->d_hy);
      op->d_hx = op->d_hy = nullptr;
      op->h_n = 0;
      op->d_hx = dalloc<double>(op->n_free);
      op->d_hy = dalloc<double>(op->n_free);
      op->h_n = op->n_free;
    }
    if (mul_host_pipelined(op, x, y)) return;
    cudaStream_t st = 0;
    SF_CUDA_CHECK(cudaMemcpyAsync(op->d_hx, x, bytes, cudaMemcpyHostToDevice, st));
    apply_impl(op, SF_F64, op->d_hx, op->d_hy, st);
    SF_CUDA_CHECK(cudaMemcpyAsync(y, op->d_hy, bytes, cudaMemcpyDeviceToHost, st));
    SF_CUDA_CHECK(cudaStreamSynchronize(st));
  });
}

int sf_evaluate_cells(sf_op* op, int dtype, int64_t ncells, const void* x_cells, void* y_cells,
                      void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(op->geom.kind != sf::GEOM_NONE, SF_ERR_STATE, "no geometry");
    SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED, "sf_evaluate_cells is 3D only");
    SF_REQUIRE(ncells >= 0, SF_ERR_ARG, "ncells < 0");
    SF_REQUIRE(op->cq_cells <= 0 || op->cq_cells == ncells, SF_ERR_ARG,
               "ncells differs from the cell quantities");
    SF_REQUIRE(op->geom.kappa == nullptr || ncells == op->cells.ncells, SF_ERR_ARG,
               "ncells differs from the coefficient field");
    if (ncells == 0) return;
    SF_REQUIRE(x_cells && y_cells, SF_ERR_ARG, "null x_cells or y_cells");
    sf::launch_general_evaluate(dtype, op->SB, op->SQ, op->A.data(), op->B.data(), ncells,
                                op->d_t2l, op->geom, x_cells, y_cells,
                                static_cast<cudaStream_t>(stream));
  });
}

int sf_rhs(sf_op* op, const double* fq, double* b, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(fq && b, SF_ERR_ARG, "null fq or b");
    SF_REQUIRE(!op->slab, SF_ERR_UNSUPPORTED, "sf_rhs does not take slab operators");
    SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED, "sf_rhs is 3D only");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (numbered(op)) {  // in lexicographic order, then into the caller's numbering
      double* bl = static_cast<double*>(lex_vec(op, 0));
      {
        LexScope lex(op);
        check_status(sf_rhs(op, fq, bl, stream), op);
      }
      sf::permute_gather(SF_F64, bl, op->d_numbering_inv, b, op->n_free, st);
      return;
    }
    SF_CUDA_CHECK(cudaMemsetAsync(b, 0, op->n_free * sizeof(double), st));
    sf::launch_general_rhs(op->SB, op->SQ, op->A.data(), op->B.data(), op->cells, op->geom, fq, b,
                           st);
  });
}

int sf_diagonal(sf_op* op, int dtype, void* d, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(d, SF_ERR_ARG, "null d");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t es = dsize(dtype);
    if (numbered(op)) {  // in lexicographic order, then into the caller's numbering
      void* dl = lex_vec(op, 0);
      {
        LexScope lex(op);
        check_status(sf_diagonal(op, dtype, dl, stream), op);
      }
      sf::permute_gather(dtype, dl, op->d_numbering_inv, d, op->n_free, st);
      return;
    }
    if (op->slab || op->D == 2) {
      SF_REQUIRE(dtype == SF_F64, SF_ERR_UNSUPPORTED,
                 "the diagonal of a slab or 2D operator is FP64");
      compute_diag(op, static_cast<double*>(d), st);
      return;
    }
    SF_CUDA_CHECK(cudaMemsetAsync(d, 0, op->n_free * es, st));
    sf::launch_general_diag(dtype, op->SB, op->SQ, op->A.data(), op->B.data(), op->cells, op->geom,
                            d, st);
  });
}

int sf_cg(sf_op* op, int mode, const double* b, double* x, double reltol, int maxiter, int* iters,
          double* relres, void* stream) {
  if (!op) return SF_ERR_ARG;
  int status = guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(!op->slab, SF_ERR_UNSUPPORTED,
               "a slab operator solves through the distributed CG steps (sf_cgd_*)");
    SF_REQUIRE(b && x, SF_ERR_ARG, "null b or x");
    SF_REQUIRE(reltol > 0 && maxiter >= 0, SF_ERR_ARG, "bad reltol / maxiter");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SF_REQUIRE(mode == SF_CG_F64 || mode == SF_CG_F64_PLAIN || mode == SF_CG_MIXED, SF_ERR_ARG,
               "unknown CG mode");
    double rel = 0.0;
    int it = 0, outer = 1;
    // a numbered operator solves in lexicographic order: b and x are permuted once
    const bool perm = numbered(op);
    const double* bs = b;
    double* xs = x;
    if (perm) {
      double* bl = static_cast<double*>(lex_vec(op, 0));
      double* xl = static_cast<double*>(lex_vec(op, 1));
      sf::permute_gather(SF_F64, b, op->d_numbering, bl, op->n_free, st);
      sf::permute_gather(SF_F64, x, op->d_numbering, xl, op->n_free, st);
      bs = bl;
      xs = xl;
    }
    {
      LexScope lex(op);  // no effect without a numbering
      if (mode == SF_CG_MIXED)
        it = cg_mixed(op, bs, xs, reltol, maxiter, &rel, &outer, st);
      else
        it = cg_f64(op, mode == SF_CG_F64, bs, xs, reltol, maxiter, &rel, st);
    }
    if (perm) sf::permute_gather(SF_F64, xs, op->d_numbering_inv, x, op->n_free, st);
    op->last_inner = it;
    op->last_outer = outer;
    op->last_relres = rel;
    if (iters) *iters = it;
    if (relres) *relres = rel;
    if (!(rel <= reltol)) throw Error(SF_ERR_NOT_CONVERGED, "CG reached its iteration cap");
  });
  return status;
}

// ---------------------------------------------------------------------------
// Distributed Jacobi CG in steps (slab operators; also a single full operator).
// The caller owns the slab-layout vectors and the scalar block s, exchanges
// the halo planes of x (before sf_cgd_start) and of p (before each
// sf_cgd_apply), and sums the listed entries of s over the ranks in place
// between the steps. Every kernel here works on the owned points only, except
// the apply, which reads the halo planes.
// ---------------------------------------------------------------------------
int sf_cgd_start(sf_op* op, const double* b, const double* x, double* r, double* p, double* q,
                 double* s, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(b && x && r && p && q && s, SF_ERR_ARG, "null vector or scalar block");
    require_own_numbering(op, "sf_cgd_start");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long off = owned_offset(op), n = owned_count(op);
    const double* dinv = ensure_dinv(op, st);
    double* partials = static_cast<double*>(workspace(op, cg_partials(op) * sizeof(double)));
    sf::cg_reset(s, st);
    apply_impl(op, SF_F64, x, q, st);
    sf::cg_start<double>(b + off, q + off, dinv + off, r + off, p + off, n, partials, s, st);
  });
}

int sf_cgd_init(sf_op* op, double* s, double reltol, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    SF_REQUIRE(s && reltol > 0, SF_ERR_ARG, "null scalar block or bad reltol");
    sf::cg_init(s, reltol * reltol, static_cast<cudaStream_t>(stream));
  });
}

int sf_cgd_apply(sf_op* op, const double* p, double* q, double* s, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(p && q && s, SF_ERR_ARG, "null p, q or scalar block");
    require_own_numbering(op, "sf_cgd_apply");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* partials = static_cast<double*>(workspace(op, cg_partials(op) * sizeof(double)));
    if (tiled(op, SF_F64)) {
      sf::CartFuse fuse;
      fuse.dot = partials;
      sf::cartesian_apply(op->cart, SF_F64, p, q, st, fuse);
      sf::dot_finish(partials, sf::cartesian_tiles(op->cart, SF_F64), s + sf::CG_PART_PQ,
                     s + sf::CG_DONE, st);
    } else {
      apply_impl(op, SF_F64, p, q, st);
      sf::vec_dot<double>(p, q, op->n_free, partials, s + sf::CG_PART_PQ, s, s + sf::CG_DONE, st);
    }
  });
}

int sf_cgd_update(sf_op* op, double* r, const double* q, double* s, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(r && q && s, SF_ERR_ARG, "null r, q or scalar block");
    require_own_numbering(op, "sf_cgd_update");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long off = owned_offset(op), n = owned_count(op);
    const double* dinv = ensure_dinv(op, st);
    double* partials = static_cast<double*>(workspace(op, cg_partials(op) * sizeof(double)));
    sf::cg_update<double>(s, r + off, q + off, dinv + off, n, partials, st, true);
  });
}

int sf_cgd_direction(sf_op* op, double* x, double* p, const double* r, double* s, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(x && p && r && s, SF_ERR_ARG, "null x, p, r or scalar block");
    require_own_numbering(op, "sf_cgd_direction");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long off = owned_offset(op), n = owned_count(op);
    const double* dinv = ensure_dinv(op, st);
    sf::cg_check(s, st);
    sf::cg_direction<double>(s, x + off, p + off, r + off, dinv + off, n, nullptr, st);
  });
}

int sf_set_option(sf_op* op, const char* name, double value) {
  if (!op || !name) return SF_ERR_ARG;
  return guarded(op, [&] {
    const std::string n(name);
    if (n == "mixed_inner_reltol") {
      SF_REQUIRE(value > 0 && value < 1, SF_ERR_ARG, "mixed_inner_reltol must be in (0,1)");
      op->mixed_inner_reltol = value;
    } else if (n == "jacobi_table") {
      SF_REQUIRE(value == 0 || value == 1, SF_ERR_ARG, "jacobi_table must be 0 or 1");
      op->jacobi_table = value == 1;
    } else if (n == "numbered_fused") {
      SF_REQUIRE(value == -1 || value == 0 || value == 1, SF_ERR_ARG,
                 "numbered_fused must be -1 (by the numbering's locality), 0 or 1");
      op->numbered_fused = (int)value;
    } else if (n == "host_groups") {
      SF_REQUIRE(value >= 1 && value <= 64 && value == (int)value, SF_ERR_ARG,
                 "host_groups must be an integer in 1..64");
      op->host_groups = (int)value;
    } else if (n == "tile_candidate_f64" || n == "tile_candidate_f32") {
      const int dt = n == "tile_candidate_f64" ? SF_F64 : SF_F32;
      SF_REQUIRE(op->cartesian_ok, SF_ERR_STATE, "the tiled Cartesian kernel is not in use");
      const int nc = sf::cartesian_candidates(op->cart, dt);
      SF_REQUIRE(value >= 0 && value < nc && value == (int)value, SF_ERR_ARG,
                 "tile candidate out of range (0.." + std::to_string(nc - 1) + ")");
      op->cart.choice[dt == SF_F64 ? 0 : 1] = (int)value;
    } else {
      throw Error(SF_ERR_ARG, "unknown option " + n);
    }
  });
}

int sf_autotune(sf_op* op, int dtype, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    const size_t es = dsize(dtype);
    if (!(op->cartesian_ok && sf::cartesian_supported(op->cart, dtype)) || op->n_free == 0) return;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = op->n_free;
    const int nc = sf::cartesian_candidates(op->cart, dtype);
    if (nc > 1) {
      Scratch sc;
      void* x = sc.get(n * es);
      void* y = sc.get(n * es);
      SF_CUDA_CHECK(cudaMemsetAsync(x, 0, n * es, st));
      op->cart.choice[dtype == SF_F64 ? 0 : 1] = fastest(nc, st, [&](int k) {
        sf::cartesian_apply_candidate(op->cart, dtype, k, x, y, st);
      });
    }
  });
}

const char* sf_cg_kernel_name(const sf_op* op) {
  if (!op) return "null handle";
  return "apply with the (p, Ap) sum, update and direction kernels";
}

const char* sf_kernel_name(const sf_op* op, int dtype) {
  if (!op) return "null handle";
  if (dtype != SF_F64 && dtype != SF_F32) return "invalid dtype";
  if (op->cartesian_ok && sf::cartesian_supported(op->cart, dtype))
    return sf::cartesian_candidate_name(op->cart, dtype, op->cart.choice[dtype == SF_F64 ? 0 : 1]);
  return "general element kernel";
}

int sf_get_info(const sf_op* op, const char* key, double* value) {
  if (!op || !key || !value) return SF_ERR_ARG;
  const std::string k(key);
  const bool tiled = op->cartesian_ok && sf::cartesian_supported(op->cart, SF_F64);
  if (k == "n_free") *value = (double)op->n_free;
  else if (k == "n_cells") *value = (double)op->cells.ncells;
  else if (k == "tiled_kernel") *value = tiled ? 1.0 : 0.0;
  else if (k == "kernels_per_apply") *value = tiled ? (double)sf::cartesian_launches(op->cart) : 1.0;
  else if (k == "geometry_kind") *value = (double)op->geom.kind;
  else if (k == "slab") *value = op->slab ? 1.0 : 0.0;
  else if (k == "numbered") *value = op->d_numbering ? 1.0 : 0.0;
  else if (k == "numbered_fused")
    *value = (op->d_numbering && (op->numbered_fused == 1 ||
                                  (op->numbered_fused < 0 && op->numbering_local))) ? 1.0 : 0.0;
  else if (k == "jacobi_table")
    *value = (op->jacobi_table && !op->slab && tiled && op->D == 3) ? 1.0 : 0.0;
  else if (k == "plane_size") *value = (double)op->plane;
  else if (k == "owned_offset") *value = (double)owned_offset(op);
  else if (k == "owned_count") *value = (double)owned_count(op);
  else if (k == "tile_candidates_f64" || k == "tile_candidates_f32") {
    const int dt = k == "tile_candidates_f64" ? SF_F64 : SF_F32;
    *value = (op->cartesian_ok && sf::cartesian_supported(op->cart, dt))
                 ? (double)sf::cartesian_candidates(op->cart, dt) : 0.0;
  }
  else return SF_ERR_ARG;
  return SF_OK;
}

int sf_last_solve_info(const sf_op* op, int* outer, int* inner, double* relres) {
  if (!op) return SF_ERR_ARG;
  if (outer) *outer = op->last_outer;
  if (inner) *inner = op->last_inner;
  if (relres) *relres = op->last_relres;
  return SF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// sf_cg_noalloc: the FP64 CG of sf_cg with its scratch in a static device array.
//
// Who needs it: callers that cannot call cudaMalloc. For example, a host
// whose device memory is owned by its own pool allocator (CUDA.jl's and
// PyTorch's caching allocators keep freed memory for reuse), or a
// time-critical loop that cannot afford the device-wide synchronisation
// cudaMalloc/cudaFree can cause. sf_cg allocates its workspace, the cached
// diagonal and a pinned host scalar on first use. This variant uses none of
// them.
//
// The scratch (vectors r, p, q, dinv and diag of up to SF_NOALLOC_MAX_FREE
// dofs, plus the CG scalars and reduction partial sums, about 10 MB) is one
// file-scope __device__ array. Every GPU that loads this library holds it
// until the process exits. Its device address is looked up with
// cudaGetSymbolAddress by the first call on each device, with that device
// current. All calls share the array, so calls that overlap on the GPU
// race. Everything a call reads from the array is written by that call
// first, and the diagonal is re-zeroed on every call before it is
// accumulated.
// ---------------------------------------------------------------------------
namespace {

constexpr long long kNoAllocMaxFree = SF_NOALLOC_MAX_FREE;
constexpr long long kNoAllocScalarWords = 32;  // CG scalars, padded to 256 bytes
constexpr int kNoAllocChunk = 8;               // iterations queued between reads of the flag
constexpr long long kNoAllocWords =
    5 * kNoAllocMaxFree + kNoAllocScalarWords + 3LL * sf::kRedBlocks;
static_assert((kNoAllocMaxFree * 8) % 256 == 0, "scratch vectors must stay 256-byte aligned");
static_assert(sf::CG_NSLOTS <= kNoAllocScalarWords, "CG scalars exceed their scratch words");

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocWords];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

// Device address of the scratch array on the current device (looked up once per device).
double* noalloc_scratch() {
  int dev = -1;
  SF_CUDA_CHECK(cudaGetDevice(&dev));
  SF_REQUIRE(dev >= 0 && dev < kNoAllocMaxDevices, SF_ERR_UNSUPPORTED,
             "device ordinal beyond the no-alloc address table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    SF_CUDA_CHECK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    SF_REQUIRE(p != nullptr, SF_ERR_CUDA, "cudaGetSymbolAddress returned null");
    g_noalloc_ptr[dev] = static_cast<double*>(p);
  }
  return g_noalloc_ptr[dev];
}

double read_scalar_noalloc(const double* d_s, int slot, cudaStream_t st) {
  double h = 0.0;
  SF_CUDA_CHECK(cudaMemcpyAsync(&h, d_s + slot, sizeof(double), cudaMemcpyDeviceToHost, st));
  SF_CUDA_CHECK(cudaStreamSynchronize(st));
  return h;
}

int cg_f64_noalloc(sf_op* op, bool jacobi, const double* b, double* x, double reltol, int maxiter,
                   double* relres, cudaStream_t st) {
  const long long n = op->n_free;
  double* base = noalloc_scratch();
  double* r = base;
  double* p = base + kNoAllocMaxFree;
  double* q = base + 2 * kNoAllocMaxFree;
  double* dinv = base + 3 * kNoAllocMaxFree;
  double* diag = base + 4 * kNoAllocMaxFree;
  double* s = base + 5 * kNoAllocMaxFree;
  double* partials = s + kNoAllocScalarWords;
  if (jacobi) {
    compute_diag(op, diag, st);
    sf::vec_invert<double>(diag, dinv, n, st);
  }
  const double* Dv = jacobi ? dinv : nullptr;
  sf::cg_reset(s, st);
  apply_impl(op, SF_F64, x, q, st);
  sf::cg_start<double>(b, q, Dv, r, p, n, partials, s, st);
  sf::cg_init(s, reltol * reltol, st);
  const double bb = read_scalar_noalloc(s, sf::CG_BB, st);
  const double nb = std::sqrt(bb) > 0 ? std::sqrt(bb) : 1.0;
  double done = read_scalar_noalloc(s, sf::CG_DONE, st);
  // Iterations are queued kNoAllocChunk at a time and the flag is read once per
  // chunk. Every kernel of an iteration does nothing once the flag is set, so the
  // iterations queued past convergence leave x, the residual and the count as
  // they were.
  for (int queued = 0; queued < maxiter && done == 0.0;) {
    const int chunk = std::min(kNoAllocChunk, maxiter - queued);
    for (int k = 0; k < chunk; ++k) {
      apply_impl(op, SF_F64, p, q, st);
      sf::vec_dot<double>(p, q, n, partials, s + sf::CG_PQ, s, s + sf::CG_DONE, st);
      sf::cg_update<double>(s, r, q, Dv, n, partials, st);
      sf::cg_direction<double>(s, x, p, r, Dv, n, nullptr, st);
    }
    queued += chunk;
    done = read_scalar_noalloc(s, sf::CG_DONE, st);
  }
  SF_REQUIRE(done != 3.0, SF_ERR_NONFINITE, "non-finite residual in CG");
  *relres = std::sqrt(read_scalar_noalloc(s, sf::CG_RR, st)) / nb;
  return (int)read_scalar_noalloc(s, sf::CG_ITERS, st);
}

}  // namespace

extern "C" int sf_cg_noalloc(sf_op* op, int mode, const double* b, double* x, double reltol,
                             int maxiter, int* iters, double* relres, void* stream) {
  if (!op) return SF_ERR_ARG;
  return guarded(op, [&] {
    require_ready(op);
    SF_REQUIRE(b && x, SF_ERR_ARG, "null b or x");
    SF_REQUIRE(reltol > 0 && maxiter >= 0, SF_ERR_ARG, "bad reltol / maxiter");
    require_own_numbering(op, "sf_cg_noalloc");
    SF_REQUIRE(op->n_free <= kNoAllocMaxFree, SF_ERR_ARG,
               "n_free = " + std::to_string(op->n_free) +
                   " exceeds the no-alloc scratch limit SF_NOALLOC_MAX_FREE = " +
                   std::to_string(kNoAllocMaxFree));
    SF_REQUIRE(mode == SF_CG_F64 || mode == SF_CG_F64_PLAIN, SF_ERR_UNSUPPORTED,
               "sf_cg_noalloc supports SF_CG_F64 and SF_CG_F64_PLAIN only");
    SF_REQUIRE(!op->slab, SF_ERR_UNSUPPORTED, "sf_cg_noalloc does not take slab operators");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double rel = 0.0;
    const int it = cg_f64_noalloc(op, mode == SF_CG_F64, b, x, reltol, maxiter, &rel, st);
    op->last_inner = it;
    op->last_outer = 1;
    op->last_relres = rel;
    if (iters) *iters = it;
    if (relres) *relres = rel;
    if (!(rel <= reltol)) throw Error(SF_ERR_NOT_CONVERGED, "CG reached its iteration cap");
  });
}

// ---------------------------------------------------------------------------
// Batched form: many independent Cartesian problems, several right-hand
// sides each, applied by one CUDA-graph launch. Problems are grouped by
// order and 1D operators. Each group runs one persistent kernel over all its
// (problem, right-hand side, tile) work items, and the groups are concurrent
// branches of the graph.
// ---------------------------------------------------------------------------
struct sf_batch {
  std::vector<sf_op*> ops;
  int nrhs = 1;
  struct Group {
    std::vector<int> members;
    bool iso = true;
    int cand[2] = {0, 0};
  };
  std::vector<Group> groups;
  struct PerDtype {
    std::vector<const void*> xs;
    std::vector<void*> ys;
    char* d_desc = nullptr;                // descriptors of all groups, back to back
    std::vector<size_t> desc_off;          // byte offset per group
    std::vector<long long> total;          // work items per group
    unsigned long long* d_counter = nullptr;  // one counter per group
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;
  } st[2];
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> ev;
  cudaStream_t cap = nullptr;
  std::string err;
};

namespace {

int bfail(sf_batch* b, int status, const std::string& msg) {
  if (b) b->err = msg;
  return status;
}

template <typename F>
int bguarded(sf_batch* b, F&& f) {
  try {
    f();
    if (b) b->err.clear();
    return SF_OK;
  } catch (const Error& e) {
    return bfail(b, e.status, e.what());
  } catch (const std::exception& e) {
    return bfail(b, SF_ERR_ARG, e.what());
  }
}

void batch_free_dtype(sf_batch::PerDtype& s) {
  if (s.exec) cudaGraphExecDestroy(s.exec);
  if (s.graph) cudaGraphDestroy(s.graph);
  dfree(s.d_desc);
  dfree(s.d_counter);
  s.exec = nullptr;
  s.graph = nullptr;
  s.d_desc = nullptr;
  s.d_counter = nullptr;
  s.dirty = true;
}

// (Re)write the descriptors of every group for the current vectors and candidates.
void batch_descriptors(sf_batch* b, int slot, int dtype) {
  auto& s = b->st[slot];
  const size_t db = sf::cartesian_batch_desc_bytes(dtype);
  std::vector<char> host;
  s.desc_off.assign(b->groups.size(), 0);
  s.total.assign(b->groups.size(), 0);
  for (size_t g = 0; g < b->groups.size(); ++g) {
    const auto& grp = b->groups[g];
    s.desc_off[g] = host.size();
    long long first = 0;
    for (int i : grp.members) {
      sf_op* op = b->ops[i];
      const size_t at = host.size();
      host.resize(at + db);
      first += sf::cartesian_batch_desc(op->cart, dtype, grp.cand[slot], s.xs[i], s.ys[i],
                                        op->n_free, op->n_free, b->nrhs, first, host.data() + at);
    }
    s.total[g] = first;
  }
  if (!s.d_desc) {
    s.d_desc = dalloc<char>(host.size());
    s.d_counter = dalloc<unsigned long long>(b->groups.size());
  }
  SF_CUDA_CHECK(cudaMemcpy(s.d_desc, host.data(), host.size(), cudaMemcpyHostToDevice));
}

void batch_launch_group(sf_batch* b, int slot, int dtype, size_t g, cudaStream_t st) {
  auto& s = b->st[slot];
  const auto& grp = b->groups[g];
  sf::cartesian_batch_launch(b->ops[grp.members[0]]->cart, dtype, grp.cand[slot],
                             s.d_desc + s.desc_off[g], (int)grp.members.size(), s.total[g],
                             s.d_counter + g, grp.iso, st);
}

// Capture: zero the counters, then one persistent kernel per group on its own branch.
void batch_capture(sf_batch* b, int slot, int dtype) {
  auto& s = b->st[slot];
  if (s.exec) cudaGraphExecDestroy(s.exec);
  if (s.graph) cudaGraphDestroy(s.graph);
  s.exec = nullptr;
  s.graph = nullptr;
  const size_t ng = b->groups.size();
  while (b->side.size() < ng) {
    cudaStream_t t;
    SF_CUDA_CHECK(cudaStreamCreateWithFlags(&t, cudaStreamNonBlocking));
    b->side.push_back(t);
  }
  while (b->ev.size() < ng + 1) {
    cudaEvent_t e;
    SF_CUDA_CHECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    b->ev.push_back(e);
  }
  if (!b->cap) SF_CUDA_CHECK(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
  SF_CUDA_CHECK(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
  try {
    SF_CUDA_CHECK(cudaMemsetAsync(s.d_counter, 0, ng * sizeof(unsigned long long), b->cap));
    SF_CUDA_CHECK(cudaEventRecord(b->ev[ng], b->cap));
    for (size_t g = 0; g < ng; ++g) {
      SF_CUDA_CHECK(cudaStreamWaitEvent(b->side[g], b->ev[ng], 0));
      batch_launch_group(b, slot, dtype, g, b->side[g]);
      SF_CUDA_CHECK(cudaEventRecord(b->ev[g], b->side[g]));
      SF_CUDA_CHECK(cudaStreamWaitEvent(b->cap, b->ev[g], 0));
    }
  } catch (...) {
    cudaGraph_t junk = nullptr;
    cudaStreamEndCapture(b->cap, &junk);
    if (junk) cudaGraphDestroy(junk);
    throw;
  }
  SF_CUDA_CHECK(cudaStreamEndCapture(b->cap, &s.graph));
  SF_CUDA_CHECK(cudaGraphInstantiate(&s.exec, s.graph, 0));
  s.dirty = false;
}

int batch_slot(int dtype) {
  if (dtype == SF_F64) return 0;
  if (dtype == SF_F32) return 1;
  throw Error(SF_ERR_ARG, "dtype must be SF_F64 or SF_F32");
}

void batch_bind(sf_batch* b, int slot, const void* const* x, void* const* y) {
  auto& s = b->st[slot];
  const size_t n = b->ops.size();
  bool changed = s.xs.size() != n;
  if (!changed)
    for (size_t i = 0; i < n; ++i)
      if (s.xs[i] != x[i] || s.ys[i] != y[i]) changed = true;
  if (changed) {
    for (size_t i = 0; i < n; ++i)
      SF_REQUIRE(x[i] && y[i] && x[i] != y[i], SF_ERR_ARG, "null or aliased x/y in the batch");
    s.xs.assign(x, x + n);
    s.ys.assign(y, y + n);
    s.dirty = true;
  }
}

}  // namespace

extern "C" int sf_batch_create(sf_batch** out, int nops, sf_op* const* ops, int nrhs) {
  if (!out || nops <= 0 || !ops || nrhs <= 0) return SF_ERR_ARG;
  *out = nullptr;
  sf_batch* b = new (std::nothrow) sf_batch();
  if (!b) return SF_ERR_ARG;
  int st = bguarded(b, [&] {
    b->nrhs = nrhs;
    b->ops.assign(ops, ops + nops);
    for (int i = 0; i < nops; ++i) {
      sf_op* op = b->ops[i];
      SF_REQUIRE(op, SF_ERR_ARG, "null handle in the batch");
      require_ready(op);
      SF_REQUIRE(op->D == 3, SF_ERR_UNSUPPORTED, "the batched form takes 3D operators");
      require_own_numbering(op, "the batched form");
      SF_REQUIRE(op->cartesian_ok && sf::cartesian_supported(op->cart, SF_F64), SF_ERR_UNSUPPORTED,
                 "batch member " + std::to_string(i) +
                     " is not a constant-coefficient Cartesian problem (tiled kernel)");
      // group by identical 1D operators (same order and quadrature)
      size_t g = 0;
      for (; g < b->groups.size(); ++g) {
        const sf_op* r = b->ops[b->groups[g].members[0]];
        if (r->SB == op->SB &&
            std::memcmp(r->cart.M, op->cart.M, sizeof(op->cart.M)) == 0 &&
            std::memcmp(r->cart.K, op->cart.K, sizeof(op->cart.K)) == 0)
          break;
      }
      if (g == b->groups.size()) b->groups.emplace_back();
      b->groups[g].members.push_back(i);
      const double* c = op->cart.c;
      if (!(c[0] == c[1] && c[1] == c[2])) b->groups[g].iso = false;
    }
  });
  if (st != SF_OK) {
    delete b;
    return st;
  }
  *out = b;
  return SF_OK;
}

extern "C" int sf_batch_destroy(sf_batch* b) {
  if (!b) return SF_OK;
  for (auto& s : b->st) batch_free_dtype(s);
  for (auto t : b->side) cudaStreamDestroy(t);
  for (auto e : b->ev) cudaEventDestroy(e);
  if (b->cap) cudaStreamDestroy(b->cap);
  delete b;
  return SF_OK;
}

extern "C" const char* sf_batch_last_error(const sf_batch* b) {
  return b ? b->err.c_str() : "null batch";
}

extern "C" int sf_batch_groups(const sf_batch* b, int* ngroups) {
  if (!b || !ngroups) return SF_ERR_ARG;
  *ngroups = (int)b->groups.size();
  return SF_OK;
}

extern "C" int sf_batch_apply(sf_batch* b, int dtype, const void* const* x, void* const* y,
                              void* stream) {
  if (!b || !x || !y) return SF_ERR_ARG;
  return bguarded(b, [&] {
    const int slot = batch_slot(dtype);
    auto& s = b->st[slot];
    batch_bind(b, slot, x, y);
    if (s.dirty) {
      batch_descriptors(b, slot, dtype);
      batch_capture(b, slot, dtype);
    }
    SF_CUDA_CHECK(cudaGraphLaunch(s.exec, static_cast<cudaStream_t>(stream)));
  });
}

extern "C" int sf_batch_autotune(sf_batch* b, int dtype, const void* const* x, void* const* y,
                                 void* stream) {
  if (!b || !x || !y) return SF_ERR_ARG;
  return bguarded(b, [&] {
    const int slot = batch_slot(dtype);
    auto& s = b->st[slot];
    batch_bind(b, slot, x, y);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    SF_CUDA_CHECK(cudaEventCreate(&e0));
    SF_CUDA_CHECK(cudaEventCreate(&e1));
    try {
      for (size_t g = 0; g < b->groups.size(); ++g) {
        auto& grp = b->groups[g];
        const int nc = sf::cartesian_candidates(b->ops[grp.members[0]]->cart, dtype);
        int best = 0;
        float best_ms = 0.f;
        for (int k = 0; k < nc; ++k) {
          grp.cand[slot] = k;
          batch_descriptors(b, slot, dtype);
          float ms = 0.f;
          for (int rep = 0; rep < 3; ++rep) {  // first run warms up
            SF_CUDA_CHECK(cudaMemsetAsync(s.d_counter + g, 0, sizeof(unsigned long long), st));
            SF_CUDA_CHECK(cudaEventRecord(e0, st));
            batch_launch_group(b, slot, dtype, g, st);
            SF_CUDA_CHECK(cudaEventRecord(e1, st));
            SF_CUDA_CHECK(cudaEventSynchronize(e1));
            float t = 0.f;
            SF_CUDA_CHECK(cudaEventElapsedTime(&t, e0, e1));
            if (rep > 0) ms += t;
          }
          if (k == 0 || ms < best_ms) {
            best = k;
            best_ms = ms;
          }
        }
        grp.cand[slot] = best;
      }
    } catch (...) {
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    s.dirty = true;  // descriptors and graph follow the chosen candidates
  });
}

extern "C" const char* sf_batch_group_kernel(const sf_batch* b, int dtype, int group) {
  if (!b || group < 0 || group >= (int)b->groups.size()) return "invalid group";
  if (dtype != SF_F64 && dtype != SF_F32) return "invalid dtype";
  const auto& grp = b->groups[group];
  return sf::cartesian_candidate_name(b->ops[grp.members[0]]->cart, dtype,
                                      grp.cand[dtype == SF_F64 ? 0 : 1]);
}

// ---------------------------------------------------------------------------
// Operator access for the other translation units (the multigrid solver).
// ---------------------------------------------------------------------------
namespace sf {

OpShape op_shape(const sf_op* op) {
  OpShape s;
  s.structured = op && op->cells.mesh == MESH_STRUCTURED && op->D == 3 && !op->slab &&
                 !op->d_numbering && op->geom.kind != GEOM_NONE &&
                 (op->cq_cells == 0 || op->cq_cells == op->cells.ncells);
  if (!op) return s;
  s.nx = op->cells.nx;
  s.ny = op->cells.ny;
  s.nz = op->cells.nz;
  s.p = op->p;
  s.n_free = op->n_free;
  return s;
}

void op_apply(sf_op* op, int dtype, const void* x, void* y, cudaStream_t st) {
  apply_impl(op, dtype, x, y, st);
}

void op_diag(sf_op* op, double* d, cudaStream_t st) { compute_diag(op, d, st); }

void op_apply_dot(sf_op* op, const double* x, double* y, double* partials, double* out, double* s,
                  const double* skip, cudaStream_t st) {
  if (tiled(op, SF_F64) && !op->d_numbering) {  // the apply's store phase forms the sums
    sf::CartFuse fuse;
    fuse.dot = partials;
    sf::cartesian_apply(op->cart, SF_F64, x, y, st, fuse);
    sf::dot_finish(partials, sf::cartesian_tiles(op->cart, SF_F64), out, skip, st);
  } else {
    apply_impl(op, SF_F64, x, y, st);
    sf::vec_dot<double>(x, y, op->n_free, partials, out, s, skip, st);
  }
}

long long op_dot_partials(const sf_op* op) { return cg_partials(op); }

bool op_cheb_apply(sf_op* op, const float* z, const float* r, const float* dinv, float* d,
                   float* z_out, double c1, double c2, int mode, cudaStream_t st) {
  if (!tiled(op, SF_F32) || op->d_numbering || op->slab || op->n_free == 0) return false;
  sf::CartFuse fuse;
  fuse.cheb.r = r;
  fuse.cheb.dinv = dinv;
  fuse.cheb.d = d;
  fuse.cheb.z_out = z_out;
  fuse.cheb.c1 = c1;
  fuse.cheb.c2 = c2;
  fuse.cheb.mode = mode;
  sf::cartesian_apply(op->cart, SF_F32, z, nullptr, st, fuse);
  return true;
}


}  // namespace sf
