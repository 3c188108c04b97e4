/*
 * sfb200.h -- C ABI of the B200 matrix-free sum-factorized Laplacian apply.
 *
 * This library replaces the CPU sum-factorization path of
 * JordiManyer/NCIHackaton2023.jl at whole-operator granularity. The
 * reference's per-cell Gridap Map protocol cannot cross into CUDA
 * efficiently cell by cell, so the boundary sits at LinearAlgebra.mul!.
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and
 * returns an int status (SF_OK == 0). No C++ exception crosses the ABI.
 * When a call fails, sf_last_error(op) returns a message. A handle is not
 * thread-safe; all device work is enqueued on the caller's stream.
 *
 * Array conventions follow the Julia reference: matrices are column-major,
 * and indices in dof tables are 1-based. Free dofs are numbered 1..n_free;
 * Dirichlet dofs carry negative ids and are read as zero and never written
 * (src/GPUKernels.jl:23-27,86-88; test/Demo_StepByStep.jl:64-71).
 */
#ifndef SFB200_H
#define SFB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sf_op sf_op;

/* status codes */
#define SF_OK 0
#define SF_ERR_ARG 1          /* invalid argument (sizes, null pointers, unsupported order) */
#define SF_ERR_CUDA 2         /* a CUDA runtime call failed */
#define SF_ERR_STATE 3        /* the handle is missing a required set-up step */
#define SF_ERR_UNSUPPORTED 4  /* valid request that this library does not implement */
#define SF_ERR_NOT_CONVERGED 5/* an iterative solve reached its iteration cap */
#define SF_ERR_NONFINITE 6    /* NaN or Inf met in a solve */

/* arithmetic types of x / y */
#define SF_F64 0
#define SF_F32 1

/* CG modes for sf_cg */
#define SF_CG_F64 0           /* FP64 Jacobi-preconditioned CG */
#define SF_CG_MIXED 1         /* FP32 apply + FP32 Jacobi CG recurrence, FP64 reliable updates */
#define SF_CG_F64_PLAIN 2     /* FP64 CG without a preconditioner (IterativeSolvers default) */

/* Library version (major*10000 + minor*100 + patch). */
int sf_version(void);

/* Text for a status code. */
const char* sf_status_string(int status);

/*
 * Create an operator from the 1D data of a SumFactorizationMap.
 * Replaces SumFactorizationMap(D, fe_orders, quad_orders)
 * (src/SumFactorizationMaps.jl:47-65) plus to_gpu(m) (:25-32).
 *   D       : 3, or 2 (quadrilaterals: structured Cartesian meshes only; the
 *             table gather, evaluate_cells, kappa, rhs, slab and batched
 *             forms return SF_ERR_UNSUPPORTED for D = 2). Other D:
 *             SF_ERR_UNSUPPORTED
 *   SB, SQ  : 1D basis size p+1 (2..10) and quadrature size (1..10)
 *   A0, B0  : SQ x SB column-major, A0[i + SQ*j] = phi_j(xi_i), B0 = phi_j'(xi_i)
 *             (evalMats / B0 at src/SumFactorizationMaps.jl:53-54)
 *   dof_map : SB^D x D column-major int32, 1-based: row k is the tensor index
 *             (j1..jD) of local dof k (m.dof_map, src/SumFactorizationMaps.jl:40-45)
 */
int sf_create(sf_op** out, int D, int SB, int SQ, const double* A0, const double* B0,
              const int32_t* dof_map);

/* Free the handle and its device buffers. NULL is accepted. */
int sf_destroy(sf_op* op);

/* Last error message of this handle ("" if none). */
const char* sf_last_error(const sf_op* op);

/* get_dimensional_parameters(m) (src/SumFactorizationMaps.jl:15-17). */
int sf_get_dimensional_parameters(const sf_op* op, int* D, int* SB, int* SQ);

/*
 * Cell-to-dof table as a Gridap Table (Utils.jl:12-15 to_gpu(::Table)).
 *   ptrs : ncells+1 int32, 1-based offsets into data
 *   data : local ids per cell in the local order of dof_map;
 *          1..n_free free, negative Dirichlet
 * This is get_cell_dof_ids(test) (src/LazyMatrices.jl:46).
 */
int sf_set_cells(sf_op* op, int64_t ncells, const int32_t* ptrs, const int32_t* data,
                 int64_t n_free);

/*
 * Declare a Cartesian mesh: nx*ny*nz cells numbered with x fastest,
 * Dirichlet on the whole boundary, and free dofs numbered lexicographically
 * (x fastest) over the (nx*p-1) x (ny*p-1) x (nz*p-1) interior grid. For an
 * operator created with D = 2, pass nz = 0: nx*ny cells, (nx*p-1) x (ny*p-1) grid.
 * node_order[j] (0-based) is the position 0..p of 1D basis function j along
 * the segment; Gridap's order is {0, p, 1, 2, ..., p-1} (_get_terms,
 * src/SumFactorizationMaps.jl:34-38). This selects the tiled Cartesian kernels.
 */
int sf_set_structured(sf_op* op, int nx, int ny, int nz, const int32_t* node_order);

/*
 * sf_set_structured with the caller's own numbering of the free dofs:
 * free_id[i] (0-based) is the caller's id of lexicographic free point i
 * (x fastest over the (nx p - 1)(ny p - 1)(nz p - 1) interior grid points), a
 * permutation of 0 .. n_free-1. This is the Cartesian mesh of the reference's
 * drivers with Gridap's own dof numbering (get_cell_dof_ids,
 * src/LazyMatrices.jl:46), which is not lexicographic. The tiled kernels still
 * run: sf_apply, sf_apply_multi and sf_mul_host read x and write y through the
 * numbering inside the kernel when it keeps neighbours near (option
 * "numbered_fused"), else permute x into lexicographic order and the result
 * back (two extra vector sweeps per apply); sf_cg permutes
 * b and x once per solve and iterates in lexicographic order; sf_diagonal and
 * sf_rhs compute lexicographically and permute the result. sf_kappa_vjp, the
 * sf_cgd_* steps, sf_cg_noalloc and the batched form reject such a handle.
 * 3D only. sf_set_cells or sf_set_structured drops the numbering.
 */
int sf_set_structured_numbering(sf_op* op, int nx, int ny, int nz, const int32_t* node_order,
                                const int32_t* free_id);

/*
 * The z-slab of cells [z0, z1) of an nx x ny x nz structured mesh (the share of
 * one rank when the mesh is split along z; the reference's Gridap model is one
 * process, so this has no single counterpart there). Vectors of a slab
 * operator hold the free points of the grid z-levels z0 p .. (z1 + 1) p, level
 * by level (plane_size = (nx p - 1)(ny p - 1) points each, x fastest):
 *   plane 0              halo: level z0 p, owned by the rank below (or the
 *                        Dirichlet boundary, then zero);
 *   planes 1 .. (z1-z0)p owned: levels z0 p + 1 .. z1 p, except that level nz p
 *                        (the top boundary, z1 = nz) is Dirichlet and stays zero;
 *   the last p planes    halo: levels z1 p + 1 .. (z1 + 1) p, owned by the rank
 *                        above (zero past the top of the mesh).
 * n_free is the whole slab vector. sf_apply reads all planes and writes the
 * owned points only; sf_diagonal (FP64) writes diag(A) at the owned points.
 * The slab must use the tiled Cartesian kernel (axis-aligned affine cells,
 * constant coefficient). sf_get_info "owned_offset" / "owned_count" give the
 * owned range.
 */
int sf_set_structured_slab(sf_op* op, int nx, int ny, int nz, int z0, int z1,
                           const int32_t* node_order);

/*
 * Geometric factors at the quadrature points, exactly the triple
 * (cell_wq, cell_jq, cell_djq) of LazyMatrix (src/LazyMatrices.jl:34-43):
 *   wq  : SQ^D weights per cell (linear qp index, i1 fastest)
 *   jq  : D x D per qp, column-major (jq[l + D*r] = jq[l,r]) = inv(grad cell map)
 *   djq : |det| per qp
 * fill = 1: the arrays hold ONE cell, shared by all cells (Gridap's Fill for
 * Cartesian meshes); fill = 0: ncells consecutive blocks.
 * The metric G = wq*djq*jq^T*jq (src/SumFactorizationKernels.jl:174-216) is
 * formed once here and kept on the device (6 symmetric components per qp),
 * or as a single constant when it is the same, up to the weights, everywhere.
 */
int sf_set_cell_quantities(sf_op* op, int fill, const double* wq, const double* jq,
                           const double* djq);

/* Diffusion coefficient kappa at every quadrature point (ncells x SQ^D) or
 * NULL for kappa = 1. The operator becomes -div(kappa grad u). */
int sf_set_coefficient(sf_op* op, const double* kappa);

/* Same, from a DEVICE array (ncells x SQ^D FP64), copied on `stream`. */
int sf_set_coefficient_device(sf_op* op, const double* kappa, void* stream);

/*
 * Vector-Jacobian product of y = A(kappa) x with respect to kappa (device
 * pointers): kappa_bar[c][q] = (grad ybar)_q^T G_q (grad x)_q, where G = wq*djq*jq^T*jq
 * is the reference's per-point metric (src/SumFactorizationKernels.jl:174-216)
 * without kappa. The gradients are recomputed by sum factorization and not
 * stored. kappa_bar is ncells x SQ^D FP64; x, ybar are n_free of dtype.
 * The product with respect to x is sf_apply(ybar), because A is symmetric.
 */
int sf_kappa_vjp(sf_op* op, int dtype, const void* x, const void* ybar, double* kappa_bar,
                 void* stream);

/*
 * y = A x over the free dofs, device pointers, enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default). Replaces
 * LinearAlgebra.mul!(y, A::LazyMatrix, x) (src/LazyMatrices.jl:52-61).
 * dtype SF_F64 or SF_F32 (FP32: data, metric and accumulation in FP32).
 */
int sf_apply(sf_op* op, int dtype, const void* x, void* y, void* stream);

/* nrhs right-hand sides: columns of length n_free at strides ldx / ldy (elements). */
int sf_apply_multi(sf_op* op, int dtype, int nrhs, const void* x, int64_t ldx, void* y,
                   int64_t ldy, void* stream);

/* mul!(y, A, x) on HOST FP64 buffers (synchronous): copies x in, applies,
 * copies y out. This is the drop-in for the reference's CPU mul!. */
int sf_mul_host(sf_op* op, const double* x, double* y);

/*
 * The Map protocol itself: Arrays.evaluate!(cache, m, x, wq, jq, djq)
 * (src/SumFactorizationMaps.jl:78-89) for a batch of cells, device pointers.
 * x_cells / y_cells: ncells x SB^D, cell-major, local order of dof_map.
 * Uses the cell quantities given to sf_set_cell_quantities (ncells must match
 * unless they were given with fill = 1).
 */
int sf_evaluate_cells(sf_op* op, int dtype, int64_t ncells, const void* x_cells,
                      void* y_cells, void* stream);

/*
 * Right-hand side of the linear form v -> integral of f v over the mesh
 * (the l(v) of profiling/drivers.jl:20, assembled by Gridap there), matrix-free:
 * b = sum over cells of P_e^T (A0^T (x) A0^T (x) A0^T) (wq |djq| f), the scalar
 * interpolation of src/SumFactorizationKernels.jl:15-38 transposed. fq: f at
 * the quadrature points, [cell][SQ^D] FP64 device array, points in the order of
 * the cell quantities (i1 fastest). b: n_free FP64 device array (overwritten;
 * Dirichlet dofs get nothing, i.e. homogeneous Dirichlet data).
 */
int sf_rhs(sf_op* op, const double* fq, double* b, void* stream);

/* diag(A) over the free dofs (device pointer of dtype), for Jacobi. */
int sf_diagonal(sf_op* op, int dtype, void* d, void* stream);

/*
 * Conjugate gradients on A x = b, device FP64 pointers b and x (x is the
 * initial guess on entry). Replaces IterativeSolvers.cg!(x, A, b) as called
 * at profiling/drivers.jl:85-95. Stops when ||r||_2 <= reltol * ||b||_2
 * (FP64 true residual for SF_CG_MIXED). Reports iterations (FP32 iterations
 * for SF_CG_MIXED) and the final relative residual.
 * An FP64 iteration is the apply (which also forms the (p, Ap) sum on the
 * tiled kernel) and two vector kernels.
 */
int sf_cg(sf_op* op, int mode, const double* b, double* x, double reltol, int maxiter,
          int* iters, double* relres, void* stream);

/*
 * Jacobi FP64 CG in steps, for an operator split over ranks (slab operators;
 * a full operator works too, as one rank). The distributed form of
 * IterativeSolvers.cg! (profiling/drivers.jl:85-95). The caller owns the
 * vectors (all n_free long, slab layout) and a device block s of
 * SF_CGD_SCALARS doubles. It keeps the halo planes of x (before sf_cgd_start)
 * and of p (before each sf_cgd_apply) current, and after the steps marked
 * "sum" adds the listed entries of s over all ranks in place (e.g. an NCCL
 * all-reduce). One solve:
 *   sf_cgd_start(b, x, r, p, q, s)       r = b - A x, p = D^-1 r   sum s[2..4]
 *   sf_cgd_init(s, reltol)
 *   repeat:  exchange p halos
 *            sf_cgd_apply(p, q, s)       q = A p                   sum s[10]
 *            sf_cgd_update(r, q, s)      r -= alpha q              sum s[11..12]
 *            sf_cgd_direction(x, p, r, s) x += alpha p, p = D^-1 r + beta p
 * until s[SF_CGD_DONE] != 0 (read it every few iterations: steps after the
 * converged one change nothing, so every rank can run the same steps).
 * s[SF_CGD_DONE]: 0 running, 2 converged (relres <= reltol), 3 non-finite
 * residual. s[SF_CGD_ITERS] iterations; s[SF_CGD_RR] and s[SF_CGD_BB] the
 * summed squared norms of r and b.
 */
#define SF_CGD_SCALARS 16
#define SF_CGD_RR 3
#define SF_CGD_BB 4
#define SF_CGD_DONE 5
#define SF_CGD_ITERS 6
int sf_cgd_start(sf_op* op, const double* b, const double* x, double* r, double* p, double* q,
                 double* s, void* stream);
int sf_cgd_init(sf_op* op, double* s, double reltol, void* stream);
int sf_cgd_apply(sf_op* op, const double* p, double* q, double* s, void* stream);
int sf_cgd_update(sf_op* op, double* r, const double* q, double* s, void* stream);
int sf_cgd_direction(sf_op* op, double* x, double* p, const double* r, double* s, void* stream);

/*
 * Named numeric options of a handle:
 *   "mixed_inner_reltol" : SF_CG_MIXED refines (FP64 true residual replaces the FP32
 *                          recurrence residual) each time the FP32 residual has
 *                          dropped by this factor (default 0.1)
 *   "tile_candidate_f64"  : force tile-shape candidate k of the tiled Cartesian kernel
 *   "tile_candidate_f32"    (0-based; see sf_get_info "tile_candidates_f64/f32")
 *   "numbered_fused"      : after sf_set_structured_numbering, how an apply on the tiled
 *                           kernel handles the numbering: 1 the kernel reads x and writes y
 *                           through it; 0 x is permuted into lexicographic order and y back;
 *                           -1 (default) 1 when most x-neighbours' ids lie within 64 of each
 *                           other (a cell-by-cell numbering), else 0
 *   "host_groups"         : sf_mul_host with pinned buffers on the tiled kernel splits the
 *                           z-levels into this many groups of tile rows, whose copies in,
 *                           applies and copies out overlap on three streams (default 8)
 *   "jacobi_table"        : 1 (default): on a whole 3D Cartesian mesh the FP64 Jacobi CG's
 *                           vector kernels read D^-1 from a table per position in a cell
 *                           (it repeats cell to cell) instead of a vector; 0: from the vector
 */
int sf_set_option(sf_op* op, const char* name, double value);

/* Outer (refinement) steps, inner iterations and relative residual of the last sf_cg. */
int sf_last_solve_info(const sf_op* op, int* outer, int* inner, double* relres);

/*
 * Read-only facts about a handle, by name:
 *   "n_free", "n_cells"      : sizes
 *   "tiled_kernel"           : 1 if sf_apply(SF_F64) uses the tiled Cartesian kernel
 *   "kernels_per_apply"      : kernel launches one sf_apply(SF_F64) makes
 *   "geometry_kind"          : 1 separable constant metric, 2 per-point table
 *   "tile_candidates_f64/f32": number of tile shapes of the tiled kernel (0 if not in use)
 *   "slab"                   : 1 for a slab operator (sf_set_structured_slab)
 *   "plane_size"             : free points per z-level (structured meshes)
 *   "owned_offset", "owned_count": the points sf_apply writes (the whole vector
 *                              unless the operator is a slab)
 *   "jacobi_table"           : 1 if sf_cg's FP64 Jacobi mode reads D^-1 from the table
 *   "numbered"               : 1 after sf_set_structured_numbering
 *   "numbered_fused"         : 1 if applies read and write through the numbering in the kernel
 */
int sf_get_info(const sf_op* op, const char* key, double* value);

/*
 * Time every tile-shape candidate of the tiled Cartesian kernel for this
 * handle's order, mesh and dtype, and keep the fastest for later sf_apply
 * calls. Temporary vectors are allocated for the timing. Without the
 * tiled kernel (table gather, deformed cells, kappa) it does nothing.
 * Replaces the launch-configuration table that the reference kept by hand
 * (test/benchmark_v3.jl:36-40).
 */
int sf_autotune(sf_op* op, int dtype, void* stream);

/* Description of the kernel sf_apply uses for dtype (static string). */
const char* sf_kernel_name(const sf_op* op, int dtype);

/* Description of the iteration sf_cg's FP64 modes run (static string). */
const char* sf_cg_kernel_name(const sf_op* op);

/*
 * Batched form: many independent Cartesian problems (handles on which the
 * tiled kernel is in use), each with nrhs right-hand sides, applied by ONE
 * CUDA-graph launch. Problems that share an order and 1D operators form a
 * group. Each group is one persistent kernel whose CTAs take (problem,
 * right-hand side, tile) work items from an atomic counter, and the groups
 * run as concurrent branches of the graph. The reference has no batched form;
 * it launched its CUDA.jl kernels one problem at a time (test/GPU_v3.jl:79-84).
 *
 * x[i], y[i]: device pointers to problem i's column-major (n_free_i x nrhs)
 * blocks. The graph is captured on the first apply and re-captured when
 * the pointers change. The handles must outlive the batch.
 */
typedef struct sf_batch sf_batch;
int sf_batch_create(sf_batch** out, int nops, sf_op* const* ops, int nrhs);
int sf_batch_destroy(sf_batch* b);
const char* sf_batch_last_error(const sf_batch* b);
int sf_batch_groups(const sf_batch* b, int* ngroups);
int sf_batch_apply(sf_batch* b, int dtype, const void* const* x, void* const* y, void* stream);
/* Pick the tile shape of every group by timing the candidates on x, y. */
int sf_batch_autotune(sf_batch* b, int dtype, const void* const* x, void* const* y, void* stream);
/* Tile shape used by a group for dtype (static string). */
const char* sf_batch_group_kernel(const sf_batch* b, int dtype, int group);

/*
 * Multigrid-preconditioned flexible CG on structured meshes. New: the
 * reference solves with IterativeSolvers.cg! and no preconditioner
 * (profiling/drivers.jl:85-95); this is the solver for the problems that CG
 * cannot finish in reasonable time (equispaced high order on perturbed cells).
 *
 * sf_mg_create(out, A, nlevels, levels, transfer, basis_change)
 *   A         the operator of the solve (its FP64 apply runs in the outer CG)
 *   levels    nlevels operators, finest first, each a whole 3D structured mesh
 *             (sf_set_structured, geometry set). Level l+1 has the cells of
 *             level l (p-coarsening) or r times fewer per axis (h-coarsening),
 *             and a space contained in level l's. levels[0] has A's mesh and order.
 *   transfer  nlevels-1 row-major tables, transfer[l] of (r p_l + 1) x (p_{l+1} + 1)
 *             doubles: entry [i][m] is coarse 1D basis function m of one coarse
 *             cell at the i-th fine node of that cell (r fine cells of order p_l
 *             along the axis, nodes in ascending position)
 *   basis_change  NULL when levels[0] uses A's basis; else the (p+1) x (p+1)
 *             row-major table [i][m] = levels[0]'s 1D basis function m at A's
 *             i-th node (ascending positions): the hierarchy then works in
 *             levels[0]'s basis and preconditions A through that change of basis.
 * Set-up estimates the largest eigenvalue of D^-1 A on every level. On failure
 * *out still receives a handle holding the message (sf_mg_last_error); destroy it.
 * The handle borrows the operators: they must outlive it.
 *
 * sf_mg_cg: x (device, FP64, initial guess on entry) solves A x = b to
 * ||b - A x|| <= reltol ||b||. mode SF_MG_MIXED runs the V-cycle in FP32 (outer
 * CG, residual and dots in FP64), SF_MG_F64 all in FP64; one handle solves in
 * one mode. Options (sf_mg_set_option): "degree" (Chebyshev smoothing steps, 4),
 * "ratio" (smoothing range lmax/ratio..1.1 lmax, 20), "coarse_steps" (10),
 * "coarse_ratio" (100). sf_mg_get_info: "levels", "lmax<l>", "n<l>", "graph".
 *
 * sf_mg_refresh: after the operators' coefficients changed (sf_set_coefficient
 * on A and on the levels), recomputes every level's diagonal and eigenvalue
 * estimate and captures the iteration again on the next solve; the levels,
 * tables and buffers are kept. Ordered after the work queued on `stream`;
 * returns when the set-up has finished. Until it succeeds, sf_mg_cg returns
 * SF_ERR_STATE.
 */
#define SF_MG_MIXED 0
#define SF_MG_F64 1
typedef struct sf_mg sf_mg;
int sf_mg_create(sf_mg** out, sf_op* A, int nlevels, sf_op* const* levels,
                 const double* const* transfer, const double* basis_change);
int sf_mg_destroy(sf_mg* mg);
const char* sf_mg_last_error(const sf_mg* mg);
int sf_mg_set_option(sf_mg* mg, const char* name, double value);
int sf_mg_get_info(const sf_mg* mg, const char* key, double* value);
int sf_mg_cg(sf_mg* mg, int mode, const double* b, double* x, double reltol, int maxiter,
             int* iters, double* relres, void* stream);
int sf_mg_refresh(sf_mg* mg, void* stream);

/*
 * sf_cg_noalloc: sf_cg without any device or pinned-host allocation. It has no
 * counterpart in the reference.
 *
 * It is for callers that cannot call cudaMalloc: for example, a host whose
 * device memory is owned by its own pool allocator (CUDA.jl's and PyTorch's
 * caching allocators keep freed memory for reuse), or a time-critical loop
 * that cannot afford the device-wide synchronisation that cudaMalloc/cudaFree
 * can cause. Same arguments and stopping rule as sf_cg. Modes SF_CG_F64 and
 * SF_CG_F64_PLAIN only (SF_CG_MIXED returns SF_ERR_UNSUPPORTED).
 *
 * Operators it rejects although sf_cg takes them (SF_ERR_UNSUPPORTED): a
 * Cartesian operator with the caller's dof numbering
 * (sf_set_structured_numbering) and a slab operator (sf_set_structured_slab).
 *
 * The call reads the device's convergence flag once per 8 queued iterations
 * and synchronises the stream to do so; it returns after the solve has
 * finished on the device.
 *
 * Limits and sharing:
 * - Its scratch is one static device array sized for n_free <= SF_NOALLOC_MAX_FREE
 *   (about 10 MB). Every GPU that loads the library holds it until exit.
 *   Larger problems are rejected with SF_ERR_ARG.
 * - The first call on each device looks up the array's device address.
 * - All calls share the array: calls that overlap on the GPU race.
 */
#define SF_NOALLOC_MAX_FREE 262144
int sf_cg_noalloc(sf_op* op, int mode, const double* b, double* x, double reltol, int maxiter,
                  int* iters, double* relres, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SFB200_H */
