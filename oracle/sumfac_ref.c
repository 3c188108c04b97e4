/*
 * sumfac_ref.c -- C restatement of the reference's CPU sum-factorization
 * path (TEST INFRASTRUCTURE ONLY: the parity reference and the timed CPU baseline).
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load the
 * shared object built from this file. The product never does.
 *
 * It follows JordiManyer/NCIHackaton2023.jl loop by loop, with the same
 * redundant D-component layout Z[r, a1, a2, a3] (r fastest):
 *   gather with Dirichlet zeros      src/LazyMatrices.jl:53, test/Demo_StepByStep.jl:64-71
 *   _sumfac_array2tensor!            src/SumFactorizationKernels.jl:135-151
 *   _sumfac_dof2quad! (vector)       src/SumFactorizationKernels.jl:40-65
 *   _sumfac_apply_weights!           src/SumFactorizationKernels.jl:174-216
 *   _sumfac_quad2dof! (vector)       src/SumFactorizationKernels.jl:105-130
 *   _sumfac_tensor2array!            src/SumFactorizationKernels.jl:156-172
 *   assemble_vector! skipping ids<0  src/LazyMatrices.jl:57-58
 * The contraction sums run in the reference's index order. The reference
 * specialises its loops on (D, SB, SQ) with @generated + @turbo. The same
 * is done here: the cell kernel is an always-inline function, called with
 * compile-time sizes for the common (SB, SQ) pairs.
 *
 * Threads: the reference is single-threaded (benchmark.sh:5 uses ncpus=1).
 * nthreads = 1 reproduces that. nthreads > 1 runs the cells of each colour
 * in parallel (OpenMP). Cells of one colour must share no dof, which the
 * caller guarantees. This is the labelled "restatement, N cores" variant.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXS 10

typedef struct {
  const double* A0; /* SQ x SB column-major */
  const double* B0;
  const int32_t* dof_map; /* SB^3 x 3 column-major, 1-based */
  int64_t ncells;
  const int32_t* cell_ids; /* ncells x SB^3, 1-based free ids, <0 Dirichlet */
  int fill;                /* 1: wq/jq/djq hold one cell for all */
  const double* wq;        /* SQ^3 per cell */
  const double* jq;        /* 9 per point, column-major jq[l + 3r] */
  const double* djq;       /* per point */
  const double* kappa;     /* SQ^3 per cell or NULL */
} sfref_problem;

static inline __attribute__((always_inline)) double matel(const double* A0, const double* B0, int SQ,
                                                          int d, int k, int i, int j) {
  /* gradMats[d,k] = (d != k) ? A0 : B0 (src/SumFactorizationMaps.jl:57-58) */
  return (d != k) ? A0[i + SQ * j] : B0[i + SQ * j];
}

static inline __attribute__((always_inline)) void cell_eval(const int SB, const int SQ,
                                                            const sfref_problem* P,
                                                            const int* tpos, int64_t c,
                                                            const double* x, double* y,
                                                            double* Z1, double* Z2, double* Z3,
                                                            double* Z4) {
  const double* A0 = P->A0;
  const double* B0 = P->B0;
  const int nloc = SB * SB * SB;
  const int nq = SQ * SQ * SQ;
  const int32_t* ids = P->cell_ids + (size_t)c * nloc;
  /* array2tensor with the gather: Z1[r, j1, j2, j3] = x_e[k] for all r */
  for (int k = 0; k < nloc; ++k) {
    const int32_t id = ids[k];
    const double v = id > 0 ? x[id - 1] : 0.0;
    const int t = tpos[k];
    for (int r = 0; r < 3; ++r) Z1[r + 3 * t] = v;
  }
  /* dof2quad, d = 1: Z2[k,i1,j2,j3] = sum_j1 M[1,k][i1,j1] Z1[k,j1,j2,j3] */
  for (int j3 = 0; j3 < SB; ++j3)
    for (int j2 = 0; j2 < SB; ++j2)
      for (int i1 = 0; i1 < SQ; ++i1)
        for (int k = 0; k < 3; ++k) {
          double s = 0.0;
          for (int j1 = 0; j1 < SB; ++j1)
            s += matel(A0, B0, SQ, 0, k, i1, j1) * Z1[k + 3 * (j1 + SB * (j2 + SB * j3))];
          Z2[k + 3 * (i1 + SQ * (j2 + SB * j3))] = s;
        }
  /* d = 2: Z3[k,i1,i2,j3] = sum_j2 M[2,k][i2,j2] Z2[k,i1,j2,j3] */
  for (int j3 = 0; j3 < SB; ++j3)
    for (int i2 = 0; i2 < SQ; ++i2)
      for (int i1 = 0; i1 < SQ; ++i1)
        for (int k = 0; k < 3; ++k) {
          double s = 0.0;
          for (int j2 = 0; j2 < SB; ++j2)
            s += matel(A0, B0, SQ, 1, k, i2, j2) * Z2[k + 3 * (i1 + SQ * (j2 + SB * j3))];
          Z3[k + 3 * (i1 + SQ * (i2 + SQ * j3))] = s;
        }
  /* d = 3: Z4[k,i1,i2,i3] = sum_j3 M[3,k][i3,j3] Z3[k,i1,i2,j3] */
  for (int i3 = 0; i3 < SQ; ++i3)
    for (int i2 = 0; i2 < SQ; ++i2)
      for (int i1 = 0; i1 < SQ; ++i1)
        for (int k = 0; k < 3; ++k) {
          double s = 0.0;
          for (int j3 = 0; j3 < SB; ++j3)
            s += matel(A0, B0, SQ, 2, k, i3, j3) * Z3[k + 3 * (i1 + SQ * (i2 + SQ * j3))];
          Z4[k + 3 * (i1 + SQ * (i2 + SQ * i3))] = s;
        }
  /* apply_weights: Z[r] <- wq*djq*sum_k (sum_l jq[l,r] jq[l,k]) Z[k] */
  const size_t cq = P->fill ? 0 : (size_t)c;
  for (int q = 0; q < nq; ++q) {
    const double* J = P->jq + (cq * nq + q) * 9;
    double z[3];
    for (int r = 0; r < 3; ++r) {
      double cr = 0.0;
      for (int k = 0; k < 3; ++k) {
        double jrk = 0.0;
        for (int l = 0; l < 3; ++l) jrk += J[l + 3 * r] * J[l + 3 * k];
        cr += jrk * Z4[k + 3 * q];
      }
      z[r] = cr;
    }
    double s = P->wq[cq * nq + q] * P->djq[cq * nq + q];
    if (P->kappa) s *= P->kappa[(size_t)c * nq + q];
    for (int r = 0; r < 3; ++r) Z4[r + 3 * q] = z[r] * s;
  }
  /* quad2dof, d = 3: Z3[k,i1,i2,j3] = sum_i3 M[3,k][i3,j3] Z4[k,i1,i2,i3] */
  for (int j3 = 0; j3 < SB; ++j3)
    for (int i2 = 0; i2 < SQ; ++i2)
      for (int i1 = 0; i1 < SQ; ++i1)
        for (int k = 0; k < 3; ++k) {
          double s = 0.0;
          for (int i3 = 0; i3 < SQ; ++i3)
            s += matel(A0, B0, SQ, 2, k, i3, j3) * Z4[k + 3 * (i1 + SQ * (i2 + SQ * i3))];
          Z3[k + 3 * (i1 + SQ * (i2 + SQ * j3))] = s;
        }
  /* d = 2: Z2[k,i1,j2,j3] = sum_i2 M[2,k][i2,j2] Z3[k,i1,i2,j3] */
  for (int j3 = 0; j3 < SB; ++j3)
    for (int j2 = 0; j2 < SB; ++j2)
      for (int i1 = 0; i1 < SQ; ++i1)
        for (int k = 0; k < 3; ++k) {
          double s = 0.0;
          for (int i2 = 0; i2 < SQ; ++i2)
            s += matel(A0, B0, SQ, 1, k, i2, j2) * Z3[k + 3 * (i1 + SQ * (i2 + SQ * j3))];
          Z2[k + 3 * (i1 + SQ * (j2 + SB * j3))] = s;
        }
  /* d = 1: Z1[k,j1,j2,j3] = sum_i1 M[1,k][i1,j1] Z2[k,i1,j2,j3] */
  for (int j3 = 0; j3 < SB; ++j3)
    for (int j2 = 0; j2 < SB; ++j2)
      for (int j1 = 0; j1 < SB; ++j1)
        for (int k = 0; k < 3; ++k) {
          double s = 0.0;
          for (int i1 = 0; i1 < SQ; ++i1)
            s += matel(A0, B0, SQ, 0, k, i1, j1) * Z2[k + 3 * (i1 + SQ * (j2 + SB * j3))];
          Z1[k + 3 * (j1 + SB * (j2 + SB * j3))] = s;
        }
  /* tensor2array + assemble: y[id] += sum_r Z1[r, dof_map[k]] */
  for (int k = 0; k < nloc; ++k) {
    const int32_t id = ids[k];
    if (id > 0) {
      const int t = tpos[k];
      y[id - 1] += Z1[0 + 3 * t] + Z1[1 + 3 * t] + Z1[2 + 3 * t];
    }
  }
}

#define SFREF_BODY(SBv, SQv)                                                         \
  static void run_##SBv##_##SQv(const sfref_problem* P, const int* tpos, const int64_t* cells, \
                                int64_t ncell_list, const double* x, double* y, double* W) { \
    double* Z1 = W;                                                                  \
    double* Z2 = Z1 + 3 * MAXS * MAXS * MAXS;                                        \
    double* Z3 = Z2 + 3 * MAXS * MAXS * MAXS;                                        \
    double* Z4 = Z3 + 3 * MAXS * MAXS * MAXS;                                        \
    for (int64_t t = 0; t < ncell_list; ++t)                                         \
      cell_eval(SBv, SQv, P, tpos, cells ? cells[t] : t, x, y, Z1, Z2, Z3, Z4);      \
  }

SFREF_BODY(2, 2) SFREF_BODY(2, 3) SFREF_BODY(3, 3) SFREF_BODY(3, 4) SFREF_BODY(4, 4)
SFREF_BODY(4, 5) SFREF_BODY(5, 4) SFREF_BODY(5, 5) SFREF_BODY(5, 6) SFREF_BODY(6, 6)
SFREF_BODY(6, 7) SFREF_BODY(7, 7) SFREF_BODY(7, 8) SFREF_BODY(8, 8) SFREF_BODY(9, 9)
SFREF_BODY(9, 10) SFREF_BODY(10, 10)

static void run_generic(int SB, int SQ, const sfref_problem* P, const int* tpos,
                        const int64_t* cells, int64_t n, const double* x, double* y, double* W) {
  double* Z1 = W;
  double* Z2 = Z1 + 3 * MAXS * MAXS * MAXS;
  double* Z3 = Z2 + 3 * MAXS * MAXS * MAXS;
  double* Z4 = Z3 + 3 * MAXS * MAXS * MAXS;
  for (int64_t t = 0; t < n; ++t) cell_eval(SB, SQ, P, tpos, cells ? cells[t] : t, x, y, Z1, Z2, Z3, Z4);
}

typedef void (*runfn)(const sfref_problem*, const int*, const int64_t*, int64_t, const double*,
                      double*, double*);

static runfn pick(int SB, int SQ) {
#define P_(a, b) \
  if (SB == a && SQ == b) return run_##a##_##b;
  P_(2, 2) P_(2, 3) P_(3, 3) P_(3, 4) P_(4, 4) P_(4, 5) P_(5, 4) P_(5, 5) P_(5, 6) P_(6, 6)
  P_(6, 7) P_(7, 7) P_(7, 8) P_(8, 8) P_(9, 9) P_(9, 10) P_(10, 10)
#undef P_
  return NULL;
}

/*
 * y = A x (mul!, src/LazyMatrices.jl:52-61). y is zeroed first.
 * colors: ncells int32 colour ids (cells of one colour share no dof) or NULL
 * (then nthreads must be 1). Returns 0 on success.
 */
int sfref_mul(int SB, int SQ, const double* A0, const double* B0, const int32_t* dof_map,
              int64_t ncells, const int32_t* cell_ids, int64_t n_free, int fill, const double* wq,
              const double* jq, const double* djq, const double* kappa, const double* x, double* y,
              int nthreads, const int32_t* colors, int ncolors) {
  if (SB < 1 || SB > MAXS || SQ < 1 || SQ > MAXS) return 1;
  sfref_problem P = {A0, B0, dof_map, ncells, cell_ids, fill, wq, jq, djq, kappa};
  const int nloc = SB * SB * SB;
  int tpos[MAXS * MAXS * MAXS];
  for (int k = 0; k < nloc; ++k) {
    const int j1 = dof_map[k] - 1, j2 = dof_map[k + nloc] - 1, j3 = dof_map[k + 2 * nloc] - 1;
    tpos[k] = j1 + SB * (j2 + SB * j3);
  }
  memset(y, 0, (size_t)n_free * sizeof(double));
  runfn f = pick(SB, SQ);
  const size_t wsz = 4 * 3 * MAXS * MAXS * MAXS;
  if (nthreads <= 1 || !colors) {
    double* W = (double*)malloc(wsz * sizeof(double));
    if (!W) return 2;
    if (f) f(&P, tpos, NULL, ncells, x, y, W);
    else run_generic(SB, SQ, &P, tpos, NULL, ncells, x, y, W);
    free(W);
    return 0;
  }
  /* bucket cells by colour */
  int64_t* start = (int64_t*)calloc((size_t)ncolors + 1, sizeof(int64_t));
  int64_t* order = (int64_t*)malloc((size_t)ncells * sizeof(int64_t));
  if (!start || !order) return 2;
  for (int64_t c = 0; c < ncells; ++c) start[colors[c] + 1]++;
  for (int k = 0; k < ncolors; ++k) start[k + 1] += start[k];
  int64_t* fillp = (int64_t*)malloc((size_t)ncolors * sizeof(int64_t));
  for (int k = 0; k < ncolors; ++k) fillp[k] = start[k];
  for (int64_t c = 0; c < ncells; ++c) order[fillp[colors[c]]++] = c;
  free(fillp);
#ifdef _OPENMP
  omp_set_num_threads(nthreads);
#endif
  for (int col = 0; col < ncolors; ++col) {
    const int64_t b = start[col], e = start[col + 1];
#pragma omp parallel
    {
      double* W = (double*)malloc(wsz * sizeof(double));
#pragma omp for schedule(static)
      for (int64_t t = b; t < e; t += 64) {
        const int64_t n = (e - t) < 64 ? (e - t) : 64;
        if (f) f(&P, tpos, order + t, n, x, y, W);
        else run_generic(SB, SQ, &P, tpos, order + t, n, x, y, W);
      }
      free(W);
    }
  }
  free(start);
  free(order);
  return 0;
}

int sfref_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
