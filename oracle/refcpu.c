/*
 * refcpu.c -- CPU restatement of fastSolver's HODLR direct solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle: the parity tests,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg call it as the
 * checker.  Nothing in the product (fastsolver_b200/) links or calls it.
 *
 * It restates, function by function, the FP64 CPU path of
 * Charles-Chao-Chen/fastSolver (paths are relative to that project):
 *
 *   ref_build_tree        src/htree/hodlr_matrix.cc:44-82, 138-169, 354-386
 *                         (balanced N/2, N-N/2 split, col_beg chaining, V tree
 *                         with the children's ranks swapped); node order is the
 *                         BFS order of solve_bfs (src/solver/fast_solver.cc:136-171)
 *   ref_leaf_solve        src/solver/solver_tasks.cc:424-450 (dgesv on a leaf)
 *   ref_schur2_solve      src/solver/solver_tasks.cc:452-549 (2r x 2r permuted
 *                         Schur system of the leaf-internal branch)
 *   ref_gemm_reduce       src/solver/gemm.cc:315-384 (W += alpha V^T U[:,cols])
 *   ref_lu_node_solve     src/solver/solver_tasks.cc:139-305 (r x r reduced form)
 *   ref_gemm_broadcast    src/solver/gemm.cc:417-478 (d = beta d + alpha u eta)
 *   ref_bfs_solve         src/solver/fast_solver.cc:136-255 (reverse-BFS walk;
 *                         per node 4 reduces -> LU -> 2 broadcasts)
 *   ref_fill_circulant_u  src/legion_matrix/init_matrix_tasks.cc:176-219
 *   ref_fill_circulant_k  src/htree/hodlr_matrix.cc:528-567
 *   ref_drand48_fill      src/legion_matrix/init_matrix_tasks.cc:43-77 and
 *                         src/solver/direct_solve.cc:134-147 (drand48_r stream,
 *                         reseeded per region, row-major fill)
 *   ref_dense_solve       src/solver/direct_solve.cc:168-195 (dense dgesv)
 *   ref_rel_error         src/solver/direct_solve.cc:216-225 (the "Err:" formula)
 *
 * plus two routines with no reference counterpart that the GPU refinement
 * path needs an oracle for: ref_hodlr_matvec (A x from D, U, V) and the dense
 * assembly ref_hodlr_dense.
 *
 * Parity unpinned: the reference cannot be built or run without Legion, and
 * its known-answer test (test/single_launch.cc:20-75) stores no expected
 * numbers (it compares against a dense solve), so this oracle is checked
 * against tests/golden/, which tests/golden/make_golden.py computes from the
 * same known-answer inputs with numpy alone, not against outputs of the
 * reference itself.
 *
 * Arithmetic is LAPACK/BLAS dgesv_/dgemm_ as in the reference
 * (include/core/lapack_blas.h:28-55).  The reference links an unpinned system
 * netlib/MKL LAPACK; here the same Fortran-ABI routines are resolved at run
 * time from the OpenBLAS that scipy bundles (exported as scipy_dgemm_,
 * scipy_dgesv_), via ref_load_blas(path).
 *
 * Data layout (global, column-major):
 *   X  N x C   [b | U_1 .. U_L]: rows of every leaf hold b and the U block of
 *              each ancestor level (column block of node c = [c.col_beg,
 *              c.col_beg + c.ncol)), LD = ldx
 *   V  N x rL  V factor of node c (rows of c) in columns
 *              [c.col_beg - m, c.col_beg - m + c.vncol), LD = ldv
 *   D  N x nmax  leaf diagonal blocks stacked vertically (leaf rows, columns
 *              0..n-1), LD = ldd -- the K region layout of hodlr_matrix.cc:431-445
 */
#include <dlfcn.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef void (*dgemm_fn)(const char *, const char *, const int *, const int *,
                         const int *, const double *, const double *,
                         const int *, const double *, const int *,
                         const double *, double *, const int *);
typedef void (*dgesv_fn)(const int *, const int *, double *, const int *,
                         int *, double *, const int *, int *);
typedef void (*setthreads_fn)(int);

static dgemm_fn p_dgemm = 0;
static dgesv_fn p_dgesv = 0;
static setthreads_fn p_setthreads = 0;

/* Resolve dgemm/dgesv from a BLAS/LAPACK shared library.  Returns 0 on
 * success, -1 if the library cannot be opened, -2 if a symbol is missing. */
int ref_load_blas(const char *path) {
  void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
  if (!h) return -1;
  p_dgemm = (dgemm_fn)dlsym(h, "scipy_dgemm_");
  if (!p_dgemm) p_dgemm = (dgemm_fn)dlsym(h, "dgemm_");
  p_dgesv = (dgesv_fn)dlsym(h, "scipy_dgesv_");
  if (!p_dgesv) p_dgesv = (dgesv_fn)dlsym(h, "dgesv_");
  p_setthreads = (setthreads_fn)dlsym(h, "scipy_openblas_set_num_threads");
  if (!p_setthreads) p_setthreads = (setthreads_fn)dlsym(h, "openblas_set_num_threads");
  if (!p_dgemm || !p_dgesv) return -2;
  return 0;
}

int ref_blas_loaded(void) { return p_dgemm && p_dgesv; }

void ref_set_blas_threads(int n) {
  if (p_setthreads) p_setthreads(n);
}

int ref_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static void dgemm(char ta, char tb, int m, int n, int k, double alpha,
                  const double *A, int lda, const double *B, int ldb,
                  double beta, double *C, int ldc) {
  if (m <= 0 || n <= 0) return;
  if (k <= 0) {
    /* BLAS semantics: C = beta C when k == 0 */
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < m; ++i) C[i + (size_t)j * ldc] *= beta;
    return;
  }
  p_dgemm(&ta, &tb, &m, &n, &k, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}

static int dgesv(int n, int nrhs, double *A, int lda, int *ipiv, double *B,
                 int ldb) {
  int info = 0;
  if (n <= 0) return 0;
  if (nrhs <= 0) {
    /* still factor A: solve against one scratch column */
    int one = 1;
    double *tmp = (double *)calloc((size_t)n, sizeof(double));
    p_dgesv(&n, &one, A, &lda, ipiv, tmp, &n, &info);
    free(tmp);
    return info;
  }
  p_dgesv(&n, &nrhs, A, &lda, ipiv, B, &ldb, &info);
  return info;
}

/* ------------------------------------------------------------------------ */
/* Tree                                                                     */
/* ------------------------------------------------------------------------ */

/* Node record, REF_NODE_FIELDS ints per node, BFS order, node 0 = root. */
enum {
  F_NROW = 0, F_NCOL, F_ROWBEG, F_COLBEG, F_LCHILD, F_RCHILD, F_PARENT,
  F_DEPTH, F_VNCOL, F_ISLEAF, REF_NODE_FIELDS
};

int ref_node_fields(void) { return REF_NODE_FIELDS; }

/* Builds the U tree of hodlr_matrix.cc:44-82 / 138-169 for leafSize == 1:
 * the root holds nrhs columns; a node with nrow > threshold splits into
 * N/2 and N - N/2 rows; each child carries `rank` columns starting at
 * parent.col_beg + parent.ncol.  The V tree (hodlr_matrix.cc:354-386) has the
 * same rows with the children's column counts swapped; its ncol is stored as
 * F_VNCOL.  Nodes are written in BFS order (fast_solver.cc:152-171).
 * Returns the node count, or -1 if cap is too small, -2 on a bad argument
 * (the reference asserts nrow > rank at every leaf, hodlr_matrix.cc:167). */
int ref_build_tree(int N, int nrhs, int rank, int threshold, int *out,
                   int cap) {
  if (N <= 0 || nrhs < 0 || rank <= 0 || threshold <= 0) return -2;
  if (cap < 1) return -1;
  int *t = out;
  int nn = 1;
  int *root = t;
  root[F_NROW] = N; root[F_NCOL] = nrhs; root[F_ROWBEG] = 0; root[F_COLBEG] = 0;
  root[F_LCHILD] = -1; root[F_RCHILD] = -1; root[F_PARENT] = -1;
  root[F_DEPTH] = 0; root[F_VNCOL] = 0; root[F_ISLEAF] = 1;
  for (int i = 0; i < nn; ++i) {
    int *p = t + (size_t)i * REF_NODE_FIELDS;
    int n = p[F_NROW];
    if (n > threshold) {
      if (nn + 2 > cap) return -1;
      int li = nn, ri = nn + 1;
      nn += 2;
      int *l = t + (size_t)li * REF_NODE_FIELDS;
      int *r = t + (size_t)ri * REF_NODE_FIELDS;
      l[F_NROW] = n / 2;       r[F_NROW] = n - n / 2;
      l[F_NCOL] = rank;        r[F_NCOL] = rank;
      l[F_COLBEG] = p[F_COLBEG] + p[F_NCOL];
      r[F_COLBEG] = p[F_COLBEG] + p[F_NCOL];
      l[F_ROWBEG] = p[F_ROWBEG];
      r[F_ROWBEG] = p[F_ROWBEG] + l[F_NROW];
      l[F_LCHILD] = l[F_RCHILD] = r[F_LCHILD] = r[F_RCHILD] = -1;
      l[F_PARENT] = r[F_PARENT] = i;
      l[F_DEPTH] = r[F_DEPTH] = p[F_DEPTH] + 1;
      /* V tree: lchild gets rchild's ncol and vice versa (hodlr_matrix.cc:359-360) */
      l[F_VNCOL] = r[F_NCOL];
      r[F_VNCOL] = l[F_NCOL];
      l[F_ISLEAF] = r[F_ISLEAF] = 1;
      p[F_LCHILD] = li; p[F_RCHILD] = ri; p[F_ISLEAF] = 0;
    } else {
      if (!(n > rank)) return -2;
    }
  }
  return nn;
}

/* ------------------------------------------------------------------------ */
/* Task bodies                                                              */
/* ------------------------------------------------------------------------ */

/* solver_tasks.cc:424-450: dgesv(D_leaf, X_leaf) on all nrhs columns.
 * D is overwritten by its LU factors, X by the solution.  Returns INFO. */
int ref_leaf_solve(int n, int nrhs, double *D, int ldd, double *X, int ldx,
                   int *ipiv) {
  int *piv = ipiv;
  int *tmp = 0;
  if (!piv) { tmp = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1)); piv = tmp; }
  int info = dgesv(n, nrhs, D, ldd, piv, X, ldx);
  free(tmp);
  return info;
}

/* gemm.cc:315-384: W(r x ncol) += alpha * V^T(r x k) * U[:, col_beg:col_beg+ncol]
 * (beta = 1 into the reduction region). */
void ref_gemm_reduce(double alpha, int k, int r, int ncol, const double *V,
                     int ldv, const double *U, int ldu, int col_beg,
                     double *W, int ldw) {
  dgemm('t', 'n', r, ncol, k, alpha, V, ldv, U + (size_t)col_beg * ldu, ldu,
        1.0, W, ldw);
}

/* gemm.cc:417-478: X[:, d_col_beg : d_col_beg+c] = beta * X + alpha *
 * X[:, u_col_beg : u_col_beg+r] * eta(r x c); U and d share one region. */
void ref_gemm_broadcast(double alpha, double beta, int k, int r, int c,
                        double *U, int ldu, int u_col_beg, const double *eta,
                        int lde, int d_col_beg) {
  dgemm('n', 'n', k, c, r, alpha, U + (size_t)u_col_beg * ldu, ldu, eta, lde,
        beta, U + (size_t)d_col_beg * ldu, ldu);
}

/* solver_tasks.cc:139-305 (LUSolveTask): with V0Tu0 (r1 x r0), V1Tu1 (r0 x r1),
 * V0Td0 (r1 x c), V1Td1 (r0 x c):
 *   V1Td1 -= V1Tu1 * V0Td0
 *   S = I - V1Tu1 * V0Tu0               (r0 x r0)
 *   eta0 = S^{-1} V1Td1   -> V1Td1
 *   eta1 = V0Td0 - V0Tu0 * eta0  -> V0Td0
 * Returns the dgesv INFO. */
int ref_lu_node_solve(int r0, int r1, int c, const double *V0Tu0, int ld00,
                      const double *V1Tu1, int ld11, double *V0Td0, int ld0d,
                      double *V1Td1, int ld1d) {
  dgemm('n', 'n', r0, c, r1, -1.0, V1Tu1, ld11, V0Td0, ld0d, 1.0, V1Td1, ld1d);
  int N = r0;
  double *S = (double *)calloc((size_t)N * N, sizeof(double));
  for (int i = 0; i < N; ++i) S[i * (N + 1)] = 1.0;
  dgemm('n', 'n', r0, r0, r1, -1.0, V1Tu1, ld11, V0Tu0, ld00, 1.0, S, N);
  int *ipiv = (int *)malloc(sizeof(int) * (size_t)N);
  int info = dgesv(N, c, S, N, ipiv, V1Td1, ld1d);
  free(ipiv);
  free(S);
  if (info != 0) return info;
  dgemm('n', 'n', r1, c, r0, -1.0, V0Tu0, ld00, V1Td1, ld1d, 1.0, V0Td0, ld0d);
  return 0;
}

/* solver_tasks.cc:483-535: the 2r x 2r form.  S = [[V0Tu0, I],[I, V1Tu1]]
 * with V0Tu0 (r1 x r0) top-left, V1Tu1 (r0 x r1) bottom-right, identity
 * blocks placed at S[(r1 + i) % (r0 + r1), i]; right-hand side
 * [V0Td0; V1Td1].  On return V0Td0 <- eta0 (r0 x c, first r0 rows of the
 * solution) and V1Td1 <- eta1 (r1 x c).  Returns the dgesv INFO. */
int ref_schur2_solve(int r0, int r1, int c, const double *V0Tu0, int ld00,
                     const double *V1Tu1, int ld11, double *V0Td0, int ld0d,
                     double *V1Td1, int ld1d) {
  int s = r0 + r1;
  double *S = (double *)calloc((size_t)s * s, sizeof(double));
  double *R = (double *)malloc(sizeof(double) * (size_t)s * (c > 0 ? c : 1));
  for (int i = 0; i < s; ++i) S[(r1 + i) % s + (size_t)i * s] = 1.0;
  for (int j = 0; j < r0; ++j)
    for (int i = 0; i < r1; ++i) S[i + (size_t)j * s] = V0Tu0[i + (size_t)j * ld00];
  for (int j = 0; j < r1; ++j)
    for (int i = 0; i < r0; ++i)
      S[(r1 + i) + (size_t)(r0 + j) * s] = V1Tu1[i + (size_t)j * ld11];
  for (int j = 0; j < c; ++j) {
    for (int i = 0; i < r1; ++i) R[i + (size_t)j * s] = V0Td0[i + (size_t)j * ld0d];
    for (int i = 0; i < r0; ++i) R[r1 + i + (size_t)j * s] = V1Td1[i + (size_t)j * ld1d];
  }
  int *ipiv = (int *)malloc(sizeof(int) * (size_t)s);
  int info = dgesv(s, c, S, s, ipiv, R, s);
  if (info == 0) {
    for (int j = 0; j < c; ++j) {
      for (int i = 0; i < r0; ++i) V0Td0[i + (size_t)j * ld0d] = R[i + (size_t)j * s];
      for (int i = 0; i < r1; ++i) V1Td1[i + (size_t)j * ld1d] = R[r0 + i + (size_t)j * s];
    }
  }
  free(ipiv);
  free(S);
  free(R);
  return info;
}

/* ------------------------------------------------------------------------ */
/* Walk                                                                     */
/* ------------------------------------------------------------------------ */

#define ND(t, i) ((t) + (size_t)(i) * REF_NODE_FIELDS)

/* Collect the leaves under node `i`, left to right. */
static int collect_leaves(const int *t, int i, int *out, int k) {
  const int *p = ND(t, i);
  if (p[F_ISLEAF]) { out[k++] = i; return k; }
  k = collect_leaves(t, p[F_LCHILD], out, k);
  return collect_leaves(t, p[F_RCHILD], out, k);
}

/* gemm.cc:208-229 + 144-205: create a zeroed r x ncol result and sum
 * V^T U[:, cols] over the leaves under `child`, leaf by leaf (the REDOP_ADD
 * accumulation, applied in left-to-right leaf order). */
static void reduce_subtree(const int *t, int child, int *leafbuf,
                           const double *V, int ldv, int voff, int vrows_cols,
                           const double *X, int ldx, int col_beg, int ncol,
                           double *W, int ldw) {
  for (int j = 0; j < ncol; ++j) memset(W + (size_t)j * ldw, 0, sizeof(double) * (size_t)vrows_cols);
  int nl = collect_leaves(t, child, leafbuf, 0);
  for (int q = 0; q < nl; ++q) {
    const int *lf = ND(t, leafbuf[q]);
    int rb = lf[F_ROWBEG];
    ref_gemm_reduce(1.0, lf[F_NROW], vrows_cols, ncol,
                    V + rb + (size_t)voff * ldv, ldv, X + rb, ldx, col_beg, W, ldw);
  }
}

static void broadcast_subtree(const int *t, int child, int *leafbuf,
                              double *X, int ldx, int u_col_beg, int r,
                              const double *eta, int lde, int c) {
  int nl = collect_leaves(t, child, leafbuf, 0);
  for (int q = 0; q < nl; ++q) {
    const int *lf = ND(t, leafbuf[q]);
    int rb = lf[F_ROWBEG];
    ref_gemm_broadcast(-1.0, 1.0, lf[F_NROW], r, c, X + rb, ldx, u_col_beg, eta, lde, 0);
  }
}

/* fast_solver.cc:191-255 `visit` for an internal node; inside a Legion leaf
 * (at most leaf_size real leaves below, mark_legion_leaf at
 * hodlr_matrix.cc:317-337) the node is solved by serial_leaf_solve's internal
 * branch (solver_tasks.cc:452-549) with the 2r x 2r form. */
static int visit_internal(const int *t, int nn, int i, double *X, int ldx,
                          const double *V, int ldv, int m, int schur2, int leaf_size) {
  const int *p = ND(t, i);
  const int *b0 = ND(t, p[F_LCHILD]);
  const int *b1 = ND(t, p[F_RCHILD]);
  int r0 = b0[F_NCOL], r1 = b1[F_NCOL];
  int v0c = b0[F_VNCOL], v1c = b1[F_VNCOL]; /* = r1, r0 */
  int c0 = b0[F_COLBEG], c1 = b1[F_COLBEG];
  int c = c0; /* rd0 = rd1 = [0, col_beg) */
  int *leafbuf = (int *)malloc(sizeof(int) * (size_t)nn);
  if (!schur2 && collect_leaves(t, i, leafbuf, 0) <= leaf_size) schur2 = 1;
  double *V0Tu0 = (double *)malloc(sizeof(double) * (size_t)v0c * r0);
  double *V1Tu1 = (double *)malloc(sizeof(double) * (size_t)v1c * r1);
  double *V0Td0 = (double *)malloc(sizeof(double) * (size_t)v0c * (c > 0 ? c : 1));
  double *V1Td1 = (double *)malloc(sizeof(double) * (size_t)v1c * (c > 0 ? c : 1));
  int voff0 = c0 - m, voff1 = c1 - m;
  reduce_subtree(t, p[F_LCHILD], leafbuf, V, ldv, voff0, v0c, X, ldx, c0, r0, V0Tu0, v0c);
  reduce_subtree(t, p[F_RCHILD], leafbuf, V, ldv, voff1, v1c, X, ldx, c1, r1, V1Tu1, v1c);
  reduce_subtree(t, p[F_LCHILD], leafbuf, V, ldv, voff0, v0c, X, ldx, 0, c, V0Td0, v0c);
  reduce_subtree(t, p[F_RCHILD], leafbuf, V, ldv, voff1, v1c, X, ldx, 0, c, V1Td1, v1c);
  int info;
  const double *eta0, *eta1;
  if (!schur2) {
    info = ref_lu_node_solve(r0, r1, c, V0Tu0, v0c, V1Tu1, v1c, V0Td0, v0c, V1Td1, v1c);
    eta0 = V1Td1; eta1 = V0Td0; /* fast_solver.cc:238-240 */
  } else {
    info = ref_schur2_solve(r0, r1, c, V0Tu0, v0c, V1Tu1, v1c, V0Td0, v0c, V1Td1, v1c);
    eta0 = V0Td0; eta1 = V1Td1; /* solver_tasks.cc:524-525 */
  }
  if (info == 0) {
    broadcast_subtree(t, p[F_LCHILD], leafbuf, X, ldx, c0, r0, eta0, r0, c);
    broadcast_subtree(t, p[F_RCHILD], leafbuf, X, ldx, c1, r1, eta1, r1, c);
  }
  free(leafbuf); free(V0Tu0); free(V1Tu1); free(V0Td0); free(V1Td1);
  return info;
}

/* fast_solver.cc:136-255 (solve_bfs + visit).  Visits the nodes in reverse
 * BFS order; nodes of equal depth touch disjoint rows, so each depth is run as
 * one parallel loop over `nthreads` OpenMP threads with single-threaded BLAS
 * (the reference runs one Legion task per CPU processor, sequential BLAS).
 * `m` is the root's column count (nrhs).  D is overwritten with the leaf LU
 * factors, X[:, 0:m] with the solution.  schur2 != 0 uses the 2r x 2r node
 * form instead of LUSolveTask's r x r form.  Returns 0 or the first nonzero
 * INFO (leaf: its value; node: 100000 + value). */
int ref_bfs_solve_ls(const int *t, int nn, double *X, int ldx, const double *V,
                     int ldv, double *D, int ldd, int nthreads, int schur2,
                     int leaf_size);

int ref_bfs_solve(const int *t, int nn, double *X, int ldx, const double *V,
                  int ldv, double *D, int ldd, int nthreads, int schur2) {
  return ref_bfs_solve_ls(t, nn, X, ldx, V, ldv, D, ldd, nthreads, schur2, 1);
}

/* ref_bfs_solve with the reference's task granularity leafSize (the nodes
 * inside a Legion leaf take the 2r x 2r form). */
int ref_bfs_solve_ls(const int *t, int nn, double *X, int ldx, const double *V,
                     int ldv, double *D, int ldd, int nthreads, int schur2,
                     int leaf_size) {
  int m = t[F_NCOL];
  int maxd = 0;
  for (int i = 0; i < nn; ++i) if (ND(t, i)[F_DEPTH] > maxd) maxd = ND(t, i)[F_DEPTH];
  int status = 0;
  if (nthreads < 1) nthreads = 1;
  for (int d = maxd; d >= 0; --d) {
    int lo = -1, hi = -1; /* BFS order: nodes of depth d are contiguous */
    for (int i = 0; i < nn; ++i)
      if (ND(t, i)[F_DEPTH] == d) { if (lo < 0) lo = i; hi = i; }
    if (lo < 0) continue;
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int i = hi; i >= lo; --i) {
      const int *p = ND(t, i);
      int info;
      if (p[F_ISLEAF]) {
        int rb = p[F_ROWBEG];
        info = ref_leaf_solve(p[F_NROW], p[F_COLBEG] + p[F_NCOL], D + rb, ldd,
                              X + rb, ldx, 0);
      } else {
        info = visit_internal(t, nn, i, X, ldx, V, ldv, m, schur2, leaf_size);
        if (info) info += 100000;
      }
      if (info) {
#ifdef _OPENMP
#pragma omp critical
#endif
        { if (!status) status = info; }
      }
    }
    if (status) return status;
  }
  return status;
}

/* ------------------------------------------------------------------------ */
/* Matvec and dense assembly (no reference counterpart)                     */
/* ------------------------------------------------------------------------ */

/* y = A x for the HODLR matrix A = blockdiag(D_leaf) + sum over sibling pairs
 * (c0, c1) of U_c0 V_c1^T (rows c0, cols c1) and U_c1 V_c0^T.  U is the
 * original U (N x rL, column block of node c at c.col_beg - m), V as above.
 * x, y: N x m. */
void ref_hodlr_matvec(const int *t, int nn, const double *D, int ldd,
                      const double *U, int ldu, const double *V, int ldv,
                      const double *x, int ldxx, double *y, int ldy, int m) {
  int mroot = t[F_NCOL];
  for (int j = 0; j < m; ++j) memset(y + (size_t)j * ldy, 0, sizeof(double) * (size_t)t[F_NROW]);
  double *tmp = 0;
  size_t tmpsz = 0;
  for (int i = 0; i < nn; ++i) {
    const int *p = ND(t, i);
    if (p[F_ISLEAF]) {
      int rb = p[F_ROWBEG];
      dgemm('n', 'n', p[F_NROW], m, p[F_NROW], 1.0, D + rb, ldd, x + rb, ldxx,
            1.0, y + rb, ldy);
      continue;
    }
    for (int s = 0; s < 2; ++s) {
      const int *c = ND(t, s == 0 ? p[F_LCHILD] : p[F_RCHILD]);   /* row side */
      const int *o = ND(t, s == 0 ? p[F_RCHILD] : p[F_LCHILD]);   /* col side */
      int rc = c[F_NCOL];
      size_t need = (size_t)rc * m;
      if (need > tmpsz) { free(tmp); tmp = (double *)malloc(sizeof(double) * need); tmpsz = need; }
      /* tmp = V_o^T x_o (V_o has vncol(o) = ncol(c) columns) */
      dgemm('t', 'n', rc, m, o[F_NROW], 1.0,
            V + o[F_ROWBEG] + (size_t)(o[F_COLBEG] - mroot) * ldv, ldv,
            x + o[F_ROWBEG], ldxx, 0.0, tmp, rc);
      dgemm('n', 'n', c[F_NROW], m, rc, 1.0,
            U + c[F_ROWBEG] + (size_t)(c[F_COLBEG] - mroot) * ldu, ldu, tmp, rc,
            1.0, y + c[F_ROWBEG], ldy);
    }
  }
  free(tmp);
}

/* Dense N x N assembly of the same matrix (column-major, LD = lda). */
void ref_hodlr_dense(const int *t, int nn, const double *D, int ldd,
                     const double *U, int ldu, const double *V, int ldv,
                     double *A, int lda) {
  int N = t[F_NROW];
  int mroot = t[F_NCOL];
  for (int j = 0; j < N; ++j) memset(A + (size_t)j * lda, 0, sizeof(double) * (size_t)N);
  for (int i = 0; i < nn; ++i) {
    const int *p = ND(t, i);
    if (p[F_ISLEAF]) {
      int rb = p[F_ROWBEG], n = p[F_NROW];
      for (int j = 0; j < n; ++j)
        memcpy(A + rb + (size_t)(rb + j) * lda, D + rb + (size_t)j * ldd, sizeof(double) * (size_t)n);
      continue;
    }
    for (int s = 0; s < 2; ++s) {
      const int *c = ND(t, s == 0 ? p[F_LCHILD] : p[F_RCHILD]);
      const int *o = ND(t, s == 0 ? p[F_RCHILD] : p[F_LCHILD]);
      dgemm('n', 't', c[F_NROW], o[F_NROW], c[F_NCOL], 1.0,
            U + c[F_ROWBEG] + (size_t)(c[F_COLBEG] - mroot) * ldu, ldu,
            V + o[F_ROWBEG] + (size_t)(o[F_COLBEG] - mroot) * ldv, ldv, 0.0,
            A + c[F_ROWBEG] + (size_t)o[F_ROWBEG] * lda, lda);
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Generators of the reference's known-answer test                           */
/* ------------------------------------------------------------------------ */

/* glibc drand48_r: 48-bit LCG x' = (0x5DEECE66D x + 0xB) mod 2^48 seeded by
 * srand48_r(seed) as x = (seed << 16) | 0x330E, returning x' / 2^48.
 * Fills an nrow x ncol block row by row (init_matrix_tasks.cc:66-76). */
void ref_drand48_fill(long seed, int nrow, int ncol, double *out, int ld) {
  uint64_t x = (((uint64_t)(uint32_t)seed) << 16) | 0x330Eu;
  const uint64_t a = 0x5DEECE66Dull, c = 0xBull, mask = (1ull << 48) - 1;
  for (int i = 0; i < nrow; ++i)
    for (int j = 0; j < ncol; ++j) {
      x = (a * x + c) & mask;
      out[i + (size_t)j * ld] = ldexp((double)x, -48);
    }
}

/* init_matrix_tasks.cc:176-219: value (j + i + row_beg) % r at column
 * col_beg + j, row i, for j in [0, ncol - col_beg). */
void ref_fill_circulant_u(int nrow, int ncol, int col_beg, int row_beg, int r,
                          double *ptr, int ld) {
  for (int j = 0; j < ncol - col_beg; ++j)
    for (int i = 0; i < nrow; ++i)
      ptr[i + (size_t)(j + col_beg) * ld] = (double)((j + i + row_beg) % r);
}

/* hodlr_matrix.cc:528-567 for one leaf: K = U U^T + diag I with
 * U(i, j) = (row_glo + i + j) % r, written at K[0:n, 0:n] (LD = ld). */
void ref_fill_circulant_k(int n, int row_glo, int r, double diag, double *K,
                          int ld) {
  double *U = (double *)malloc(sizeof(double) * (size_t)n * r);
  for (int j = 0; j < r; ++j)
    for (int i = 0; i < n; ++i) U[i + (size_t)j * n] = (double)((row_glo + i + j) % r);
  for (int j = 0; j < n; ++j) memset(K + (size_t)j * ld, 0, sizeof(double) * (size_t)n);
  for (int i = 0; i < n; ++i) K[i + (size_t)ld * i] = diag;
  dgemm('n', 't', n, n, r, 1.0, U, n, U, n, 1.0, K, ld);
  free(U);
}

/* direct_solve.cc:168-195: dense dgesv, B overwritten. Returns INFO. */
int ref_dense_solve(int n, int nrhs, double *A, int lda, double *B, int ldb) {
  int *ipiv = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
  int info = dgesv(n, nrhs, A, lda, ipiv, B, ldb);
  free(ipiv);
  return info;
}

/* direct_solve.cc:216-225: sqrt(sum (x - x_ref)^2 / sum x_ref^2). */
double ref_rel_error(int n, int m, const double *x, int ldx, const double *xref,
                     int ldr) {
  double diff = 0, den = 0;
  for (int j = 0; j < m; ++j)
    for (int i = 0; i < n; ++i) {
      double a = x[i + (size_t)j * ldx], b = xref[i + (size_t)j * ldr];
      diff += (a - b) * (a - b);
      den += b * b;
    }
  return sqrt(diff / den);
}
