/*
 * hodlr_gpu.h -- C ABI of the B200 HODLR direct solver.
 *
 * Drop-in for the four task bodies of Charles-Chao-Chen/fastSolver's HODLR
 * solve (paths relative to that project) plus the handle API that walks the
 * tree the way FastSolver::bfs_solve does.
 *
 * Conventions
 *   - Matrices are column-major FP64 with an explicit leading dimension, as the
 *     reference's Legion regions are (raw_rect_ptr with LD == rows,
 *     src/solver/solver_tasks.cc:408-410).
 *   - Every pointer passed to a task body is a DEVICE pointer on the current
 *     CUDA device; `stream` is a cudaStream_t passed as void* (NULL = legacy
 *     default stream).
 *   - Every call returns an int status: 0 = ok; > 0 = LAPACK-style INFO (the
 *     1-based index of the first exactly-zero pivot); < 0 = bad argument
 *     (-i: argument i is invalid) or one of the HODLR_ERR_* codes below.
 *     The reference aborts via assert instead (solver_tasks.cc:284, 438, 516).
 *   - Task bodies with an `info` argument are asynchronous when `info` is a
 *     device pointer: they return after the launch and write INFO there.  When
 *     `info` is NULL they synchronize `stream` and return INFO as the status.
 *   - No entry point falls back to the CPU: without a usable CUDA device they
 *     return HODLR_ERR_CUDA.
 */
#ifndef HODLR_GPU_H
#define HODLR_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

typedef void *hodlr_stream_t; /* cudaStream_t */

#define HODLR_OK 0
#define HODLR_ERR_CUDA (-1000)     /* CUDA runtime error / no device */
#define HODLR_ERR_NOMEM (-1001)    /* device allocation failed */
#define HODLR_ERR_STATE (-1002)    /* call out of order (e.g. solve before factor) */
#define HODLR_ERR_NOCONV (-1003)   /* refinement did not reach the tolerance */
#define HODLR_ERR_TIMEOUT (-1004)  /* a bounded device wait gave up */
#define HODLR_ERR_UNSUPPORTED (-1005)
#define HODLR_ERR_IO (-1006)       /* text file could not be opened / parsed */

#define HODLR_PREC_FP64 0  /* FP64 throughout (the reference's arithmetic) */
#define HODLR_PREC_MIXED 1 /* FP32 leaf LU + split-BF16 tensor-core GEMMs,
                              FP64 node LU, residual and refinement */

/* ------------------------------------------------------------------------ */
/* Task bodies                                                              */
/* ------------------------------------------------------------------------ */

/* Leaf solve: dgesv of one leaf block on all its columns [b | U_anc].
 * D (n x n, ldd) is overwritten by P*L*U (LAPACK dgetrf layout), X
 * (n x nrhs, ldx) by D^{-1} X, ipiv (n ints, device) by LAPACK pivots (1-based).
 * Replaces LeafSolveTask::cpu_task, real-leaf branch:
 *   src/solver/solver_tasks.cc:341-412 (task), 424-450 (dgesv at 437). */
int hodlr_leaf_solve(int n, int nrhs, double *D, int ldd, double *X, int ldx,
                     int *ipiv, int *info, hodlr_stream_t stream);

/* Upward reduce: W(r x ncol) += alpha * V(k x r)^T * U[:, col_beg:col_beg+ncol].
 * U is k x (col_beg+ncol) (ldu).  Replaces GEMM_Reduce_Task::cpu_task:
 *   src/solver/gemm.cc:315-384 (dgemm at 376; beta = 1 into the REDOP_ADD
 *   region, which gemm_reduce zeroes first, gemm.cc:216-221). */
int hodlr_gemm_reduce(double alpha, int k, int r, int ncol, const double *V,
                      int ldv, const double *U, int ldu, int col_beg,
                      double *W, int ldw, hodlr_stream_t stream);

/* Same result as hodlr_gemm_reduce, allocating no device memory: for callers
 * that cannot allocate, e.g. task bodies under a runtime that owns the GPU's
 * memory (Legion/Realm reserves the framebuffer and hands tasks only mapped
 * regions) or services that pre-reserve all device memory.  No counterpart in
 * the reference.  Its split-K partial sums live in a fixed 8 MiB array in the
 * library's device image (held by every GPU that loads the library until the
 * process exits); r * ncol must not exceed 2^20, else the call returns
 * HODLR_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress) and should come before any stream capture.
 * All calls share the array: calls that overlap on the GPU race.
 * Asynchronous on `stream`. */
int hodlr_gemm_reduce_noalloc(double alpha, int k, int r, int ncol,
                              const double *V, int ldv, const double *U,
                              int ldu, int col_beg, double *W, int ldw,
                              hodlr_stream_t stream);

/* Node solve, r x r reduced Schur form.  V0Tu0 is r1 x r0, V1Tu1 r0 x r1,
 * V0Td0 r1 x c, V1Td1 r0 x c:
 *   V1Td1 -= V1Tu1 V0Td0;  S = I - V1Tu1 V0Tu0;  V1Td1 <- eta0 = S^{-1} V1Td1;
 *   V0Td0 <- eta1 = V0Td0 - V0Tu0 eta0.
 * Replaces LUSolveTask::cpu_task: src/solver/solver_tasks.cc:139-305. */
int hodlr_node_lu_solve(int r0, int r1, int c, const double *V0Tu0, int ld00,
                        const double *V1Tu1, int ld11, double *V0Td0,
                        int ld0d, double *V1Td1, int ld1d, int *info,
                        hodlr_stream_t stream);

/* Node solve, 2r x 2r permuted Schur form [[V0Tu0, I], [I, V1Tu1]] with
 * right-hand side [V0Td0; V1Td1]; on return V0Td0 <- eta0 (first r0 rows of
 * the solution), V1Td1 <- eta1.  Replaces the leaf-internal branch of
 * serial_leaf_solve: src/solver/solver_tasks.cc:483-535 (dgesv at 515).
 * Uniform rank (r0 == r1) as in the reference's HodlrMatrix. */
int hodlr_node_schur2_solve(int r0, int r1, int c, const double *V0Tu0,
                            int ld00, const double *V1Tu1, int ld11,
                            double *V0Td0, int ld0d, double *V1Td1, int ld1d,
                            int *info, hodlr_stream_t stream);

/* Downward broadcast: X[:, d_col_beg:d_col_beg+c] =
 *   beta * X[:, d_col_beg:...] + alpha * X[:, u_col_beg:u_col_beg+r] * eta(r x c)
 * on one k-row region X (ldx); the u and d column ranges must not overlap.
 * Replaces GEMM_Broadcast_Task::cpu_task: src/solver/gemm.cc:417-478 (dgemm at
 * 473; the solver calls it with alpha = -1, beta = 1, fast_solver.cc:250-253). */
int hodlr_gemm_broadcast(double alpha, double beta, int k, int r, int c,
                         double *X, int ldx, int u_col_beg, const double *eta,
                         int lde, int d_col_beg, hodlr_stream_t stream);

/* ------------------------------------------------------------------------ */
/* Batched (per-level) task bodies                                          */
/* ------------------------------------------------------------------------ */

/* One leaf of a batched leaf solve (device-resident array of these). */
typedef struct {
  double *D;  /* n x n, ldd */
  double *X;  /* n x nrhs, ldx */
  int *ipiv;  /* n ints */
  int *perm;  /* n ints: final row order (row i of P^T D is row perm[i]) */
  long long ldd;
  long long ldx;
  int n;
  int nrhs;
} hodlr_leaf_desc;

/* All leaves of a level (or of many systems) in one launch pair.  `descs` is
 * a device array of `count` descriptors, max_n the largest n among them;
 * info (device, `count` ints) receives each leaf's INFO.  Asynchronous.
 * Batched form of solver_tasks.cc:424-450 over the leaves that
 * fast_solver.cc:197-201 visits. */
int hodlr_leaf_solve_batched(int count, const hodlr_leaf_desc *descs,
                             int max_n, int max_nrhs, int *info,
                             hodlr_stream_t stream);

/* FP32 GEMM engine of the mixed-precision path (no reference counterpart):
 * C = beta * C + alpha * op(A) * B, column-major, op(A) = A (transa = 0,
 * A m x k) or A^T (transa = 1, A k x m), B k x n.  engine 0: FP32 FMA pipe;
 * engine 1: tcgen05 tensor cores, split-BF16 (hi*hi + hi*lo + lo*hi, FP32
 * accumulate; relative error ~2^-16 of |A||B|).  Synchronous. */
int hodlr_gemm_f32(int transa, int m, int n, int k, float alpha, const float *A,
                   int lda, const float *B, int ldb, float beta, float *C,
                   int ldc, int engine, hodlr_stream_t stream);

/* Test hook of the timeout path of the tensor-core engine (no reference
 * counterpart: the reference has no device waits).  Every bounded mbarrier
 * wait of the engine gives up after `polls` tries (<= 0 restores the default,
 * 2^22, a few seconds), and with skip_one_commit != 0 the next engine launch
 * leaves out the completion signal of one tile, so one of its waits runs out:
 * the kernel then raises the device error flag, waits (bounded) for its own
 * tensor-core work, frees its tensor memory and returns.  Every call that
 * synchronizes (hodlr_factor, hodlr_solve_fused with sync, the refined and
 * batched solves, hodlr_gemm_f32) reads and clears the flag and returns
 * HODLR_ERR_TIMEOUT when it was raised; calls that only enqueue work leave it
 * for the next synchronizing call.  Synchronizes the device. */
int hodlr_debug_tc_wait_hook(long long polls, int skip_one_commit);

/* The same for the grid barriers of the persistent sweep kernel (the level
 * walk of the refinement sweeps): every barrier wait gives up after `polls`
 * tries (<= 0: the default, 2^22), and with skip_one_arrival != 0 one CTA of
 * the next sweep launch leaves before its first arrival, so the other CTAs'
 * waits run out; they raise the device flag and leave.  The refined and
 * batched solves then return HODLR_ERR_TIMEOUT.  Synchronizes the device. */
int hodlr_debug_sweep_barrier_hook(long long polls, int skip_one_arrival);

/* ------------------------------------------------------------------------ */
/* Handle API: the solver that walks the tree (FastSolver + HodlrMatrix)     */
/* ------------------------------------------------------------------------ */

typedef struct hodlr_system_s *hodlr_system;

/* Host-only: build the tree hodlr_create would build and write its node
 * records (10 ints each, BFS order, see hodlr_tree_nodes) into `out`.
 * Returns the node count, or < 0 (bad argument / cap too small = -6).
 * Restates src/htree/hodlr_matrix.cc:138-169 and 354-386; needs no GPU. */
int hodlr_build_tree(int N, int nrhs, int rank, int threshold, int *out,
                     int cap);

/* Build the HODLR tree of one N x N system with nrhs right-hand sides, rank r
 * at every level and dense leaves of at most `threshold` rows (N/2, N - N/2
 * split; leafSize = 1).  Mirrors HodlrMatrix::HodlrMatrix + create_tree:
 * src/htree/hodlr_matrix.cc:22-33, 44-82, 138-169, 354-472.  Allocates the
 * system's device arrays on the current device. */
int hodlr_create(hodlr_system *sys, int N, int nrhs, int rank, int threshold);
int hodlr_destroy(hodlr_system sys);

/* Tree shape: node count, max depth, leaf count, total columns C = m + r*L,
 * largest leaf.  Any output pointer may be NULL. */
int hodlr_tree_info(hodlr_system sys, int *nnodes, int *max_depth,
                    int *nleaves, int *ncols, int *max_leaf);
/* Node records, 10 ints each in BFS order (nrow, ncol, row_beg, col_beg,
 * lchild, rchild, parent, depth, vncol, is_leaf), into host array `out`. */
int hodlr_tree_nodes(hodlr_system sys, int *out, int cap);

/* Matrix data in the global layout: D (N x max_leaf, leaf blocks stacked),
 * U and V (N x (C - m), column block of node c at c.col_beg - m), B (N x m).
 * `host` != 0: the pointers are host memory (copied synchronously on
 * `stream`); 0: device memory (copied device-to-device).  Any may be NULL to
 * leave that part unchanged. */
int hodlr_set_matrix(hodlr_system sys, const double *D, long long ldd,
                     const double *U, long long ldu, const double *V,
                     long long ldv, int host, hodlr_stream_t stream);
int hodlr_set_rhs(hodlr_system sys, const double *B, long long ldb, int host,
                  hodlr_stream_t stream);
/* Copy the system's D, U, V, B out (same layouts; NULL skips a part). */
int hodlr_get_matrix(hodlr_system sys, double *D, long long ldd, double *U,
                     long long ldu, double *V, long long ldv, double *B,
                     long long ldb, int host, hodlr_stream_t stream);

/* Device-side generators.  hodlr_init_circulant: the reference's test matrix
 * A = diag*I + U U^T, U(i, j) = (i + j) mod r (init_matrix_tasks.cc:176-219,
 * hodlr_matrix.cc:528-567); hodlr_init_rhs_drand48: drand48_r(seed) stream
 * reseeded per leaf, row-major fill (init_matrix_tasks.cc:43-77);
 * hodlr_init_gaussian: leaf blocks G/sqrt(n) + 2I, U,V iid
 * N(0,1)/sqrt(r n_child) rescaled so every off-diagonal block has spectral
 * norm `offdiag_norm`, b iid N(0,1) (Philox4x32-10 counter RNG). */
int hodlr_init_circulant(hodlr_system sys, double diag, hodlr_stream_t stream);
int hodlr_init_rhs_drand48(hodlr_system sys, long seed, hodlr_stream_t stream);
int hodlr_init_gaussian(hodlr_system sys, unsigned long long seed,
                        double offdiag_norm, hodlr_stream_t stream);

/* Fused FP64 factor+solve of the current RHS, the reference's bfs_solve
 * (src/solver/fast_solver.cc:56-72, 136-255): leaf solves on [b | U], then per
 * level 4 reduces -> node LU -> 2 broadcasts.  The solution is left in the
 * system (hodlr_get_solution).  Asynchronous unless `sync`. */
int hodlr_solve_fused(hodlr_system sys, int schur2, int sync,
                      hodlr_stream_t stream);

/* Factor/solve split (no reference counterpart: the reference always fuses).
 * hodlr_factor keeps the leaf LU (with the inverses of its diagonal blocks),
 * the transformed U blocks and every node's solve matrix M
 * ([eta0; eta1] = M [V0Td0; V1Td1]) in `precision`; hodlr_solve applies
 * them to the current RHS. */
int hodlr_factor(hodlr_system sys, int precision, hodlr_stream_t stream);
int hodlr_solve(hodlr_system sys, hodlr_stream_t stream);

/* Mixed-precision solve with FP64 iterative refinement until
 * max_j ||b_j - A x_j|| / ||b_j|| <= tol (or maxiter sweeps).  One call =
 * factor (FP32, carrying b) + refinement sweeps; iters and relres (host
 * pointers, may be NULL) report the result.  Returns HODLR_ERR_NOCONV if
 * the tolerance was not met. */
int hodlr_solve_refined(hodlr_system sys, int precision, double tol,
                        int maxiter, int *iters, double *relres,
                        hodlr_stream_t stream);

/* The same refined solve from host memory to host memory: copies D, U, V
 * and B in (as hodlr_set_matrix / hodlr_set_rhs with host = 1), solves, and
 * copies the solution out to X (N x nrhs, ldx), all on `stream`; returns
 * when X holds the result and no copy still reads the caller's buffers.
 * With PREC_MIXED, V's copy (first read by the tree levels) runs on a
 * second stream under the leaf factorization; from pinned host memory the
 * copy and the factorization overlap.  U and V may be NULL only for a
 * system without off-diagonal blocks.  Return values as
 * hodlr_solve_refined; negative: the position of an invalid argument. */
int hodlr_solve_refined_host(hodlr_system sys, const double *D, long long ldd,
                             const double *U, long long ldu, const double *V,
                             long long ldv, const double *B, long long ldb,
                             double *X, long long ldx, int precision, double tol,
                             int maxiter, int *iters, double *relres,
                             hodlr_stream_t stream);

/* y = A x (FP64 HODLR matvec) for x, y device arrays N x ncols (ldx, ldy),
 * ncols <= nrhs. */
int hodlr_matvec(hodlr_system sys, const double *x, long long ldx, double *y,
                 long long ldy, int ncols, hodlr_stream_t stream);

/* max_j ||b_j - A x_j||_2 / ||b_j||_2 of the current solution (host result). */
int hodlr_relres(hodlr_system sys, double *relres, hodlr_stream_t stream);

/* Copy the solution (N x m) out: host != 0 -> host memory. */
int hodlr_get_solution(hodlr_system sys, double *X, long long ldx, int host,
                       hodlr_stream_t stream);

/* Task granularity of the reference (HodlrMatrix's leafSize argument,
 * src/htree/hodlr_matrix.cc:22-33, 317-337): a Legion leaf is a topmost node
 * whose subtree holds at most leaf_size real leaves (default 1: the real
 * leaves).  It decides (a) the drand48 right-hand side, one stream reseeded
 * per Legion leaf (init_rhs, hodlr_matrix.cc:175-209); (b) the blocks of the
 * text files (one seed line per Legion leaf, hodlr_matrix.cc:569-605); (c) the
 * node form of the FP64 fused solve: internal nodes inside a Legion leaf use
 * the 2r x 2r form of serial_leaf_solve's internal branch
 * (solver_tasks.cc:452-549), the others LUSolveTask's r x r form.  leaf_size
 * > 1 needs 2r <= 144 (HODLR_ERR_UNSUPPORTED otherwise).  Discards the FP64
 * factorization. */
int hodlr_set_leaf_size(hodlr_system sys, int leaf_size);
/* Number of Legion leaves (HodlrMatrix::get_num_leaf); the reference's
 * counter also counts the nodes below a Legion leaf when leafSize > 1, this
 * returns the data blocks (tasks) only. */
int hodlr_get_num_leaf(hodlr_system sys);
/* Node ids (BFS numbering, as hodlr_tree_nodes) of the Legion leaves, left to
 * right, into ids (cap entries; NULL: count only).  Returns the count. */
int hodlr_legion_leaves(hodlr_system sys, int *ids, int cap);

/* ---- The reference's text format (src/legion_matrix/save_region_task.cc:
 * 37-67): every row of a block on its own line, each value printed with 20
 * significant digits ("%.20g") and followed by a tab, blocks appended to the
 * file, an optional seed line in front of a block.  Host memory. */
/* Append rows 0..nrow-1, columns col_beg..col_beg+ncol-1 of the column-major
 * X (ldx) to `filename`, after a seed line if print_seed (save_data). */
int hodlr_text_write(const char *filename, const double *X, long long ldx,
                     int nrow, int col_beg, int ncol, long seed, int print_seed);
/* Read nrow x ncol values row by row (whitespace separated, as the dense check
 * reads the solution file, src/solver/direct_solve.cc:201-213) into X (ldx).
 * With nblocks > 0 the file holds nblocks blocks of block_rows[b] rows (sum =
 * nrow), each after a seed line; the seeds go to `seeds` (may be NULL).
 * Returns 0, an argument error or HODLR_ERR_IO (missing file, short or
 * malformed data). */
int hodlr_text_read(const char *filename, double *X, long long ldx, int nrow,
                    int ncol, int nblocks, const int *block_rows, long *seeds);
/* HodlrMatrix::save_rhs / save_solution (hodlr_matrix.cc:569-605): remove the
 * file, then write every Legion leaf's rows of b (with `seed` in front of each
 * block) or of the solution.  hodlr_load_rhs reads a file save_rhs wrote
 * (for the system's Legion leaves) into b; *seed (may be NULL) receives the
 * first block's seed.  Synchronous. */
int hodlr_save_rhs(hodlr_system sys, const char *filename, long seed);
int hodlr_save_solution(hodlr_system sys, const char *filename);
int hodlr_load_rhs(hodlr_system sys, const char *filename, long *seed);

/* Per-phase device time.  While profiling is on (off by default), every
 * launch group is bracketed by CUDA events; hodlr_phase_times synchronizes
 * and returns, per phase, the accumulated milliseconds and the number of
 * launches since the last reset (ms / launches: arrays of HODLR_PHASES,
 * either may be NULL).  Phases: 0 getrf (the forward blocked leaf
 * factorization, all of 8-10), 1 getrs (backward leaf solve / leaf apply),
 * 2 reduce, 3 node factor, 4 node apply, 5 broadcast, 6 matvec, 7 precision
 * conversion, 8 leaf panels (panel LU + row interchanges), 9 leaf trailing
 * updates (A22 -= L21 U12), 10 leaf panel solves (U12 = L11^{-1} A12),
 * 11 the persistent level walk of a refinement sweep (reduce, slot sums,
 * node apply and broadcast of every level in one launch; 2, 4 and 5 then
 * stay 0 for the sweeps). */
#define HODLR_PHASES 12
int hodlr_set_profiling(hodlr_system sys, int on);
int hodlr_phase_times(hodlr_system sys, double *ms, long long *launches,
                      int reset);

/* ---- Batches of independent systems (no reference counterpart: the
 * reference solves one system per Legion run).  A batch merges the level
 * schedules of `count` systems of any size, rank, leaf size and RHS count
 * (created by hodlr_create, matrices and RHS loaded): every leaf panel of
 * every system runs in one launch, then level j (deepest first) of every
 * system in one launch per phase, and the residual matvecs of all systems
 * in one launch.  1 <= count <= 16384.  The systems must outlive the batch
 * and must not be destroyed, re-created or put into another batch while it
 * exists; loading new matrices or RHS into them is fine (a solve reads their
 * buffers). */
typedef struct hodlr_batch_s *hodlr_batch;
int hodlr_batch_create(hodlr_batch *out, const hodlr_system *systems, int count);
int hodlr_batch_destroy(hodlr_batch batch);

/* Mixed-precision solve of every system of the batch with FP64 iterative
 * refinement until each system's max_j ||b_j - A x_j|| / ||b_j|| <= tol (or
 * maxiter sweeps, all systems sweeping together).  iters, relres_max (host
 * scalars), relres (host array of `count`, each system's residual) and
 * failed (the system whose factorization reported a nonzero INFO, -1 if
 * none) may be NULL.  Returns 0, the failing system's INFO (leaf INFO, or
 * 100000 + node INFO, as hodlr_solve_fused), or HODLR_ERR_NOCONV.  On a
 * non-default stream the factor pass and the sweep are captured as CUDA
 * graphs on first use and replayed afterwards.  Each system's solution is
 * read with hodlr_get_solution; each system is left factored (hodlr_solve
 * applies the same factors to a new RHS). */
int hodlr_batch_solve_refined(hodlr_batch batch, double tol, int maxiter, int *iters,
                              double *relres_max, double *relres, int *failed,
                              hodlr_stream_t stream);

/* Per-phase device time of the batch's merged launches (as hodlr_phase_times). */
int hodlr_batch_set_profiling(hodlr_batch batch, int on);
int hodlr_batch_phase_times(hodlr_batch batch, double *ms, long long *launches, int reset);

/* ---- Launch schedule and autotuner (no reference counterpart: the
 * reference's task granularity is fixed by its tree).  A schedule fixes how
 * the solve is cut into launches:
 *   leaf_nb      FP32 leaf panel width: 0 = by the largest leaf (64 up to 512
 *                rows, else 32), or 32, or 64 (leaves of <= 512 rows only);
 *   leaf_ob32    FP32 leaf outer block width (a multiple of the panel width,
 *                rounded down; 0 = one-level blocking; blocks of at most 128
 *                columns solve their block rows with the inverses of the
 *                block's triangles, wider ones panel by panel);
 *   leaf_ob64    the same for the FP64 path (panel width 32, or 16 above 512
 *                rows);
 *   reduce_rows  rows per split-K slot of the reduce V^T [d | u] (16..65536,
 *                a multiple of 16; at most 64 slots per child);
 *   bcast_rows   rows per item of the broadcast d -= u eta (16..65536, a
 *                multiple of 16).
 * Defaults: {0, 128, 0, 512, 512}.  Setting a schedule discards the system's
 * factors (factor again before hodlr_solve); results are identical up to
 * floating-point summation order. */
typedef struct {
  int leaf_nb;
  int leaf_ob32;
  int leaf_ob64;
  int reduce_rows;
  int bcast_rows;
} hodlr_schedule;

typedef struct {
  hodlr_schedule schedule;
  double ms; /* mean time of one timed solve; < 0: the schedule failed */
} hodlr_tune_trial;

int hodlr_get_schedule(hodlr_system sys, hodlr_schedule *out);
int hodlr_set_schedule(hodlr_system sys, const hodlr_schedule *in);

/* Autotuner: times candidate schedules on the system's current matrix and
 * RHS with CUDA events (one untimed solve, then `reps` timed ones, each a
 * full solve: precision MIXED = the refined solve to `tol`, FP64 = the fused
 * FP64 solve), searching one field at a time (outer block, panel width,
 * reduce rows, broadcast rows) from the current schedule, and installs the
 * fastest.  Runs on a private stream after a device synchronization.  The
 * system is left with the best schedule; its solution is the last trial's
 * (solve again for the factors of the chosen schedule).  best, best_ms, log
 * (log_cap entries) and n_log (trials run, may exceed log_cap) may be NULL. */
int hodlr_autotune(hodlr_system sys, int precision, double tol, int reps,
                   hodlr_schedule *best, double *best_ms, hodlr_tune_trial *log,
                   int log_cap, int *n_log);
/* The same for a batch (mixed precision): one schedule for all its systems,
 * timed as the batched solve; the batch's merged plans are rebuilt. */
int hodlr_batch_autotune(hodlr_batch batch, double tol, int reps, hodlr_schedule *best,
                         double *best_ms, hodlr_tune_trial *log, int log_cap,
                         int *n_log);

/* Number of kernels this library launched on this thread since the last
 * reset (every launch from a hodlr_* call is counted). */
long long hodlr_launch_count(void);
void hodlr_reset_launch_count(void);

/* Human-readable text of a status code. */
const char *hodlr_status_string(int status);

#ifdef __cplusplus
}
#endif

#endif /* HODLR_GPU_H */
