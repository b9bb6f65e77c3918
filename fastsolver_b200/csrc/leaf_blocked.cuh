// leaf_blocked.cuh -- batched blocked factorization of the leaves on [D | X].
#pragma once
#include "common.cuh"

namespace hodlr {

// Panel width: the panel (n x NB) lives in shared memory, so it narrows for
// leaves above 512 rows (the library accepts leaves of up to 1024 rows).
template <typename T>
inline int leaf_nb(int max_n) {
  if (sizeof(T) == 8) return max_n <= 512 ? 32 : 16;
  return max_n <= 512 ? 64 : 32;
}

// One leaf of a batched factorization.
template <typename T>
struct LeafFactorTask {
  T *D;            // n x n, ldd: LU factors on output (LAPACK layout)
  T *X;            // n x ncols, ldx: D^{-1} X on output
  int *ipiv;       // n: LAPACK pivots
  int *perm;       // n: final row order
  T *Linv;         // npanels x NB x NB: inverses of the unit-lower diagonal blocks
  T *Uinv;         // npanels x NB x NB: inverses of the upper diagonal blocks
  int *swapflag;   // npanels: panel had row interchanges
  T *LinvB;        // nblocks x OB x OB: inverses of the unit-lower outer diagonal blocks
  T *UinvB;        // nblocks x OB x OB: inverses of the upper outer diagonal blocks
  long long ldd;
  long long ldx;
  int n;
  int ncols;
  int info_slot;
  int pad;
};

// X <- (P L U)^{-1} X on every leaf with the blocked factors of a previous
// factorization (LU in D, final row order in perm, per-panel Linv / Uinv);
// X has task.ncols columns.  One CTA per (leaf, column chunk).
template <typename T>
void launch_leaf_apply(const LeafFactorTask<T> *tasks, int count, int max_n, int max_cols, int nb,
                       cudaStream_t s);

template <typename T>
void launch_leaf_init(const LeafFactorTask<T> *tasks, int count, int *info, cudaStream_t s);
// Inverse of outer block J's unit-lower diagonal block (ob x ob, ob a
// multiple of nb and at most 128) from the block's factored panels and their
// nb x nb inverses, into task.LinvB + J ob^2 (column-major, ld ob, zero
// outside the leaf); with `upper`, the inverses of the upper diagonal blocks
// of all `nblocks` blocks into task.UinvB (J unused).
template <typename T>
void launch_leaf_block_inverse(const LeafFactorTask<T> *tasks, int count, int nb, int ob, int J,
                               bool upper, int nblocks, cudaStream_t s);
template <typename T>
void launch_leaf_panel(const LeafFactorTask<T> *tasks, int count, int max_n, int nb, int k0,
                       int panel, int *info, cudaStream_t s);
// Row interchanges of panels [p0, p0 + np) on the D columns [a0, a1) and
// [b0, b1) (clamped to each leaf's n) and, with with_x, on X.  max_cols:
// an upper bound of the columns touched in any leaf (e.g. largest n + ncols).
template <typename T>
void launch_leaf_laswp(const LeafFactorTask<T> *tasks, int count, int max_cols, int nb, int p0,
                       int np, int a0, int a1, int b0, int b1, bool with_x, cudaStream_t s);

}  // namespace hodlr
