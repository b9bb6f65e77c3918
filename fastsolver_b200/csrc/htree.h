// htree.h -- HODLR tree and global data layout (host side).
//
// Legion-free restatement of fastSolver's tree construction
// (src/htree/hodlr_matrix.cc:44-82 create_tree, 138-169
// create_balanced_tree, 354-386 create_Vtree; src/htree/node.cc:4-16 Node)
// for leafSize == 1 (every real leaf is its own task):
//   * the root holds the nrhs right-hand-side columns (col_beg 0);
//   * a node with nrow > threshold splits into nrow/2 and nrow - nrow/2 rows;
//     each child carries `rank` columns starting at parent.col_beg +
//     parent.ncol, so a leaf at depth L owns columns [0, nrhs + rank*L) of
//     X = [b | U_1 .. U_L];
//   * the V tree has the same rows with the children's ranks swapped
//     (vncol of a child = ncol of its sibling).
// Nodes are stored in BFS order, the order FastSolver::solve_bfs builds
// (src/solver/fast_solver.cc:136-171), so reverse index order is its visit
// order.
//
// Global layout (column-major, device):
//   X  N x C   [b | U]: U block of node c in columns [c.col_beg, c.col_beg+c.ncol)
//   V  N x (C - nrhs): V factor of node c (rows of c) in columns
//              [c.col_beg - nrhs, c.col_beg - nrhs + c.vncol)
//   D  N x max_leaf: leaf diagonal blocks stacked vertically (the K region of
//              hodlr_matrix.cc:431-445 with one Legion leaf per real leaf)
#pragma once

#include <vector>

namespace hodlr {

struct Node {
  int nrow, ncol, row_beg, col_beg;
  int lchild, rchild, parent, depth, vncol, is_leaf;
};
static_assert(sizeof(Node) == 10 * sizeof(int), "Node is 10 ints");

struct Tree {
  int N = 0, nrhs = 0, rank = 0, threshold = 0;
  std::vector<Node> nodes;  // BFS order, nodes[0] = root
  int max_depth = 0;
  int ncols = 0;     // C = max over leaves of col_beg + ncol
  int max_leaf = 0;  // largest leaf row count
  std::vector<int> leaves;                          // leaf ids, left to right
  std::vector<std::vector<int>> internal_at_depth;  // internal node ids by depth
  std::vector<int> nreal;                           // real leaves in each node's subtree
  int vcols() const { return ncols - nrhs; }
};

// Returns 0 on success, < 0 on a bad argument (-1 N, -2 nrhs, -3 rank,
// -4 threshold; -4 also when a leaf would not exceed the rank, which the
// reference asserts at hodlr_matrix.cc:167).
int build_tree(int N, int nrhs, int rank, int threshold, Tree &t);

// Legion leaves at granularity `leaf_size` (>= 1), left to right: the
// topmost nodes whose subtree holds at most leaf_size real leaves
// (mark_legion_leaf, hodlr_matrix.cc:317-337).  With leaf_size == 1 they are
// the real leaves.  A Legion leaf is one task of the reference: its
// right-hand side is generated from one drand48 stream (init_matrix_tasks.cc:
// 43-77), it is written as one block of the text output
// (save_region_task.cc:37-67), and every internal node inside it is solved
// with the 2r x 2r form of the leaf-internal branch (solver_tasks.cc:452-549)
// instead of LUSolveTask's r x r form.
std::vector<int> legion_leaves(const Tree &t, int leaf_size);

// True if internal node `id` lies inside a Legion leaf (is one or is below one).
inline bool inside_legion_leaf(const Tree &t, int id, int leaf_size) {
  return t.nreal[id] <= leaf_size;
}

}  // namespace hodlr
