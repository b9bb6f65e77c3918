// htree.cpp -- HODLR tree construction (see htree.h).
#include "htree.h"

#include <algorithm>
#include <functional>

namespace hodlr {

int build_tree(int N, int nrhs, int rank, int threshold, Tree &t) {
  if (N <= 0) return -1;
  if (nrhs <= 0) return -2;
  if (rank <= 0) return -3;
  if (threshold <= 0) return -4;
  t = Tree();
  t.N = N; t.nrhs = nrhs; t.rank = rank; t.threshold = threshold;
  Node root{N, nrhs, 0, 0, -1, -1, -1, 0, 0, 1};
  t.nodes.push_back(root);
  for (size_t i = 0; i < t.nodes.size(); ++i) {
    Node p = t.nodes[i];
    if (p.nrow > threshold) {
      const int li = (int)t.nodes.size(), ri = li + 1;
      Node l{p.nrow / 2, rank, p.row_beg, p.col_beg + p.ncol, -1, -1, (int)i, p.depth + 1, 0, 1};
      Node r{p.nrow - p.nrow / 2, rank, p.row_beg + p.nrow / 2, p.col_beg + p.ncol, -1, -1,
             (int)i, p.depth + 1, 0, 1};
      l.vncol = r.ncol;  // hodlr_matrix.cc:359-360
      r.vncol = l.ncol;
      t.nodes.push_back(l);
      t.nodes.push_back(r);
      t.nodes[i].lchild = li;
      t.nodes[i].rchild = ri;
      t.nodes[i].is_leaf = 0;
    } else if (!(p.nrow > rank)) {
      return -4;
    }
  }
  t.max_depth = 0;
  for (const Node &n : t.nodes) t.max_depth = std::max(t.max_depth, n.depth);
  t.internal_at_depth.assign(t.max_depth + 1, {});
  for (int i = 0; i < (int)t.nodes.size(); ++i)
    if (!t.nodes[i].is_leaf) t.internal_at_depth[t.nodes[i].depth].push_back(i);
  // leaves left to right (in-order of the split)
  std::function<void(int)> walk = [&](int i) {
    const Node &n = t.nodes[i];
    if (n.is_leaf) { t.leaves.push_back(i); return; }
    walk(n.lchild);
    walk(n.rchild);
  };
  walk(0);
  for (int i : t.leaves) {
    const Node &n = t.nodes[i];
    t.ncols = std::max(t.ncols, n.col_beg + n.ncol);
    t.max_leaf = std::max(t.max_leaf, n.nrow);
  }
  // real leaves per subtree: children come after their parent in BFS order
  t.nreal.assign(t.nodes.size(), 0);
  for (int i = (int)t.nodes.size() - 1; i >= 0; --i) {
    const Node &n = t.nodes[i];
    t.nreal[i] = n.is_leaf ? 1 : t.nreal[n.lchild] + t.nreal[n.rchild];
  }
  return 0;
}

std::vector<int> legion_leaves(const Tree &t, int leaf_size) {
  std::vector<int> out;
  std::function<void(int)> walk = [&](int i) {
    const Node &n = t.nodes[i];
    if (t.nreal[i] <= leaf_size) { out.push_back(i); return; }
    walk(n.lchild);
    walk(n.rchild);
  };
  if (!t.nodes.empty()) walk(0);
  return out;
}

}  // namespace hodlr
