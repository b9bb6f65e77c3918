// textio.cu -- the reference's text format for right-hand sides and
// solutions (host code, no device work except the copies of the handle-level
// calls).
//
// Writer: save_data of src/legion_matrix/save_region_task.cc:37-67 -- the
// file is opened for appending; an optional seed line; then one line per
// row, every value printed with 20 significant digits (operator<< with
// setprecision(20), i.e. "%.20g") and followed by a tab.
// Writers per system: HodlrMatrix::save_rhs / save_solution and
// save_HodlrMatrix (src/htree/hodlr_matrix.cc:569-605) -- the old file is
// removed, then every Legion leaf, left to right, appends its rows (the RHS
// file with the seed line in front of each Legion leaf's block).
// Reader: the whitespace-separated, row-by-row read of the dense check
// (src/solver/direct_solve.cc:201-213), extended to skip (and return) the
// seed line in front of each block of a file written with seeds.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

#include "common.cuh"
#include "solver.h"

using namespace hodlr;

static System &system_of(hodlr_system_s *h) { return h->sys; }

namespace {

// Appends rows [0, nrow) x columns [col_beg, col_beg + ncol) of the
// column-major host array X (ldx) to `f`, with an optional seed line.
int write_block(FILE *f, const double *X, long long ldx, int nrow, int col_beg, int ncol,
                long seed, bool print_seed) {
  if (print_seed && std::fprintf(f, "%ld\n", seed) < 0) return HODLR_ERR_IO;
  char buf[64];
  for (int i = 0; i < nrow; ++i) {
    for (int j = 0; j < ncol; ++j) {
      std::snprintf(buf, sizeof(buf), "%.20g\t", X[i + (long long)(col_beg + j) * ldx]);
      if (std::fputs(buf, f) < 0) return HODLR_ERR_IO;
    }
    if (std::fputc('\n', f) == EOF) return HODLR_ERR_IO;
  }
  return 0;
}

// Reads one whitespace-separated token as a double ("inf", "nan" included).
bool read_value(FILE *f, double *v) {
  char tok[128];
  if (std::fscanf(f, "%127s", tok) != 1) return false;
  char *end = nullptr;
  errno = 0;
  *v = std::strtod(tok, &end);
  return end != tok && *end == '\0';
}

bool read_seed(FILE *f, long *seed) {
  char tok[64];
  if (std::fscanf(f, "%63s", tok) != 1) return false;
  char *end = nullptr;
  const long v = std::strtol(tok, &end, 10);
  if (end == tok || *end != '\0') return false;
  if (seed) *seed = v;
  return true;
}

}  // namespace

extern "C" {

int hodlr_text_write(const char *filename, const double *X, long long ldx, int nrow,
                     int col_beg, int ncol, long seed, int print_seed) {
  if (!filename) return -1;
  if (!X && nrow > 0 && ncol > 0) return -2;
  if (nrow < 0) return -4;
  if (ldx < (nrow > 1 ? nrow : 1)) return -3;
  if (col_beg < 0) return -5;
  if (ncol < 0) return -6;
  FILE *f = std::fopen(filename, "a");
  if (!f) return HODLR_ERR_IO;
  int rc = write_block(f, X, ldx, nrow, col_beg, ncol, seed, print_seed != 0);
  if (std::fclose(f) != 0 && rc == 0) rc = HODLR_ERR_IO;
  return rc;
}

int hodlr_text_read(const char *filename, double *X, long long ldx, int nrow, int ncol,
                    int nblocks, const int *block_rows, long *seeds) {
  if (!filename) return -1;
  if (!X && nrow > 0 && ncol > 0) return -2;
  if (nrow < 0) return -4;
  if (ldx < (nrow > 1 ? nrow : 1)) return -3;
  if (ncol < 0) return -5;
  if (nblocks < 0 || (nblocks > 0 && !block_rows)) return -6;
  if (nblocks > 0) {
    long long tot = 0;
    for (int b = 0; b < nblocks; ++b) {
      if (block_rows[b] < 0) return -7;
      tot += block_rows[b];
    }
    if (tot != nrow) return -7;
  }
  FILE *f = std::fopen(filename, "r");
  if (!f) return HODLR_ERR_IO;
  int rc = 0;
  int row = 0;
  const int nb = nblocks > 0 ? nblocks : 1;
  for (int b = 0; b < nb && rc == 0; ++b) {
    const int rows = nblocks > 0 ? block_rows[b] : nrow;
    if (nblocks > 0 && !read_seed(f, seeds ? seeds + b : nullptr)) {
      rc = HODLR_ERR_IO;
      break;
    }
    for (int i = 0; i < rows && rc == 0; ++i, ++row)
      for (int j = 0; j < ncol; ++j)
        if (!read_value(f, X + row + (long long)j * ldx)) {
          rc = HODLR_ERR_IO;
          break;
        }
  }
  std::fclose(f);
  return rc;
}

// The system's right-hand side (with_seed: save_rhs, a seed line per Legion
// leaf) or solution (save_solution) in the reference's format.
static int save_system(hodlr_system_s *h, const char *filename, bool rhs, long seed) {
  if (!h) return -1;
  if (!filename) return -2;
  System &S = system_of(h);
  try {
    std::vector<double> X((size_t)S.N * S.m);
    HODLR_CUDA_TRY(cudaMemcpy(X.data(), rhs ? S.B.p : S.Xsol.p, sizeof(double) * X.size(),
                              cudaMemcpyDeviceToHost));
    std::remove(filename);  // the reference removes the old file first
    FILE *f = std::fopen(filename, "a");
    if (!f) return HODLR_ERR_IO;
    int rc = 0;
    for (int id : legion_leaves(S.tree, S.leaf_size)) {
      const Node &n = S.tree.nodes[id];
      rc = write_block(f, X.data() + n.row_beg, S.N, n.nrow, 0, S.m, seed, rhs);
      if (rc) break;
    }
    if (std::fclose(f) != 0 && rc == 0) rc = HODLR_ERR_IO;
    return rc;
  } catch (const CudaError &) {
    return HODLR_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    return HODLR_ERR_NOMEM;
  }
}

int hodlr_save_rhs(hodlr_system h, const char *filename, long seed) {
  return save_system(h, filename, true, seed);
}

int hodlr_save_solution(hodlr_system h, const char *filename) {
  return save_system(h, filename, false, 0);
}

int hodlr_load_rhs(hodlr_system h, const char *filename, long *seed) {
  if (!h) return -1;
  if (!filename) return -2;
  System &S = system_of(h);
  try {
    const std::vector<int> ll = legion_leaves(S.tree, S.leaf_size);
    std::vector<int> rows;
    for (int id : ll) rows.push_back(S.tree.nodes[id].nrow);
    std::vector<long> seeds(ll.size(), 0);
    std::vector<double> B((size_t)S.N * S.m);
    int rc = hodlr_text_read(filename, B.data(), S.N, S.N, S.m, (int)rows.size(), rows.data(),
                             seeds.data());
    if (rc) return rc;
    if (seed) *seed = seeds.empty() ? 0 : seeds[0];
    HODLR_CUDA_TRY(cudaMemcpy(S.B.p, B.data(), sizeof(double) * B.size(),
                              cudaMemcpyHostToDevice));
    return 0;
  } catch (const CudaError &) {
    return HODLR_ERR_CUDA;
  } catch (const std::bad_alloc &) {
    return HODLR_ERR_NOMEM;
  }
}

}  // extern "C"
