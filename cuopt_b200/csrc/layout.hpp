// Host-side construction of the device matrix layout used by every SpMV-fused kernel.
//
// The reference keeps A and its transpose in CSR and hands both to cuSPARSE
// (cpp/src/pdlp/cusparse_view.cu:271-925, transpose built in
// cpp/src/mip_heuristics/problem/problem.cu:367-470).  Here the LP is first relabelled
// internally — constraints and variables are re-ordered, which leaves the LP unchanged — so that
//   * rows longer than `long_row_threshold` come first and are processed warp-per-row (CSR);
//   * the remaining rows are sorted by length (descending) inside windows of `sort_window` rows and
//     stored as sliced ELL with 32-row slices, column-major inside a slice, so that lane t of a
//     warp reads element k of row t at address base + 32k + t: every matrix load of a warp is one
//     contiguous 128/256-byte segment, and every per-row vector access of the fused epilogue is
//     contiguous too (vectors live in the same internal order).
// Both A (rows = constraints) and A^T (rows = variables) get this layout; the index arrays refer to
// internal ids of the other dimension.
#pragma once

#include <cstdint>
#include <vector>

namespace cuopt_b200 {

struct sell_host {
  int rows   = 0;  // internal rows
  int cols   = 0;
  int n_long = 0;  // rows [0, n_long) are long rows (CSR, warp per row)
  int n_slices = 0;
  std::vector<int64_t> long_off;   // n_long + 1, absolute element offsets
  std::vector<int64_t> slice_off;  // n_slices + 1, absolute element offsets (multiples of 32 apart)
  std::vector<int> idx;            // internal column ids
  std::vector<double> val;         // unscaled values (padding: 0)
  std::vector<int64_t> src;        // position of each stored element in the user's CSR (-1: pad)
  int64_t stored() const { return (int64_t)idx.size(); }
};

struct lp_layout {
  int m = 0, n = 0;
  int64_t nnz = 0;
  std::vector<int> row_new2old, row_old2new;  // constraint permutation
  std::vector<int> col_new2old, col_old2new;  // variable permutation
  sell_host a;   // internal A  (m x n)
  sell_host at;  // internal A^T (n x m)
};

struct layout_options {
  int long_row_threshold = 96;   // rows with more non-zeros are handled warp-per-row
  int sort_window        = 1 << 15;
};

// Builds the internal layout from the user's CSR (row offsets m+1, column indices, values).
lp_layout build_layout(int m, int n, const int* row_off, const int* col_idx, const double* val,
                       const layout_options& opt = layout_options{});

}  // namespace cuopt_b200
