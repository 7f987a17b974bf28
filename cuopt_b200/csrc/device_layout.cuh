// On-device construction of the PDLP matrix layout (counterpart of the reference's problem_t
// transpose build, cpp/src/mip_heuristics/problem/problem.cu:367-470, and of the cuSPARSE
// descriptors of cusparse_view.cu:271-925).
//
// From the user's CSR (device arrays) it builds, entirely on the GPU and deterministically:
//   * an internal relabelling of constraints and variables: rows longer than `long_threshold` first
//     (by length, descending), then the remaining rows sorted by length (descending, stable) inside
//     windows of `window` rows — the LP is unchanged, only its numbering;
//   * A and A^T in that numbering, each as long-row CSR + sliced ELL with 32-row slices stored
//     column-major inside a slice (lane t reads element k of row t at base + 32k + t);
//   * for every stored element its position in the user's CSR (-1 for padding), used to map
//     gradients with respect to A back to the user's order.
// Sorting and scans use CUB's stable radix sort / scan (one-off setup); everything else is plain
// kernels in device_layout.cu.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace cuopt_b200 {

template <typename T>
struct dev_sell;

struct dev_matrix {
  int rows = 0, cols = 0, n_long = 0, n_slices = 0;
  int64_t stored_count = 0;
  dbuf<int64_t> long_off, slice_off;
  dbuf<int> idx;
  dbuf<double> val;  // unscaled FP64 values (padding: 0)
  dbuf<int> src;     // user CSR position of each stored element (-1: padding)
  int64_t stored() const { return stored_count; }
};

struct device_layout {
  int m = 0, n = 0;
  int64_t nnz = 0;
  dbuf<int> row_new2old, row_old2new, col_new2old, col_old2new;
  dev_matrix A, AT;
};

struct layout_params {
  int long_threshold = 96;
  int window         = 1 << 15;
  // Block-diagonal batches: instance of every user row / column (device, < 65536), or null.
  const int* row_inst = nullptr;
  const int* col_inst = nullptr;
};

// d_off (m+1), d_idx (nnz), d_val (nnz): the user's CSR on the device.  Throws on CUDA errors or
// on column indices outside [0, n).
void build_device_layout(int m, int n, const int* d_off, const int* d_idx, const double* d_val,
                         cudaStream_t s, device_layout& out, const layout_params& p = {});

// Gathers / scatters between user order and internal order.
// dst[i] = sign * src[perm[i]]  (perm = new2old)
void permute_gather(const double* src, const int* perm, int count, double sign, double* dst,
                    cudaStream_t s);
// dst[perm[i]] = sign * src[i]
void permute_scatter(const double* src, const int* perm, int count, double sign, double* dst,
                     cudaStream_t s);

}  // namespace cuopt_b200
