// Tiled copy of a PDHG sweep matrix, for sweeps whose gathered vector does not fit in L1.
//
// On uniformly random sparsity every non-zero of a sliced-ELL sweep gathers one element of the
// iterate from a random address, and the SMs can issue such gathers at about one per cycle each
// (cuOptProfileGatherRate), well below what HBM streams: the sweep is bound by the gather requests,
// not by the matrix bytes.  The tiled copy turns those gathers into shared-memory reads: the rows
// are cut into row blocks of R consecutive rows and the gathered vector into panels of W
// consecutive elements; a thread block owns one row block and a group of panels, copies each panel
// into shared memory with one bulk copy, and accumulates the panel's products into per-row sums
// that also live in shared memory.  Every panel is read once per row block (cols x 4 bytes per
// row block from L2, in large bulk transfers) instead of once per non-zero (a 32-byte sector).
//
// Entry layout: the entries of tile (row block b, panel p) are stored contiguously, sorted by
// (row, column) inside the tile, as a 32-bit key (row_local << 17 | col_local) and an FP32 value,
// and padded so that no row's run crosses a 32-entry boundary: a warp reads one 32-entry chunk
// (coalesced) and sums each row's products with a segmented scan, and only one warp ever updates a
// given row's sum within a tile.  Padding entries carry the row kTilePadRow and value 0.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "device_layout.cuh"

namespace cuopt_b200 {

constexpr int kTileMaxRows      = 32764;  // rows of a row block (a multiple of 4, < kTilePadRow)
constexpr uint32_t kTilePadRow  = 32767;
constexpr int kTileColBits      = 17;     // col_local < 2^17
constexpr int kTileThreads      = 1024;

struct tile_matrix {
  int rows = 0, cols = 0;  // output rows, gathered vector length
  int R = 0, W = 0;        // rows per row block, columns per panel (a multiple of 4)
  int row_blocks = 0, panels = 0, groups = 0;
  int64_t entries = 0;     // padded entry count
  dbuf<int64_t> tile_off;  // row_blocks * panels + 1 entry offsets (multiples of 32)
  dbuf<uint32_t> key;
  dbuf<float> val;
  size_t smem_bytes() const { return (size_t)R * sizeof(float) + 2 * (size_t)W * sizeof(float); }
  // Bytes one sweep copies into shared memory (every panel once per row block).
  double staging_bytes() const { return (double)row_blocks * (double)cols * sizeof(float); }
};

// Builds the tiled copy of M (rows x cols, values `vals` in FP32 at M's stored positions) for a
// device with `sms` SMs and `smem_limit` bytes of shared memory per block.  Returns false, leaving
// `out` empty, when some row has more than 32 entries in one tile.
bool build_tile_matrix(const dev_matrix& M, const float* vals, int sms, size_t smem_limit,
                       cudaStream_t s, tile_matrix& out);

}  // namespace cuopt_b200
