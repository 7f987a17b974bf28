// See tile_layout.cuh.  Built on the device, deterministically: every entry's sort key is
// (tile, row, column), so the order inside a tile does not depend on the input order.
#include "tile_layout.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>

namespace cuopt_b200 {

namespace {

constexpr int kT = 256;

int grid_for(int64_t n)
{
  return (int)std::min<int64_t>(std::max<int64_t>(1, (n + kT - 1) / kT), 1 << 20);
}

struct tile_geom {
  int R, W, panels;
};

// Sort key (tile << 32 | row_local << 17 | col_local) and value of every stored element of M
// (one warp per long row / slice, as the sweeps walk it); padding elements get the key ~0.
__global__ void tile_keys_kernel(const int64_t* long_off, const int64_t* slice_off, int n_long,
                                 int n_slices, int rows, const int* idx, const int* src,
                                 const float* vals, tile_geom g, uint64_t* keys, float* out_vals)
{
  const int lane = threadIdx.x & 31;
  const int gw   = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw   = (gridDim.x * blockDim.x) >> 5;
  auto emit = [&](int64_t p, int row) {
    const int s_ = src[p];
    uint64_t k   = ~0ull;
    if (s_ >= 0) {
      const int col    = idx[p];
      const uint64_t t = (uint64_t)(row / g.R) * (uint64_t)g.panels + (uint64_t)(col / g.W);
      k = (t << 32) | ((uint64_t)(row % g.R) << kTileColBits) | (uint64_t)(col % g.W);
    }
    keys[p]     = k;
    out_vals[p] = s_ >= 0 ? vals[p] : 0.0f;
  };
  for (int w = gw; w < n_long + n_slices; w += nw) {
    if (w < n_long) {
      for (int64_t p = long_off[w] + lane; p < long_off[w + 1]; p += kWarp) emit(p, w);
    } else {
      const int s        = w - n_long;
      const int64_t base = slice_off[s];
      const int len      = (int)((slice_off[s + 1] - base) >> 5);
      const int row      = n_long + s * kWarp + lane;
      for (int k = 0; k < len; ++k) emit(sell_pos(base, k, lane), row < rows ? row : rows - 1);
    }
  }
}

__global__ void tile_count_kernel(const uint64_t* keys, int64_t count, int* tile_len)
{
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < count;
       e += (int64_t)gridDim.x * blockDim.x)
    if (keys[e] != ~0ull) atomicAdd(&tile_len[keys[e] >> 32], 1);
}

// Padded length of tile t: each row's run starts a new 32-entry chunk when it would otherwise
// cross a chunk boundary.  Runs longer than 32 set *bad.
__global__ void tile_pad_kernel(const uint64_t* keys, const int64_t* raw_off, int tiles,
                                int64_t* padded_len, int* bad)
{
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += gridDim.x * blockDim.x) {
    int64_t pos = 0;
    for (int64_t e = raw_off[t]; e < raw_off[t + 1];) {
      const uint32_t row = (uint32_t)(keys[e] >> kTileColBits) & 0x7FFFu;
      int64_t f          = e + 1;
      while (f < raw_off[t + 1] && (((uint32_t)(keys[f] >> kTileColBits) & 0x7FFFu) == row)) ++f;
      const int64_t run = f - e;
      if (run > 32) atomicExch(bad, 1);
      if ((pos & 31) + run > 32) pos = (pos + 31) & ~int64_t(31);
      pos += run;
      e = f;
    }
    padded_len[t] = (pos + 31) & ~int64_t(31);
  }
}

__global__ void tile_fill_kernel(const uint64_t* keys, const float* vals, const int64_t* raw_off,
                                 const int64_t* tile_off, int tiles, uint32_t* out_key,
                                 float* out_val)
{
  const uint32_t pad = kTilePadRow << kTileColBits;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tiles; t += gridDim.x * blockDim.x) {
    const int64_t base = tile_off[t];
    int64_t pos        = 0;
    for (int64_t e = raw_off[t]; e < raw_off[t + 1];) {
      const uint32_t row = (uint32_t)(keys[e] >> kTileColBits) & 0x7FFFu;
      int64_t f          = e + 1;
      while (f < raw_off[t + 1] && (((uint32_t)(keys[f] >> kTileColBits) & 0x7FFFu) == row)) ++f;
      const int64_t run = f - e;
      if ((pos & 31) + run > 32) {
        const int64_t next = (pos + 31) & ~int64_t(31);
        for (; pos < next; ++pos) {
          out_key[base + pos] = pad;
          out_val[base + pos] = 0.0f;
        }
      }
      for (; e < f; ++e, ++pos) {
        out_key[base + pos] = (uint32_t)keys[e];
        out_val[base + pos] = vals[e];
      }
    }
    for (const int64_t end = tile_off[t + 1] - base; pos < end; ++pos) {
      out_key[base + pos] = pad;
      out_val[base + pos] = 0.0f;
    }
  }
}

__global__ void widen_kernel(const int* a, int64_t* b, int count)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    b[i] = a[i];
}

struct temp_bytes {
  dbuf<char> buf;
  void* get(size_t bytes)
  {
    if (bytes > buf.size()) buf.resize(bytes);
    return buf.data();
  }
};

}  // namespace

bool build_tile_matrix(const dev_matrix& M, const float* vals, int sms, size_t smem_limit,
                       cudaStream_t s, tile_matrix& out)
{
  const int rows = M.rows, cols = M.cols;
  const int64_t stored = M.stored();
  if (rows <= 0 || cols <= 0 || stored <= 0 || sms <= 0 || stored >= (1ll << 31)) return false;
  // Geometry: one wave of `sms` blocks when the rows allow it (row blocks x panel groups = sms).
  const int rb_min = (rows + kTileMaxRows - 1) / kTileMaxRows;
  int groups = 1, rb = rb_min;
  if (rb_min <= sms) {
    groups = sms / rb_min;
    rb     = sms / groups;
  }
  int R = 0, W = 0, panels = 0;
  auto shape = [&]() {  // R, W and the panel count for `rb` row blocks
    R = (int)(((int64_t)rows + rb - 1) / rb);
    R = std::min(kTileMaxRows, (R + 3) & ~3);
    rb = (rows + R - 1) / R;
    const int64_t w_room = ((int64_t)smem_limit - (int64_t)R * 4 - 1024) / 8;
    W = (int)std::min<int64_t>({w_room, (1 << kTileColBits) - 4, ((int64_t)cols + 3) & ~3ll});
    W &= ~3;
    panels = W > 0 ? (cols + W - 1) / W : 0;
  };
  shape();
  if (panels > 0 && panels < groups) {
    // Fewer panels than groups: spend the blocks on more (smaller) row blocks instead.
    groups = panels;
    rb     = std::max(rb_min, sms / groups);
    shape();
  }
  if (W < 256) return false;
  groups = std::max(1, std::min(groups, panels));
  const int tiles  = rb * panels;
  if ((int64_t)tiles >= (1ll << 31)) return false;

  alloc_scope scope(s);
  temp_bytes tmp;
  dbuf<uint64_t> keys(stored), keys_sorted(stored);
  dbuf<float> v(stored), v_sorted(stored);
  const tile_geom g{R, W, panels};
  tile_keys_kernel<<<grid_for((int64_t)(M.n_long + M.n_slices) * 32), kT, 0, s>>>(
    M.long_off.data(), M.slice_off.data(), M.n_long, M.n_slices, rows, M.idx.data(),
    M.src.data(), vals, g, keys.data(), v.data());
  B200_LAUNCH_CHECK();
  int tile_bits = 1;
  while ((1ll << tile_bits) <= tiles) ++tile_bits;
  size_t bytes = 0;
  B200_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, bytes, keys.data(), keys_sorted.data(),
                                                  v.data(), v_sorted.data(), (int)stored, 0,
                                                  std::min(64, 32 + tile_bits + 1), s));
  B200_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(tmp.get(bytes), bytes, keys.data(),
                                                  keys_sorted.data(), v.data(), v_sorted.data(),
                                                  (int)stored, 0,
                                                  std::min(64, 32 + tile_bits + 1), s));
  keys.release();
  v.release();
  dbuf<int> tile_len(tiles + 1);
  dbuf<int64_t> raw_len(tiles + 1), raw_off(tiles + 1), pad_len(tiles + 1);
  tile_len.zero(s);
  tile_count_kernel<<<grid_for(stored), kT, 0, s>>>(keys_sorted.data(), stored, tile_len.data());
  B200_LAUNCH_CHECK();
  widen_kernel<<<grid_for(tiles + 1), kT, 0, s>>>(tile_len.data(), raw_len.data(), tiles + 1);
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, raw_len.data(), raw_off.data(),
                                                tiles + 1, s));
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.get(bytes), bytes, raw_len.data(),
                                                raw_off.data(), tiles + 1, s));
  dbuf<int> bad(1);
  bad.zero(s);
  pad_len.zero(s);
  tile_pad_kernel<<<grid_for(tiles), kT, 0, s>>>(keys_sorted.data(), raw_off.data(), tiles,
                                                 pad_len.data(), bad.data());
  B200_LAUNCH_CHECK();
  int hbad = 0;
  B200_CUDA_CHECK(cudaMemcpyAsync(&hbad, bad.data(), sizeof(int), cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  if (hbad) return false;
  out.tile_off.resize(tiles + 1);
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, bytes, pad_len.data(),
                                                out.tile_off.data(), tiles + 1, s));
  B200_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(tmp.get(bytes), bytes, pad_len.data(),
                                                out.tile_off.data(), tiles + 1, s));
  int64_t entries = 0;
  B200_CUDA_CHECK(cudaMemcpyAsync(&entries, out.tile_off.data() + tiles, sizeof(int64_t),
                                  cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  out.key.resize(std::max<int64_t>(entries, 32));
  out.val.resize(std::max<int64_t>(entries, 32));
  tile_fill_kernel<<<grid_for(tiles), kT, 0, s>>>(keys_sorted.data(), v_sorted.data(),
                                                  raw_off.data(), out.tile_off.data(), tiles,
                                                  out.key.data(), out.val.data());
  B200_LAUNCH_CHECK();
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  out.rows       = rows;
  out.cols       = cols;
  out.R          = R;
  out.W          = W;
  out.row_blocks = rb;
  out.panels     = panels;
  out.groups     = groups;
  out.entries    = entries;
  return true;
}

}  // namespace cuopt_b200
