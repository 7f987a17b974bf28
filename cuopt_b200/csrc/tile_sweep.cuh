// Tiled PDHG sweep (see tile_layout.cuh): products of a tiled matrix with a gathered vector whose
// panels are staged into shared memory by bulk copies, followed by a row pass that combines the
// panel groups' partial sums and applies the same epilogue functors as sell_map_kernel.
#pragma once

#include "kernels.cuh"
#include "tile_layout.cuh"

namespace cuopt_b200 {

struct tile_view {
  int rows, cols, R, W, row_blocks, panels, groups;
  const int64_t* tile_off;
  const uint32_t* key;
  const float* val;
};

inline tile_view view_of(const tile_matrix& t)
{
  return tile_view{t.rows,   t.cols,   t.R,          t.W,          t.row_blocks,
                   t.panels, t.groups, t.tile_off.data(), t.key.data(), t.val.data()};
}

// Bounded number of mbarrier polls before a wait gives up (each poll may suspend the thread for a
// short hardware-defined time); a copy of one panel completes within microseconds.
constexpr long long kTileWaitPolls = 1ll << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void tile_mbar_init(uint64_t* bar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void tile_mbar_fence_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One arrival that also announces `bytes` of transaction, then the bulk copy that completes them.
__device__ __forceinline__ void tile_bulk_load(float* dst, const float* src, uint32_t bytes,
                                               uint64_t* bar)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
  asm volatile(
    "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
      smem_addr(dst)),
    "l"(src), "r"(bytes), "r"(smem_addr(bar))
    : "memory");
}
__device__ __forceinline__ bool tile_mbar_try_wait(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
    : "=r"(ok)
    : "r"(smem_addr(bar)), "r"(parity)
    : "memory");
  return ok != 0;
}
// Waits for phase `parity` of `bar`; false (and *err = 1) when the poll limit runs out.
__device__ __forceinline__ bool tile_mbar_wait(uint64_t* bar, uint32_t parity, int* err)
{
  for (long long i = 0; i < kTileWaitPolls; ++i)
    if (tile_mbar_try_wait(bar, parity)) return true;
  atomicExch(err, 1);
  return false;
}

// Block (row block b, panel group g): partial[g * rows + row] = sum over the group's panels of the
// row's products.  Panels are double-buffered: the copy of panel p + 2 is issued as soon as every
// warp has finished panel p.
__global__ void __launch_bounds__(kTileThreads, 1)
  tile_sweep_kernel(const tile_view T, const float* __restrict__ g, float* __restrict__ partial,
                    int* __restrict__ err)
{
  extern __shared__ __align__(16) float tile_smem[];
  __shared__ __align__(8) uint64_t bar[2];
  const int R = T.R, W = T.W;
  float* acc        = tile_smem;
  float* const buf0 = tile_smem + R;
  float* const buf1 = tile_smem + R + W;
  const int rb = blockIdx.x / T.groups, grp = blockIdx.x % T.groups;
  const int p0 = (int)((int64_t)grp * T.panels / T.groups);
  const int p1 = (int)((int64_t)(grp + 1) * T.panels / T.groups);
  const int row0 = rb * R, nrow = min(R, T.rows - row0);
  for (int r = threadIdx.x; r < R; r += kTileThreads) acc[r] = 0.0f;
  if (threadIdx.x == 0) {
    tile_mbar_init(&bar[0]);
    tile_mbar_init(&bar[1]);
    tile_mbar_fence_init();
  }
  __syncthreads();
  auto issue = [&](int p, int b) {
    const int c0  = p * W;
    const int cnt = min(W, T.cols - c0);
    // Rounded up to 16 bytes: the gathered vectors carry 4 elements of padding.
    tile_bulk_load(b ? buf1 : buf0, g + c0, (uint32_t)(((cnt + 3) & ~3) * sizeof(float)),
                   &bar[b]);
  };
  int issued0 = 0, issued1 = 0;  // copies issued into each buffer (thread 0)
  if (threadIdx.x == 0) {
    if (p0 < p1) issue(p0, 0), ++issued0;
    if (p0 + 1 < p1) issue(p0 + 1, 1), ++issued1;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int kWarps = kTileThreads / kWarp;
  // The first kTilePrefetch chunks of a warp in a tile are loaded one tile ahead, into registers,
  // so their HBM latency overlaps the previous tile's work; further chunks load on demand.
  constexpr int kTilePrefetch = 4;
  uint32_t ck[kTilePrefetch], nk[kTilePrefetch];
  float cv[kTilePrefetch], nv[kTilePrefetch];
  auto prefetch = [&](int p, uint32_t(&k)[kTilePrefetch], float(&v)[kTilePrefetch]) {
    int64_t e0 = 0, e1 = 0;
    if (p < p1) {
      const int64_t t = (int64_t)rb * T.panels + p;
      e0 = T.tile_off[t];
      e1 = T.tile_off[t + 1];
    }
#pragma unroll
    for (int i = 0; i < kTilePrefetch; ++i) {
      const int64_t e = e0 + ((int64_t)warp + (int64_t)i * kWarps) * kWarp;
      if (e < e1) {
        k[i] = __ldcs(T.key + e + lane);
        v[i] = __ldcs(T.val + e + lane);
      } else {
        k[i] = kTilePadRow << kTileColBits;
        v[i] = 0.0f;
      }
    }
  };
  // One 32-entry chunk: products with the panel, summed per row run, added to the row's sum.
  auto chunk = [&](const float* panel, uint32_t kk, float v) {
    const int r = (int)(kk >> kTileColBits);
    if (__all_sync(0xffffffffu, r == (int)kTilePadRow)) return;  // nothing loaded into this chunk
    float s      = v * panel[kk & ((1u << kTileColBits) - 1)];
    const int rn = __shfl_down_sync(0xffffffffu, r, 1);
    // Segmented inclusive sum over the chunk's row runs (rows are sorted inside a chunk), only
    // when some row has more than one entry in it.
    if (__any_sync(0xffffffffu, lane < 31 && rn == r)) {
#pragma unroll
      for (int d = 1; d < kWarp; d <<= 1) {
        const float o = __shfl_up_sync(0xffffffffu, s, d);
        const int ro  = __shfl_up_sync(0xffffffffu, r, d);
        if (lane >= d && ro == r) s += o;
      }
    }
    if ((lane == 31 || rn != r) && r != (int)kTilePadRow) acc[r] += s;
  };
  bool ok = true;
  prefetch(p0, ck, cv);
  for (int p = p0; p < p1; ++p) {
    const int k = p - p0, b = k & 1;
    prefetch(p + 1, nk, nv);
    ok = tile_mbar_wait(&bar[b], (uint32_t)((k >> 1) & 1), err) && ok;
    const float* panel = b ? buf1 : buf0;
#pragma unroll
    for (int i = 0; i < kTilePrefetch; ++i) chunk(panel, ck[i], cv[i]);
    const int64_t t  = (int64_t)rb * T.panels + p;
    const int64_t e1 = T.tile_off[t + 1];
    for (int64_t e = T.tile_off[t] + ((int64_t)warp + (int64_t)kTilePrefetch * kWarps) * kWarp;
         e < e1; e += (int64_t)kWarps * kWarp)
      chunk(panel, __ldcs(T.key + e + lane), __ldcs(T.val + e + lane));
    __syncthreads();
    if (threadIdx.x == 0 && p + 2 < p1) {
      issue(p + 2, b);
      ++(b ? issued1 : issued0);
    }
#pragma unroll
    for (int i = 0; i < kTilePrefetch; ++i) {
      ck[i] = nk[i];
      cv[i] = nv[i];
    }
  }
  if (!ok && threadIdx.x == 0) {
    // A wait gave up: give the last copy into each buffer a bounded time to land before exit.
    if (issued0 > 0) tile_mbar_wait(&bar[0], (uint32_t)((issued0 - 1) & 1), err);
    if (issued1 > 0) tile_mbar_wait(&bar[1], (uint32_t)((issued1 - 1) & 1), err);
  }
  float* out = partial + (size_t)grp * T.rows + row0;
  for (int r = threadIdx.x; r < nrow; r += kTileThreads) out[r] = acc[r];
}

// Row pass after tile_sweep_kernel: acc_r = sum of the groups' partial sums (in group order, in
// FP64), then the epilogue of the sweep, exactly as sell_map_kernel applies it.
template <class Epi>
__global__ void __launch_bounds__(kBlock) tile_epilogue_kernel(int rows, int groups,
                                                               const float* __restrict__ partial,
                                                               Epi epi, double* partials)
{
  constexpr int K = Epi::kRed;
  red_t<K> red;
#pragma unroll
  for (int q = 0; q < (K > 0 ? K : 1); ++q) red.v[q] = 0.0;
  for (int r = blockIdx.x * kBlock + threadIdx.x; r < rows; r += gridDim.x * kBlock) {
    const auto pre = epi.load(r);
    double acc     = 0.0;
    for (int q = 0; q < groups; ++q) acc += (double)partial[(size_t)q * rows + r];
    epi(r, acc, pre, red);
  }
  block_reduce_store<K, has_max_red<Epi>::value>(red, partials);
}

}  // namespace cuopt_b200
