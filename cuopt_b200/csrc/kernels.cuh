// sm_100a kernels of the PDLP path.
//
// Every matrix sweep is one launch of `sell_map_kernel`: warps either walk one long row (CSR,
// lanes stride along the row) or one 32-row slice of the sliced-ELL part (lane t owns row t and
// reads element k at base + 32k + t, so each warp load is one contiguous segment).  The row's dot
// product is handed to an epilogue functor that performs the PDHG projection / reflection /
// Halpern step (or a termination / fixed-point-error term) for that row, so x, y and the reflected
// iterate cross HBM once per sweep.  Epilogues may also contribute to up to four block-level sums
// that are reduced deterministically (fixed tree, then one ordered pass over blocks).
#pragma once

#include <type_traits>

#include "common.cuh"

namespace cuopt_b200 {

constexpr int kBlock         = 256;
constexpr int kWarpsPerBlock = kBlock / kWarp;

template <typename T>
struct dev_sell {
  int rows;
  int n_long;
  int n_slices;
  const int64_t* long_off;
  const int64_t* slice_off;
  const int* idx;
  const T* val;
  // Optional work lists (block-diagonal batches with finished instances): when set, a sweep visits
  // only the listed long rows / slices, work_long / work_slices of them.
  const int* long_list  = nullptr;
  const int* slice_list = nullptr;
  int work_long         = 0;
  int work_slices       = 0;
  B200_HD int long_count() const { return long_list ? work_long : n_long; }
  B200_HD int slice_count() const { return slice_list ? work_slices : n_slices; }
};

B200_HD inline int long_blocks(int n_long, int wpb = kWarpsPerBlock) { return ceil_div(n_long, wpb); }
// Grid of sell_map_kernel (and of the setup kernels, which always see full views).
template <typename T>
inline int sell_grid(const dev_sell<T>& a, int wpb = kWarpsPerBlock)
{
  const int g = long_blocks(a.long_count(), wpb) + ceil_div(a.slice_count(), wpb);
  return g > 0 ? g : 1;  // an empty work list still launches one (idle) block
}

// Scalars that change between iterations live on the device so captured graphs stay valid.
struct pdlp_scalars {
  double tau;      // primal step  = eta / omega
  double sigma;    // dual step    = eta * omega
  double eta;      // step size
  double omega;    // primal weight
  long long t0;    // iterations since the last restart, at the start of the next step
};

__device__ __forceinline__ double halpern_weight(const pdlp_scalars* st, int it_off)
{
  const double t = (double)(st->t0 + it_off);
  return (t + 1.0) / (t + 2.0);
}

template <int K>
struct red_t {
  double v[K > 0 ? K : 1];
};

// Block reduction of K doubles (sums, or maxima when MAX); threads 0..K-1 write
// partials[slot * K + r].
template <int K, bool MAX = false>
__device__ __forceinline__ void block_reduce_store(red_t<K>& r, double* partials, int slot)
{
  if constexpr (K > 0) {
    __shared__ double sm[kWarpsPerBlock][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < K; ++q) {
      double v = MAX ? warp_max(r.v[q]) : warp_sum(r.v[q]);
      if (lane == 0) sm[warp][q] = v;
    }
    __syncthreads();
    if (threadIdx.x < K) {
      double s = MAX ? sm[0][threadIdx.x] : 0.0;
#pragma unroll
      for (int w = 0; w < kWarpsPerBlock; ++w)
        s = MAX ? fmax(s, sm[w][threadIdx.x]) : s + sm[w][threadIdx.x];
      partials[(size_t)slot * K + threadIdx.x] = s;
    }
  }
}
template <int K, bool MAX = false>
__device__ __forceinline__ void block_reduce_store(red_t<K>& r, double* partials)
{
  block_reduce_store<K, MAX>(r, partials, (int)blockIdx.x);
}

// Epilogues may declare `static constexpr bool kMaxRed = true`: their block values are then
// combined by maxima instead of sums.
template <class E, class = void>
struct has_max_red : std::false_type {};
template <class E>
struct has_max_red<E, std::void_t<decltype(E::kMaxRed)>> : std::bool_constant<E::kMaxRed> {};

// out[q] = sum over blocks of partials[b*K+q], summed by one block (ordered, compensated).
template <int K>
__device__ __forceinline__ void ordered_block_sum(const double* partials, int nblocks, double* out)
{
  __shared__ double sm[kBlock];
  for (int q = 0; q < K; ++q) {
    ksum acc;
    for (int b = threadIdx.x; b < nblocks; b += kBlock) acc.add(partials[(size_t)b * K + q]);
    sm[threadIdx.x] = acc.value();
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sm[threadIdx.x] += sm[threadIdx.x + s];
      __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = sm[0];
    __syncthreads();
  }
}
template <int K>
__global__ void __launch_bounds__(kBlock) finalize_sum_kernel(const double* partials, int nblocks,
                                                              double* out)
{
  ordered_block_sum<K>(partials, nblocks, out);
}

// p[0 .. n) = v.
static __global__ void fill_kernel(double* p, int n, double v)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// out[q] = max over blocks of partials[b*K+q] (single block).
template <int K>
__global__ void __launch_bounds__(kBlock) finalize_max_kernel(const double* partials, int nblocks,
                                                              double* out)
{
  __shared__ double sm[kBlock];
  for (int q = 0; q < K; ++q) {
    double v = -INFINITY;
    for (int b = threadIdx.x; b < nblocks; b += kBlock) v = fmax(v, partials[(size_t)b * K + q]);
    sm[threadIdx.x] = v;
    __syncthreads();
    for (int s = kBlock / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + s]);
      __syncthreads();
    }
    if (threadIdx.x == 0) out[q] = sm[0];
    __syncthreads();
  }
}

// 4 consecutive values of one lane chunk (16-byte aligned), streamed with evict-first loads.
__device__ __forceinline__ void load_chunk(const float* p, double (&v)[4])
{
  const float4 t = __ldcs(reinterpret_cast<const float4*>(p));
  v[0]           = t.x;
  v[1]           = t.y;
  v[2]           = t.z;
  v[3]           = t.w;
}
__device__ __forceinline__ void load_chunk(const double* p, double (&v)[4])
{
  const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
  const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
  v[0]            = a.x;
  v[1]            = a.y;
  v[2]            = b.x;
  v[3]            = b.y;
}
__device__ __forceinline__ int4 load_idx_chunk(const int* p)
{
  return __ldcs(reinterpret_cast<const int4*>(p));
}

// Epilogues of block-diagonal batches may declare `bool skip_range(int r0, int r1)`: true when
// rows r0..r1 belong only to finished instances, so a warp can skip their dot products.
template <class E, class = void>
struct has_skip_range : std::false_type {};
template <class E>
struct has_skip_range<E, std::void_t<decltype(&E::skip_range)>> : std::true_type {};

template <class Epi>
__device__ __forceinline__ bool skip_rows(const Epi& epi, int r0, int r1)
{
  if constexpr (has_skip_range<Epi>::value)
    return epi.skip_range(r0, r1);
  else
    return false;
}

// Generic fused sweep: acc_r = sum_k A[r,k] * g[idx[r,k]], then epi(r, acc_r, pre, red).
// The epilogue's per-row operands (`pre`) are loaded before the matrix loop so their memory latency
// overlaps the gathers.  Sliced rows are read in 4-element lane chunks, two chunks in flight.
// `vb` is the block's index in the sweep's grid (blockIdx.x, or a virtual index in a persistent
// kernel that walks the grid).
// Gathered-vector loads.  A kernel that writes the gathered vector itself (the persistent
// iterations below) reads it through L2 (ld.global.cg), which its grid barrier keeps coherent;
// every other sweep uses plain loads of the restrict-qualified vector, which no sweep writes
// (an explicit __ldg measured slower on the mixed-precision primal sweep: 73.1 against 69.9 us on
// the 1M x 2M LP).
template <bool COH, typename T>
__device__ __forceinline__ T gather_load(const T* __restrict__ g, int i)
{
  if constexpr (COH)
    return __ldcg(g + i);
  else
    return g[i];
}

// Where a sweep reads the matrix's values and indices from: global memory with evict-first loads
// (every sweep but one), or a copy of the block's own virtual blocks in shared memory (the
// cluster power iteration), whose element k of the view's arrays sits at k - shift.
struct global_matrix {
  static constexpr int64_t shift = 0;
  template <typename T>
  __device__ __forceinline__ T ld(const T* p) const
  {
    return ld_stream(p);
  }
  template <typename T>
  __device__ __forceinline__ void chunk(const T* p, double (&v)[4]) const
  {
    load_chunk(p, v);
  }
  __device__ __forceinline__ int4 idx_chunk(const int* p) const { return load_idx_chunk(p); }
};
struct shared_matrix {
  int64_t shift;
  template <typename T>
  __device__ __forceinline__ T ld(const T* p) const
  {
    return *p;
  }
  __device__ __forceinline__ void chunk(const float* p, double (&v)[4]) const
  {
    const float4 t = *reinterpret_cast<const float4*>(p);
    v[0]           = t.x;
    v[1]           = t.y;
    v[2]           = t.z;
    v[3]           = t.w;
  }
  __device__ __forceinline__ void chunk(const double* p, double (&v)[4]) const
  {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    v[0]            = a.x;
    v[1]            = a.y;
    v[2]            = b.x;
    v[3]            = b.y;
  }
  __device__ __forceinline__ int4 idx_chunk(const int* p) const
  {
    return *reinterpret_cast<const int4*>(p);
  }
};

// WPB: warps (rows or slices) per block.  Only the grouping of warps into blocks depends on it,
// not any row's arithmetic; sweeps with block reductions (kRed > 0) use kWarpsPerBlock.
template <typename TM, typename TG, class Epi, bool COH = false, int WPB = kWarpsPerBlock,
          class MS = global_matrix>
__device__ __forceinline__ void sell_map_block(const dev_sell<TM>& A, const TG* __restrict__ g,
                                               const Epi& epi, double* partials, int vb,
                                               const MS& ms = MS{})
{
  constexpr int K = Epi::kRed;
  static_assert(K == 0 || WPB == kWarpsPerBlock, "block reductions assume kWarpsPerBlock warps");
  red_t<K> red;
#pragma unroll
  for (int q = 0; q < (K > 0 ? K : 1); ++q) red.v[q] = 0.0;
  if (epi.skip()) {
    // Uniform early exit (e.g. converged power iteration): every block still stores zeros.
    block_reduce_store<K, has_max_red<Epi>::value>(red, partials, vb);
    return;
  }
  const int lane = threadIdx.x & 31, warp = (threadIdx.x >> 5) & (WPB - 1);
  const int lb   = long_blocks(A.long_count(), WPB);
  if (vb < lb) {
    const int q   = vb * WPB + warp;
    const int row = q < A.long_count() ? (A.long_list ? A.long_list[q] : q) : 0;
    if (q < A.long_count() && !skip_rows(epi, row, row)) {
      const auto pre  = epi.load(row);
      const int64_t b = A.long_off[row] - ms.shift, e = A.long_off[row + 1] - ms.shift;
      double acc      = 0.0;
      for (int64_t k = b + lane; k < e; k += kWarp)
        acc += (double)ms.ld(A.val + k) * (double)gather_load<COH>(g, ms.ld(A.idx + k));
      acc = warp_sum(acc);
      if (lane == 0) epi(row, acc, pre, red);
    }
  } else {
    const int q = (vb - lb) * WPB + warp;
    const int s = q < A.slice_count() ? (A.slice_list ? A.slice_list[q] : q) : 0;
    if (q < A.slice_count() &&
        !skip_rows(epi, A.n_long + s * kWarp, min(A.n_long + s * kWarp + kWarp, A.rows) - 1)) {
      const int row      = A.n_long + s * kWarp + lane;
      const bool valid   = row < A.rows;
      const auto pre     = epi.load(valid ? row : A.rows - 1);
      const int64_t base = A.slice_off[s];
      const int nchunk   = (int)((A.slice_off[s + 1] - base) >> 7);  // 32 lanes x 4 elements
      const TM* v        = A.val + (base - ms.shift) + lane * kChunk;
      const int* ix      = A.idx + (base - ms.shift) + lane * kChunk;
      double acc         = 0.0;
      int q              = 0;
      for (; q + 2 <= nchunk; q += 2) {
        const int4 i0 = ms.idx_chunk(ix), i1 = ms.idx_chunk(ix + 32 * kChunk);
        double v0[4], v1[4];
        ms.chunk(v, v0);
        ms.chunk(v + 32 * kChunk, v1);
        const TG g0 = gather_load<COH>(g, i0.x), g1 = gather_load<COH>(g, i0.y);
        const TG g2 = gather_load<COH>(g, i0.z), g3 = gather_load<COH>(g, i0.w);
        const TG g4 = gather_load<COH>(g, i1.x), g5 = gather_load<COH>(g, i1.y);
        const TG g6 = gather_load<COH>(g, i1.z), g7 = gather_load<COH>(g, i1.w);
        acc += v0[0] * (double)g0;
        acc += v0[1] * (double)g1;
        acc += v0[2] * (double)g2;
        acc += v0[3] * (double)g3;
        acc += v1[0] * (double)g4;
        acc += v1[1] * (double)g5;
        acc += v1[2] * (double)g6;
        acc += v1[3] * (double)g7;
        v += 64 * kChunk;
        ix += 64 * kChunk;
      }
      if (q < nchunk) {
        const int4 i0 = ms.idx_chunk(ix);
        double v0[4];
        ms.chunk(v, v0);
        const TG g0 = gather_load<COH>(g, i0.x), g1 = gather_load<COH>(g, i0.y);
        const TG g2 = gather_load<COH>(g, i0.z), g3 = gather_load<COH>(g, i0.w);
        acc += v0[0] * (double)g0;
        acc += v0[1] * (double)g1;
        acc += v0[2] * (double)g2;
        acc += v0[3] * (double)g3;
      }
      if (valid) epi(row, acc, pre, red);
    }
  }
  block_reduce_store<K, has_max_red<Epi>::value>(red, partials, vb);
}

template <typename TM, typename TG, class Epi>
__global__ void __launch_bounds__(kBlock) sell_map_kernel(const dev_sell<TM> A,
                                                          const TG* __restrict__ g, Epi epi,
                                                          double* partials)
{
  sell_map_block(A, g, epi, partials, (int)blockIdx.x);
}

// Blocks vb0, vb0 + 1, ... of a sweep's grid only (measurement of one row-length class: the
// long rows are blocks [0, long_blocks), the slices the rest).
template <typename TM, typename TG, class Epi>
__global__ void __launch_bounds__(kBlock) sell_map_range_kernel(const dev_sell<TM> A,
                                                                const TG* __restrict__ g, Epi epi,
                                                                double* partials, int vb0)
{
  sell_map_block(A, g, epi, partials, vb0 + (int)blockIdx.x);
}

// The same sweep with WPB warps per block (the plain sweeps' block shape is autotuned).
template <typename TM, typename TG, class Epi, int WPB>
__global__ void __launch_bounds__(WPB * kWarp) sell_map_wpb_kernel(const dev_sell<TM> A,
                                                                  const TG* __restrict__ g,
                                                                  Epi epi, double* partials)
{
  sell_map_block<TM, TG, Epi, false, WPB>(A, g, epi, partials, (int)blockIdx.x);
}

// Launches sell_map_wpb_kernel with wpb (4, 8 or 16) warps per block.
template <typename TM, typename TG, class Epi>
void launch_sell_wpb(int wpb, const dev_sell<TM>& A, const TG* g, const Epi& epi,
                     double* partials, cudaStream_t s)
{
  const int grid = sell_grid(A, wpb);
  switch (wpb) {
    case 4:
      sell_map_wpb_kernel<TM, TG, Epi, 4><<<grid, 4 * kWarp, 0, s>>>(A, g, epi, partials);
      break;
    case 16:
      sell_map_wpb_kernel<TM, TG, Epi, 16><<<grid, 16 * kWarp, 0, s>>>(A, g, epi, partials);
      break;
    default:
      sell_map_kernel<TM, TG, Epi><<<sell_grid(A), kBlock, 0, s>>>(A, g, epi, partials);
  }
}

// ---------------------------------------------------------------------------------------------
// Persistent plain iterations: one cooperative launch runs L primal / dual sweep pairs with a
// grid-wide barrier after each sweep, instead of 2L kernel nodes of a CUDA graph.  Block b takes
// the sweep's virtual blocks b, b + gridDim.x, ... in both sweeps of every iteration, so each row's
// own iterates are read back by the thread that wrote them; the gathered vectors, written by other
// blocks, are read through L2.
//
// Every wait is bounded: a barrier that is not reached before the launch's deadline (read from
// %globaltimer) or within kBarrierPolls polls stores a status in the control block and every block
// returns; the host reads the status at its next synchronisation and fails the solve.

struct persist_ctl {
  unsigned arrivals;  // barrier arrivals of the current launch (zeroed before each launch)
  int status;         // 0, or kBarrierTimedOut / kBarrierPollLimit
};
constexpr int kBarrierTimedOut  = 1;
constexpr int kBarrierPollLimit = 2;
constexpr unsigned kBarrierPolls = 1u << 24;
// Deadline of one persistent launch of the solvers (at most 255 iterations): far above any
// legitimate run, it only bounds a launch whose grid barrier could not complete.
constexpr unsigned long long kPersistBudgetNs = 30ull * 1000 * 1000 * 1000;

__device__ __forceinline__ unsigned long long global_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p)
{
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void red_release_gpu_add(unsigned* p, unsigned v)
{
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_relaxed_gpu(const int* p)
{
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Arrive and wait until `target` arrivals have been counted.  Returns false (uniformly across
// the block) when the wait gave up or another block's wait already had.  The block's writes reach
// thread 0 through the block barrier; its arrival is a release at GPU scope (cumulative over
// them), and the poll that sees the last arrival an acquire, after which the block barrier hands
// the other blocks' writes on to every thread.
__device__ __forceinline__ bool persist_barrier(persist_ctl* c, unsigned target,
                                                unsigned long long deadline)
{
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    red_release_gpu_add(&c->arrivals, 1u);
    int st = 0;
    for (unsigned polls = 0;; ++polls) {
      if (ld_acquire_gpu(&c->arrivals) >= target) break;
      if ((st = ld_relaxed_gpu(&c->status)) != 0) break;
      if (polls >= kBarrierPolls) {
        st = kBarrierPollLimit;
        atomicCAS(&c->status, 0, st);
        break;
      }
      if ((polls & 15) == 15 && global_ns() > deadline) {
        st = kBarrierTimedOut;
        atomicCAS(&c->status, 0, st);
        break;
      }
    }
    ok = st == 0;
  }
  __syncthreads();
  return ok;
}

// Block 0's closing step of a persistent launch (after the last barrier): the iteration counter
// of the one LP, or of every active instance of a batch, moves on by L.
struct advance_one {
  pdlp_scalars* st;
  __device__ void operator()(int steps) const
  {
    if (threadIdx.x == 0) st->t0 += steps;
  }
};
struct advance_active {
  pdlp_scalars* sc;
  const int* active;
  int count;
  __device__ void operator()(int steps) const
  {
    for (int b = threadIdx.x; b < count; b += blockDim.x)
      if (active[b]) sc[b].t0 += steps;
  }
};

template <typename TX, class PE, class DE, class ADV>
__global__ void __launch_bounds__(kBlock)
  persistent_plain_kernel(const dev_sell<TX> AT, const dev_sell<TX> A, const TX* y, const TX* xbar,
                          PE pe, DE de, ADV adv, int L, int grid_p, int grid_d, persist_ctl* ctl,
                          unsigned long long budget_ns)
{
  const unsigned long long deadline = global_ns() + budget_ns;
  unsigned target                   = 0;
  for (int i = 0; i < L; ++i) {
    pe.it_off = i;
    for (int vb = blockIdx.x; vb < grid_p; vb += gridDim.x)
      sell_map_block<TX, TX, PE, true>(AT, y, pe, nullptr, vb);
    target += gridDim.x;
    if (!persist_barrier(ctl, target, deadline)) return;
    de.it_off = i;
    for (int vb = blockIdx.x; vb < grid_d; vb += gridDim.x)
      sell_map_block<TX, TX, DE, true>(A, xbar, de, nullptr, vb);
    target += gridDim.x;
    if (!persist_barrier(ctl, target, deadline)) return;
  }
  if (blockIdx.x == 0) adv(L);
}

// The barrier alone, for measuring its cost and for checking that a wait which cannot complete
// (`unreachable` > 0 asks for more arrivals than the grid has blocks) ends with a status instead
// of hanging: `rounds` barriers, then block 0 records the elapsed nanoseconds.
static __global__ void persist_barrier_probe_kernel(persist_ctl* ctl, int rounds, unsigned unreachable,
                                                    unsigned long long budget_ns,
                                                    unsigned long long* elapsed)
{
  const unsigned long long t0 = global_ns(), deadline = t0 + budget_ns;
  unsigned target = 0;
  for (int r = 0; r < rounds; ++r) {
    target += gridDim.x;
    if (!persist_barrier(ctl, target + unreachable, deadline)) break;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) *elapsed = global_ns() - t0;
}

// ---------------------------------------------------------------------------------------------
// PDHG epilogues (reflected variant, reference pdhg.cu:431-530 and pdlp.cu:2506-2563).

// The primal update of one variable j (shared by the single-LP and batch epilogues); `p` holds
// x_j, c_j, l_j, u_j and the anchor x_a,j, `st` the step scalars of j's LP.
// Receives the value a row step stores into the vector the next sweep gathers (x_bar for the
// primal step, y for the fused-Halpern dual step); the cluster-resident form copies it into the
// cluster's shared-memory copies.
struct no_sink {
  __device__ __forceinline__ void operator()(int, double) const {}
};

template <typename TX, bool MAJOR, bool HALPERN, bool SAVE_ATY, class P, class Sink = no_sink>
__device__ __forceinline__ void primal_row_step(int j, double acc, const P& p,
                                                const pdlp_scalars* st, int it_off, TX* xbar,
                                                TX* xout, TX* xhat, TX* slack, TX* aty,
                                                const Sink& sink = Sink{})
{
  const double tau  = st->tau;
  const double xj   = (double)p.x;
  const double next = xj - tau * ((double)p.c - acc);
  const double cl   = fmax(fmin(next, (double)p.up), (double)p.lo);
  if constexpr (MAJOR) {
    xhat[j]  = (TX)cl;
    slack[j] = (TX)((cl - next) / tau);
  }
  const double xb = 2.0 * cl - xj;
  if constexpr (SAVE_ATY) aty[j] = (TX)acc;
  if constexpr (HALPERN) {
    const double w = halpern_weight(st, it_off);
    xbar[j]        = (TX)xb;
    xout[j]        = (TX)(w * xb + (1.0 - w) * (double)p.xa);
  } else {
    xbar[j] = (TX)xb;
  }
  sink(j, (double)(TX)xb);
}

// The dual update of one constraint i; returns (y_bar_i - y_i)^2 for the fixed-point error.
template <typename TX, bool MAJOR, bool HALPERN, class P, class Sink = no_sink>
__device__ __forceinline__ double dual_row_step(int i, double acc, const P& p,
                                                const pdlp_scalars* st, int it_off, TX* ybar,
                                                TX* yout, TX* yhat, const Sink& sink = Sink{})
{
  const double sigma = st->sigma;
  const double yi    = (double)p.y;
  const double t     = yi / sigma - acc;
  const double tp    = fmax(-(double)p.up, fmin(t, -(double)p.lo));
  const double ny    = (t - tp) * sigma;
  if constexpr (MAJOR) yhat[i] = (TX)ny;
  const double yb = 2.0 * ny - yi;
  if constexpr (HALPERN) {
    const double w  = halpern_weight(st, it_off);
    const TX y_next = (TX)(w * yb + (1.0 - w) * (double)p.ya);
    yout[i]         = y_next;
    sink(i, (double)y_next);
  } else {
    ybar[i] = (TX)yb;
  }
  const double d = yb - yi;
  return d * d;
}

// Row j of A^T:  x_next = x - tau (c - A^T y);  x_hat = clamp(x_next, l, u);
//                slack = (x_hat - x_next) / tau;  x_bar = 2 x_hat - x;
//                (fused Halpern)  x <- w x_bar + (1 - w) x_anchor.
template <typename TX, bool MAJOR, bool HALPERN, bool SAVE_ATY>
struct primal_epi {
  static constexpr int kRed = 0;
  const TX* x;
  const TX* c;
  const TX* lo;
  const TX* up;
  const TX* xa;
  TX* xbar;
  TX* xout;
  TX* xhat;
  TX* slack;
  TX* aty;
  const pdlp_scalars* st;
  int it_off;
  struct pre_t {
    TX x, c, lo, up, xa;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int j) const
  {
    return pre_t{x[j], c[j], lo[j], up[j], HALPERN ? xa[j] : TX(0)};
  }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<0>&) const
  {
    primal_row_step<TX, MAJOR, HALPERN, SAVE_ATY>(j, acc, p, st, it_off, xbar, xout, xhat, slack,
                                                  aty);
  }
};

// Row i of A:  t = y / sigma - A x_bar;  y_hat = (t - clamp(t, -u, -l)) sigma;  y_bar = 2 y_hat - y;
//              (fused Halpern) y <- w y_bar + (1 - w) y_anchor;  (FPE) red += (y_bar - y)^2.
template <typename TX, bool MAJOR, bool HALPERN, bool FPE>
struct dual_epi {
  static constexpr int kRed = FPE ? 1 : 0;
  const TX* y;
  const TX* lo;
  const TX* up;
  const TX* ya;
  TX* ybar;
  TX* yout;
  TX* yhat;
  const pdlp_scalars* st;
  int it_off;
  struct pre_t {
    TX y, lo, up, ya;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int i) const
  {
    return pre_t{y[i], lo[i], up[i], HALPERN ? ya[i] : TX(0)};
  }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p,
                                             red_t<kRed>& r) const
  {
    const double d2 = dual_row_step<TX, MAJOR, HALPERN>(i, acc, p, st, it_off, ybar, yout, yhat);
    if constexpr (FPE) r.v[0] += d2;
  }
};

// ---------------------------------------------------------------------------------------------
// Cluster-resident plain iterations for small LPs: one thread-block cluster of C blocks runs a run
// of L plain iterations.  Every block keeps a full copy of both gathered vectors (y for the primal
// sweep, x_bar for the dual sweep) in its shared memory, so the sweeps gather from shared memory;
// a row's new value is written to global memory by its epilogue, as in the other forms, and
// stored into every block's copy through distributed shared memory (mapa + st.shared::cluster).
// A cluster barrier (arrive.release / wait.acquire: hardware, no spin loop) follows every sweep.
// Every row is computed by one warp exactly as in sell_map_kernel.
constexpr int kClusterThreads = 1024;
constexpr int kClusterGroups  = kClusterThreads / kBlock;  // 8-warp groups per block

__device__ __forceinline__ unsigned cluster_rank()
{
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size()
{
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_barrier()
{
  asm volatile(
    "barrier.cluster.arrive.release.aligned;\n"
    "barrier.cluster.wait.acquire.aligned;\n" ::
      : "memory");
}
// Stores v at shared-memory address saddr (a byte offset in this block's window) of block `rank`
// of the cluster.
__device__ __forceinline__ void dsmem_store(unsigned saddr, unsigned rank, double v)
{
  unsigned remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(saddr), "r"(rank));
  asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(remote), "d"(v) : "memory");
}
__device__ __forceinline__ void dsmem_store(unsigned saddr, unsigned rank, float v)
{
  unsigned remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(saddr), "r"(rank));
  asm volatile("st.shared::cluster.f32 [%0], %1;" ::"r"(remote), "f"(v) : "memory");
}

// Copies a row's new value into every block's shared-memory copy of its vector (base: the
// shared-memory address of the copy in this block's window).
template <typename TX>
struct dsmem_sink {
  unsigned base;
  unsigned blocks;
  __device__ __forceinline__ void operator()(int r, double v) const
  {
    const unsigned target = base + (unsigned)r * (unsigned)sizeof(TX);
    for (unsigned c = 0; c < blocks; ++c) dsmem_store(target, c, (TX)v);
  }
};

// The plain epilogues (primal_epi / dual_epi with the Halpern step fused) with the new x_bar_j,
// or y_i, also sent to the cluster's copies.
template <typename TX>
struct cluster_primal_epi {
  static constexpr int kRed = 0;
  using base_t              = primal_epi<TX, false, true, false>;
  using pre_t               = typename base_t::pre_t;
  base_t base;
  dsmem_sink<TX> sink;
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int j) const { return base.load(j); }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<0>&) const
  {
    primal_row_step<TX, false, true, false>(j, acc, p, base.st, base.it_off, base.xbar, base.xout,
                                            base.xhat, base.slack, base.aty, sink);
  }
};
template <typename TX>
struct cluster_dual_epi {
  static constexpr int kRed = 0;
  using base_t              = dual_epi<TX, false, true, false>;
  using pre_t               = typename base_t::pre_t;
  base_t base;
  dsmem_sink<TX> sink;
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int i) const { return base.load(i); }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<0>&) const
  {
    dual_row_step<TX, false, true>(i, acc, p, base.st, base.it_off, base.ybar, base.yout,
                                   base.yhat, sink);
  }
};

// Dynamic shared memory: the copy of y (m elements, padded to 16), then the copy of x_bar (n
// elements).  pe / de: the plain primal / dual epilogues (it_off set per iteration), whose gathered
// vectors are y (de.y = de.yout) and x_bar (pe.xbar).  Each block runs kClusterGroups groups of
// kWarpsPerBlock warps; group g of block `rank` takes the sweep's 8-warp virtual blocks
// rank + C g, rank + C g + C kClusterGroups, ... (gp / gd of them), so small sweeps spread over
// every block of the cluster.
template <typename TX>
__global__ void __launch_bounds__(kClusterThreads)
  cluster_plain_kernel(const dev_sell<TX> AT, const dev_sell<TX> A,
                       primal_epi<TX, false, true, false> pe, dual_epi<TX, false, true, false> de,
                       int L, int m, int gp, int gd, pdlp_scalars* st)
{
  extern __shared__ __align__(16) unsigned char cl_smem[];
  TX* ys          = reinterpret_cast<TX*>(cl_smem);
  const int m_pad = (m + 15) & ~15;
  TX* xbs         = ys + m_pad;
  const unsigned rank = cluster_rank(), blocks = cluster_size();
  for (int i = threadIdx.x; i < m; i += blockDim.x) ys[i] = de.y[i];
  // Every block of the cluster is running (and has its copy of y) before any block stores into
  // another's shared memory.
  cluster_barrier();
  const dsmem_sink<TX> to_xbs{(unsigned)__cvta_generic_to_shared(xbs), blocks};
  const dsmem_sink<TX> to_ys{(unsigned)__cvta_generic_to_shared(ys), blocks};
  const int group  = threadIdx.x / (kWarpsPerBlock * kWarp);
  const int first  = (int)rank + (int)blocks * group;
  const int stride = (int)blocks * kClusterGroups;
  for (int it = 0; it < L; ++it) {
    pe.it_off = it;
    de.it_off = it;
    const cluster_primal_epi<TX> bp{pe, to_xbs};
    for (int vb = first; vb < gp; vb += stride)
      sell_map_block<TX, TX, cluster_primal_epi<TX>>(AT, ys, bp, nullptr, vb);
    cluster_barrier();
    const cluster_dual_epi<TX> bd{de, to_ys};
    for (int vb = first; vb < gd; vb += stride)
      sell_map_block<TX, TX, cluster_dual_epi<TX>>(A, xbs, bd, nullptr, vb);
    cluster_barrier();
  }
  if (rank == 0 && threadIdx.x == 0) st->t0 += L;
}


// Row j of A^T applied to y_bar: interaction (A^T y_bar - A^T y) . (x_bar - x) and |x_bar - x|^2
// (reference adaptive_step_size_strategy.cu:352-518).
template <typename TX>
struct fpe_epi {
  static constexpr int kRed = 2;
  const TX* aty;
  const TX* xbar;
  const TX* x;
  struct pre_t {
    TX aty, xbar, x;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int j) const { return pre_t{aty[j], xbar[j], x[j]}; }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<2>& r) const
  {
    const double d  = acc - (double)p.aty;
    const double dx = (double)p.xbar - (double)p.x;
    r.v[0] += d * dx;
    r.v[1] += dx * dx;
  }
};

// Halpern update for iterations whose step kept x / y (fixed-point-error iterations).
template <typename TX>
__global__ void halpern_kernel(TX* x, const TX* xbar, const TX* xa, int n, TX* y, const TX* ybar,
                               const TX* ya, int m, const pdlp_scalars* st)
{
  const double w = halpern_weight(st, 0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n)
      x[i] = (TX)(w * (double)xbar[i] + (1.0 - w) * (double)xa[i]);
    else {
      const int r = i - n;
      y[r]        = (TX)(w * (double)ybar[r] + (1.0 - w) * (double)ya[r]);
    }
  }
}

static __global__ void advance_kernel(pdlp_scalars* st, int steps) { st->t0 += steps; }
static __global__ void set_scalars_kernel(pdlp_scalars* st, double tau, double sigma, double eta,
                                   double omega, long long t0)
{
  st->tau   = tau;
  st->sigma = sigma;
  st->eta   = eta;
  st->omega = omega;
  st->t0    = t0;
}

// ---------------------------------------------------------------------------------------------
// Termination (reference convergence_information.cu:492-811) on the unscaled FP64 problem.

// x_u = (x_hat dc) / beta ; y_u = (y_hat dr) / gamma ; s_u = (slack / dc) / gamma
// (unscale_solutions, initial_scaling.cu:684-790).
template <typename TX>
__global__ void unscale_kernel(const TX* xhat, const TX* yhat, const TX* slack, const double* dc,
                               const double* dr, double inv_beta, double inv_gamma, int n, int m,
                               double* xu, double* yu, double* su)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      const double d = dc[i];
      xu[i]          = ((double)xhat[i] * d) * inv_beta;
      const double s = (double)slack[i];
      su[i]          = (d != 0.0 ? s / d : s) * inv_gamma;
    } else {
      const int r = i - n;
      yu[r]       = ((double)yhat[r] * dr[r]) * inv_gamma;
    }
  }
}

__device__ __forceinline__ double finite_or_zero(double v) { return isfinite(v) ? v : 0.0; }

// Row i of A (unscaled): r_p = Ax - clamp(Ax, lc, uc); primal slack for the dual objective.
struct term_primal_epi {
  static constexpr int kRed = 2;
  const double* lc;
  const double* uc;
  const double* y;
  struct pre_t {
    double l, u, y;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{lc[i], uc[i], y[i]}; }
  __device__ __forceinline__ void operator()(int i, double ax, const pre_t& p, red_t<2>& r) const
  {
    const double l = p.l, u = p.u;
    const double cl = fmax(l, fmin(ax, u));
    const double rp = ax - cl;
    const double yi = p.y;
    r.v[0] += rp * rp;
    r.v[1] += fmax(yi, 0.0) * finite_or_zero(l) + fmin(yi, 0.0) * finite_or_zero(u);
  }
};

// Row j of A^T (unscaled): r_d = (c - A^T y) - slack; c.x; slack.x.
struct term_dual_epi {
  static constexpr int kRed = 3;
  const double* c;
  const double* x;
  const double* s;
  struct pre_t {
    double c, x, s;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int j) const { return pre_t{c[j], x[j], s[j]}; }
  __device__ __forceinline__ void operator()(int j, double aty, const pre_t& p, red_t<3>& r) const
  {
    const double cj = p.c, xj = p.x, sj = p.s;
    const double rd = (cj - aty) - sj;
    r.v[0] += rd * rd;
    r.v[1] += cj * xj;
    r.v[2] += sj * xj;
  }
};

// Per-constraint forms of the residuals (per_constraint_residual; reference
// convergence_information.cu:390-420, 453-470 with relative_residual_t, utils.cuh:578-590):
// max(0, max_i r_p,i - rel * max(|l_i|, |u_i|) over the finite bounds (combine_finite_abs_bounds,
// utils.cuh:180-188)) over the rows of A, and max(0, max_j r_d,j - rel * c_j) over the rows of A^T.
struct term_linf_primal_epi {
  static constexpr int kRed     = 1;
  static constexpr bool kMaxRed = true;
  const double* lc;
  const double* uc;
  double rel;
  struct pre_t {
    double l, u;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{lc[i], uc[i]}; }
  __device__ __forceinline__ void operator()(int, double ax, const pre_t& p, red_t<1>& r) const
  {
    const double rp = ax - fmax(p.l, fmin(ax, p.u));
    double cb       = 0.0;
    if (isfinite(p.u)) cb = fmax(cb, fabs(p.u));
    if (isfinite(p.l)) cb = fmax(cb, fabs(p.l));
    r.v[0] = fmax(r.v[0], rp - rel * cb);
  }
};
struct term_linf_dual_epi {
  static constexpr int kRed     = 1;
  static constexpr bool kMaxRed = true;
  const double* c;
  const double* s;
  double rel;
  struct pre_t {
    double c, s;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int j) const { return pre_t{c[j], s[j]}; }
  __device__ __forceinline__ void operator()(int, double aty, const pre_t& p, red_t<1>& r) const
  {
    const double rd = (p.c - aty) - p.s;
    r.v[0]          = fmax(r.v[0], rd - rel * p.c);
  }
};

// Plain sweep epilogues.
template <typename TX>
struct store_epi {  // out[r] = acc
  static constexpr int kRed = 0;
  TX* out;
  const int* done;  // optional early-exit flag
  struct pre_t {};
  __device__ bool skip() const { return done && *done; }
  __device__ __forceinline__ pre_t load(int) const { return pre_t{}; }
  __device__ __forceinline__ void operator()(int r, double acc, const pre_t&, red_t<0>&) const
  {
    out[r] = (TX)acc;
  }
};

// Power iteration z = A (A^T q) with q . z accumulated (reference pdlp.cu:2664-2711).
struct power_z_epi {
  static constexpr int kRed = 1;
  double* z;
  const double* q;
  const int* done;
  struct pre_t {
    double q;
  };
  __device__ bool skip() const { return *done != 0; }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{q[i]}; }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<1>& r) const
  {
    z[i] = acc;
    r.v[0] += p.q * acc;
  }
};

// ---------------------------------------------------------------------------------------------
// Reductions over plain vectors (block partials; finalize with finalize_sum_kernel).

// mode 0: sum x^2 ; mode 1: sum (a-b)^2 ; mode 2: bound norm terms of (lo, up)
template <int MODE, typename TA>
__global__ void __launch_bounds__(kBlock) vec_reduce_kernel(const TA* a, const TA* b, int n,
                                                            double* partials, const int* done)
{
  red_t<1> r;
  r.v[0] = 0.0;
  if (!(done && *done)) {
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
      if constexpr (MODE == 0) {
        const double v = (double)a[i];
        r.v[0] += v * v;
      } else if constexpr (MODE == 1) {
        const double d = (double)a[i] - (double)b[i];
        r.v[0] += d * d;
      } else {
        const double l = (double)a[i], u = (double)b[i];
        double s       = 0.0;
        if (isfinite(l) && l != u) s += l * l;
        if (isfinite(u)) s += u * u;
        r.v[0] += s;
      }
    }
  }
  block_reduce_store<1>(r, partials);
}

// ---------------------------------------------------------------------------------------------
// Power iteration helpers (reference pdlp.cu:2620-2731).  State on device:
//   pi[0] = |z|, pi[1] = sigma_max^2, pi[2] = |residual|, done flag, iteration counter.
struct power_state {
  double norm_z;
  double s2;
  double resid;
  int done;
  int iters;
};

// The power iteration's vector steps.  Each scalar a step needs is summed by the consuming block
// itself from the producer's block partials (ordered_block_sum, as finalize_sum_kernel does, so
// every block gets the value finalize_sum_kernel would store): no separate finalize launches.
//   q = z / |z|, |z|^2 from the vec_reduce partials (nz blocks).
static __global__ void __launch_bounds__(kBlock)
  power_normalize_sum_kernel(const double* z, double* q, int m, const double* part_z, int nz,
                             power_state* ps)
{
  if (ps->done) return;
  __shared__ double total;
  ordered_block_sum<1>(part_z, nz, &total);
  const double nq = sqrt(total);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    q[i] = z[i] / nq;
  if (blockIdx.x == 0 && threadIdx.x == 0) ps->norm_z = nq;
}
//   s2 = q . z from the power_z sweep's partials (ns blocks); q <- q (-s2) + z; partial sums of
//   squares of the result in part_r.
static __global__ void __launch_bounds__(kBlock)
  power_residual_sum_kernel(double* q, const double* z, int m, const double* part_s, int ns,
                            const power_state* ps, double* part_r)
{
  red_t<1> r;
  r.v[0] = 0.0;
  if (!ps->done) {
    __shared__ double s2;
    ordered_block_sum<1>(part_s, ns, &s2);
    const double s = s2;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < m; i += gridDim.x * kBlock) {
      const double v = q[i] * -s + z[i];
      q[i]           = v;
      r.v[0] += v * v;
    }
  }
  block_reduce_store<1>(r, part_r);
}
//   Record s2 and the residual (one block); done once the residual is below tol.
static __global__ void __launch_bounds__(kBlock)
  power_check_sum_kernel(power_state* ps, const double* part_s, int ns, const double* part_r,
                         int nr, double tol)
{
  if (ps->done) return;
  __shared__ double s2, rsq;
  ordered_block_sum<1>(part_s, ns, &s2);
  ordered_block_sum<1>(part_r, nr, &rsq);
  if (threadIdx.x == 0) {
    ps->s2    = s2;
    ps->resid = sqrt(rsq);
    ps->iters += 1;
    if (ps->resid < tol) ps->done = 1;
  }
}

// The power iteration of a small LP in one thread-block cluster of C blocks of kBlock threads, all
// steps up to convergence (or max_iters) in one launch.  Every block keeps full copies of z, q and
// A^T q in its shared memory: the vector steps (normalisation, residual, and their sums) run on
// the local copies in every block at once, the two sweeps are split over the blocks (virtual
// blocks rank, rank + C, ...) and send each new entry of A^T q and z, and each q . z block
// partial, to every block's copy through distributed shared memory, so a step needs two cluster
// barriers.  Every sum is formed exactly as in the multi-kernel form: the vector steps emulate
// its pg blocks of kBlock threads (grid stride pg * kBlock, one block reduction each), the sweeps
// are its virtual blocks, and every scalar is ordered_block_sum of the same block partials, so
// both forms give the same step size bit for bit.
template <typename TX>
struct cluster_atq_epi {  // (A^T q)_j to every block's copy
  static constexpr int kRed = 0;
  dsmem_sink<double> sink;
  struct pre_t {};
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int) const { return pre_t{}; }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t&, red_t<0>&) const
  {
    sink(j, acc);
  }
};
struct cluster_z_epi {  // z_i = (A atq)_i to every block's copy; q . z block partial
  static constexpr int kRed = 1;
  dsmem_sink<double> sink;
  const double* q;  // this block's copy of q
  struct pre_t {
    double q;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{q[i]}; }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<1>& r) const
  {
    sink(i, acc);
    r.v[0] += p.q * acc;
  }
};

// Largest m (constraints) the cluster power iteration takes: its vector steps run pg = m / kBlock
// emulated block reductions in every block.
constexpr int kClusterPowerMaxRows = 8192;

// Dynamic shared memory (doubles): z (m_pad), q (m_pad), A^T q (n_pad), the q . z partials of the
// sweep's ga virtual blocks (ga_pad, a copy in every block), their local staging (ga_pad), and
// the |z|^2 and residual partials of the pg emulated blocks (pg_pad each, local).
inline size_t cluster_power_smem(int m, int n, int pg, int ga)
{
  auto pad = [](int v) { return (size_t)((v + 15) & ~15); };
  return (2 * pad(m) + pad(n) + 2 * pad(ga) + 2 * pad(pg)) * sizeof(double);
}

// ordered_block_sum<1> of nb <= 32 partials, formed by warp 0: each thread's compensated sum of a
// single partial is that partial, and the block tree's levels above 16 only add zeros, so the
// warp's shuffle tree of the same pairs gives the same value.  Result in *out for the block.
__device__ __forceinline__ void small_ordered_sum(const double* p, int nb, double* out)
{
  if (threadIdx.x < kWarp) {
    double v = (int)threadIdx.x < nb ? p[threadIdx.x] : 0.0;
#pragma unroll
    for (int h = 16; h > 0; h >>= 1) v += __shfl_down_sync(0xffffffffu, v, h);
    if (threadIdx.x == 0) *out = v;
  }
  __syncthreads();
}

// Largest emulated block count of the cluster power iteration's vector steps and sums, and the
// largest number of virtual blocks of one sweep that one block of the cluster takes.
constexpr int kClusterPowerMaxBlocks = 32;
constexpr int kClusterPowerMaxOwn    = 16;

// Element range [lo, hi) of virtual block vb (8 warps) of a sweep's matrix: its long rows, or its
// slices, are contiguous in the matrix's arrays.
template <typename TX>
__device__ __forceinline__ void vb_range(const dev_sell<TX>& M, int vb, int64_t& lo, int64_t& hi)
{
  const int lb = long_blocks(M.long_count());
  if (vb < lb) {
    const int q0 = vb * kWarpsPerBlock, q1 = min(q0 + kWarpsPerBlock, M.long_count());
    lo           = M.long_off[q0];
    hi           = M.long_off[q1];
  } else {
    const int s0 = (vb - lb) * kWarpsPerBlock, s1 = min(s0 + kWarpsPerBlock, M.slice_count());
    lo           = M.slice_off[s0];
    hi           = M.slice_off[s1];
  }
}

// With `cache`, each block first copies the values and indices of its own virtual blocks of both
// sweeps into shared memory after the vectors (each range 16-byte aligned) and reads them there.
template <typename TX>
__global__ void __launch_bounds__(kBlock)
  cluster_power_kernel(const dev_sell<TX> AT, const dev_sell<TX> A, const double* z0, int m, int n,
                       int pg, int gt, int ga, power_state* ps, double tol, int max_iters,
                       int cache)
{
  extern __shared__ __align__(16) unsigned char cp_smem[];
  auto pad     = [](int v) { return (v + 15) & ~15; };
  double* zc   = reinterpret_cast<double*>(cp_smem);
  double* qc   = zc + pad(m);
  double* atqc = qc + pad(m);
  double* sc   = atqc + pad(n);  // q . z partials (every block's copy)
  double* st   = sc + pad(ga);   // this block's partials before they are sent
  double* pz   = st + pad(ga);   // |z|^2 partials
  double* pr   = pz + pad(pg);   // residual partials
  __shared__ double scalar;
  const unsigned rank = cluster_rank(), C = cluster_size();
  const int lane = threadIdx.x & (kWarp - 1), warp = threadIdx.x / kWarp;
  const dsmem_sink<double> to_z{(unsigned)__cvta_generic_to_shared(zc), C};
  const dsmem_sink<double> to_atq{(unsigned)__cvta_generic_to_shared(atqc), C};
  const unsigned sc_addr = (unsigned)__cvta_generic_to_shared(sc);

  for (int i = threadIdx.x; i < m; i += kBlock) zc[i] = z0[i];
  // The matrix copy: per sweep (0: A^T, 1: A) and own virtual block k, the range's start and the
  // byte offsets of its values and indices in the copy.
  __shared__ long long own_lo[2][kClusterPowerMaxOwn];
  __shared__ unsigned own_val[2][kClusterPowerMaxOwn], own_idx[2][kClusterPowerMaxOwn];
  unsigned char* mat = reinterpret_cast<unsigned char*>(pr + pad(pg));
  if (cache) {
    unsigned used = 0;
    for (int w = 0; w < 2; ++w) {
      const dev_sell<TX>& M = w == 0 ? AT : A;
      const int g           = w == 0 ? gt : ga;
      int k                 = 0;
      for (int vb = (int)rank; vb < g; vb += (int)C, ++k) {
        int64_t lo, hi;
        vb_range(M, vb, lo, hi);
        const unsigned vbytes = (unsigned)(((hi - lo) * (int64_t)sizeof(TX) + 15) & ~15);
        const unsigned ibytes = (unsigned)(((hi - lo) * (int64_t)sizeof(int) + 15) & ~15);
        TX* dv                = reinterpret_cast<TX*>(mat + used);
        int* di               = reinterpret_cast<int*>(mat + used + vbytes);
        for (int64_t e = lo + threadIdx.x; e < hi; e += kBlock) {
          dv[e - lo] = M.val[e];
          di[e - lo] = M.idx[e];
        }
        if (threadIdx.x == 0) {
          own_lo[w][k]  = lo;
          own_val[w][k] = used;
          own_idx[w][k] = used + vbytes;
        }
        used += vbytes + ibytes;
      }
    }
  }
  __syncthreads();
  // Sweep w's virtual block vb (the k-th of this block) from the copy or from global memory.
  auto sweep = [&](int w, int vb, int k, const double* gv, auto epi, double* partials) {
    const dev_sell<TX>& M = w == 0 ? AT : A;
    if (cache) {
      dev_sell<TX> V = M;
      V.val          = reinterpret_cast<const TX*>(mat + own_val[w][k]);
      V.idx          = reinterpret_cast<const int*>(mat + own_idx[w][k]);
      sell_map_block<TX, double, decltype(epi), false, kWarpsPerBlock, shared_matrix>(
        V, gv, epi, partials, vb, shared_matrix{own_lo[w][k]});
    } else {
      sell_map_block<TX, double, decltype(epi)>(M, gv, epi, partials, vb);
    }
  };
  // An emulated block's partial is formed by one warp: for each of the block's 8 warps w, the
  // warp's lanes take the sums of threads 32 w + lane, warp_sum pairs them as warp w's own
  // warp_sum would, and the 8 results are added in order from 0.0 (block_reduce_store's two
  // stages).  Warp k of this block forms the partials of emulated blocks k, k + 8, ...
  // |z|^2 partials of the pg emulated blocks (vec_reduce_kernel<0>).
  auto sumsq = [&]() {
    for (int b = warp; b < pg; b += kWarpsPerBlock) {
      double s = 0.0;
      for (int w = 0; w < kWarpsPerBlock; ++w) {
        double r = 0.0;
        for (int i = b * kBlock + w * kWarp + lane; i < m; i += pg * kBlock) {
          const double v = zc[i];
          r += v * v;
        }
        s += warp_sum(r);
      }
      if (lane == 0) pz[b] = s;
    }
    __syncthreads();
  };
  sumsq();
  // Every block of the cluster is running before any block stores into another's memory.
  cluster_barrier();
  int it = 0, done = 0;
  double nq = 0.0, s2 = 0.0, resid = 0.0;
  while (it < max_iters && !done) {
    // q = z / |z|  (power_normalize_sum_kernel), on the local copies.
    small_ordered_sum(pz, pg, &scalar);
    nq = sqrt(scalar);
    for (int i = threadIdx.x; i < m; i += kBlock) qc[i] = zc[i] / nq;
    __syncthreads();
    // A^T q over this block's virtual blocks, entries sent to every copy.
    for (int vb = (int)rank, k = 0; vb < gt; vb += (int)C, ++k)
      sweep(0, vb, k, qc, cluster_atq_epi<TX>{to_atq}, nullptr);
    cluster_barrier();
    // z = A (A^T q) with the q . z partial of each virtual block, both sent to every copy.
    for (int vb = (int)rank, k = 0; vb < ga; vb += (int)C, ++k) {
      sweep(1, vb, k, atqc, cluster_z_epi{to_z, qc}, st);
      if (threadIdx.x == 0)
        for (unsigned c = 0; c < C; ++c)
          dsmem_store(sc_addr + (unsigned)vb * (unsigned)sizeof(double), c, st[vb]);
    }
    cluster_barrier();
    // q <- q (-s2) + z with its squares' partials (power_residual_sum_kernel) and the next |z|^2
    // partials, then the test of power_check_sum_kernel, all on the local copies.
    small_ordered_sum(sc, ga, &scalar);
    s2 = scalar;
    for (int b = warp; b < pg; b += kWarpsPerBlock) {
      double sr = 0.0, sz = 0.0;
      for (int w = 0; w < kWarpsPerBlock; ++w) {
        double rr = 0.0, rz = 0.0;
        for (int i = b * kBlock + w * kWarp + lane; i < m; i += pg * kBlock) {
          const double zi = zc[i];
          const double v  = qc[i] * -s2 + zi;
          qc[i]           = v;
          rr += v * v;
          rz += zi * zi;
        }
        sr += warp_sum(rr);
        sz += warp_sum(rz);
      }
      if (lane == 0) {
        pr[b] = sr;
        pz[b] = sz;
      }
    }
    __syncthreads();
    small_ordered_sum(pr, pg, &scalar);
    resid = sqrt(scalar);
    ++it;
    done = resid < tol;
  }
  if (rank == 0 && threadIdx.x == 0) {
    ps->norm_z = nq;
    ps->s2     = s2;
    ps->resid  = resid;
    ps->iters  = it;
    ps->done   = done;
  }
  // No block leaves while another may still store into its shared memory.
  cluster_barrier();
}


// Golub-Kahan-Lanczos bidiagonalisation of the scaled A (the mixed-precision step size).  The
// vectors are stored unnormalised; gk_state holds their norms: u has norm beta (beta_k), v has
// norm alpha (alpha_{k-1}, or 0 before the first step).
struct gk_state {
  double beta;
  double alpha;
};

// Row j of A^T applied to u:  p_j = (A^T u)_j / beta - beta v_j / alpha  (written over v_j).
struct gk_primal_epi {
  static constexpr int kRed = 1;
  double* v;
  const gk_state* st;
  struct pre_t {
    double v;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int j) const { return pre_t{v[j]}; }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<1>& r) const
  {
    const double b = st->beta, a = st->alpha;
    const double pj = acc / b - (a > 0.0 ? b * (p.v / a) : 0.0);
    v[j]            = pj;
    r.v[0] += pj * pj;
  }
};

// Row i of A applied to v:  q_i = (A v)_i / alpha - alpha u_i / beta  (written over u_i).
struct gk_dual_epi {
  static constexpr int kRed = 1;
  double* u;
  const gk_state* st;
  struct pre_t {
    double u;
  };
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{u[i]}; }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<1>& r) const
  {
    const double a = st->alpha, b = st->beta;
    const double qi = acc / a - a * (p.u / b);
    u[i]            = qi;
    r.v[0] += qi * qi;
  }
};

// Records a new norm: FIELD 0 sets alpha (history alphas[k]), FIELD 1 sets beta (betas[k + 1]).
template <int FIELD>
static __global__ void gk_record_kernel(gk_state* st, const double* sumsq, double* hist, int k)
{
  const double v = sqrt(*sumsq);
  if (FIELD == 0) {
    st->alpha = v;
    hist[k]   = v;
  } else {
    st->beta    = v;
    hist[k + 1] = v;
  }
}

// ---------------------------------------------------------------------------------------------
// Scaling (reference initial_scaling.cu:152-569).

// For every row r of layout A: out[r] = max_k |v (s_first) (s_second)| (MODE 0) or
// sum_k |v s_first s_second|^alpha (MODE 1), where for A (TRANSPOSED=false) the product is
// (a_ij dr_i) dc_j and for A^T (TRANSPOSED=true) it is (a_ij dr_i) dc_j with i = idx, j = row.
template <int MODE, bool TRANSPOSED>
__global__ void __launch_bounds__(kBlock) row_scaled_abs_kernel(const dev_sell<double> A,
                                                                const double* dr,
                                                                const double* dc, double alpha,
                                                                double* out)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lb   = long_blocks(A.n_long);
  auto term      = [&](double v, int row, int col) {
    const double p = TRANSPOSED ? (v * dr[col]) * dc[row] : (v * dr[row]) * dc[col];
    const double a = fabs(p);
    return MODE == 0 ? a : pow(a, alpha);
  };
  if ((int)blockIdx.x < lb) {
    const int row = blockIdx.x * kWarpsPerBlock + warp;
    if (row < A.n_long) {
      double acc = 0.0;
      for (int64_t k = A.long_off[row] + lane; k < A.long_off[row + 1]; k += kWarp) {
        const double t = term(A.val[k], row, A.idx[k]);
        acc            = MODE == 0 ? fmax(acc, t) : acc + t;
      }
      acc = MODE == 0 ? warp_max(acc) : warp_sum(acc);
      if (lane == 0) out[row] = acc;
    }
  } else {
    const int s = (blockIdx.x - lb) * kWarpsPerBlock + warp;
    if (s < A.n_slices) {
      const int64_t base = A.slice_off[s];
      const int len      = (int)((A.slice_off[s + 1] - base) >> 5);
      const int row      = A.n_long + s * kWarp + lane;
      if (row < A.rows) {
        double acc = 0.0;
          for (int k = 0; k < len; ++k) {
          const int64_t p = sell_pos(base, k, lane);
          const double v  = A.val[p];
          if (v == 0.0) continue;  // padding (and explicit zeros, which contribute nothing)
          const double t = term(v, row, A.idx[p]);
          acc            = MODE == 0 ? fmax(acc, t) : acc + t;
        }
        out[row] = acc;
      }
    }
  }
}

// d[i] <- d[i] / sqrt(v[i]) where v[i] > 0 (a_divides_sqrt_b_bounded, utils.cuh:156-163)
static __global__ void apply_root_scaling_kernel(double* d, const double* v, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double b = v[i];
    if (b > 0.0) d[i] = d[i] / sqrt(b);
  }
}

// Scaled copy of the matrix values: A_s = (a dr_i) dc_j, A^T_s = (a dc_j) dr_i.
template <typename TM, bool TRANSPOSED>
__global__ void __launch_bounds__(kBlock) scale_values_kernel(const dev_sell<double> A,
                                                              const double* dr, const double* dc,
                                                              TM* out)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lb   = long_blocks(A.n_long);
  auto scaled    = [&](double v, int row, int col) {
    return TRANSPOSED ? (v * dc[row]) * dr[col] : (v * dr[row]) * dc[col];
  };
  if ((int)blockIdx.x < lb) {
    const int row = blockIdx.x * kWarpsPerBlock + warp;
    if (row < A.n_long)
      for (int64_t k = A.long_off[row] + lane; k < A.long_off[row + 1]; k += kWarp)
        out[k] = (TM)scaled(A.val[k], row, A.idx[k]);
  } else {
    const int s = (blockIdx.x - lb) * kWarpsPerBlock + warp;
    if (s < A.n_slices) {
      const int64_t base = A.slice_off[s];
      const int len      = (int)((A.slice_off[s + 1] - base) >> 5);
      const int row      = A.n_long + s * kWarp + lane;
      for (int k = 0; k < len; ++k) {
        const int64_t p = sell_pos(base, k, lane);
        out[p]          = row < A.rows ? (TM)scaled(A.val[p], row, A.idx[p]) : (TM)0;
      }
    }
  }
}

// First pass of the vector scaling: c*dc, bounds/dc (divide_check_zero), constraint bounds*dr.
static __global__ void scale_vectors_kernel(const double* c, const double* l, const double* u,
                                     const double* lc, const double* uc, const double* dc,
                                     const double* dr, int n, int m, double* cs, double* ls,
                                     double* us, double* lcs, double* ucs)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      const double d = dc[i];
      cs[i]          = c[i] * d;
      if (d == 0.0) {
        ls[i] = 0.0;
        us[i] = 0.0;
      } else {
        ls[i] = l[i] / d;
        us[i] = u[i] / d;
      }
    } else {
      const int r = i - n;
      lcs[r]      = lc[r] * dr[r];
      ucs[r]      = uc[r] * dr[r];
    }
  }
}

// Second pass: bound rescaling beta and objective rescaling gamma; converts to the iterate type.
template <typename TX>
__global__ void rescale_vectors_kernel(const double* cs, const double* ls, const double* us,
                                       const double* lcs, const double* ucs, double beta,
                                       double gamma, int n, int m, TX* c_out, TX* l_out, TX* u_out,
                                       TX* lc_out, TX* uc_out)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      c_out[i] = (TX)(cs[i] * gamma);
      l_out[i] = (TX)(ls[i] * beta);
      u_out[i] = (TX)(us[i] * beta);
    } else {
      const int r = i - n;
      lc_out[r]   = (TX)(lcs[r] * beta);
      uc_out[r]   = (TX)(ucs[r] * beta);
    }
  }
}

// Initial iterate in scaled space: v / d (d != 0) times factor, written to three buffers
// (scale_solutions, initial_scaling.cu:571-640).
template <typename TX>
__global__ void scale_initial_kernel(const double* v, const double* d, double factor, int n, TX* a,
                                     TX* b, TX* c)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double s = d[i] != 0.0 ? v[i] / d[i] : v[i];
    const TX w     = (TX)(s * factor);
    a[i]           = w;
    b[i]           = w;
    c[i]           = w;
  }
}

// ---------------------------------------------------------------------------------------------
// Infeasibility detection (reference infeasibility_information.cu:230-490, the cuPDLPx branch).
// The rays are the step's deltas x_bar - x and y_bar - y in the scaled space, clamped to the
// recession cones of the bounds.

// d_j = clamp(x_bar_j - x_j) (>= 0 on a finite lower bound, <= 0 on a finite upper bound) and
// cd_j = c_j d_j;  e_i = clamp(y_bar_i - y_i) (<= 0 without a finite lower bound, >= 0 without a
// finite upper bound) and pe_i = max(e_i, 0) fin(lc_i) + min(e_i, 0) fin(uc_i).
template <typename TX>
__global__ void ray_vectors_kernel(const TX* x, const TX* xbar, const TX* l, const TX* u,
                                   const TX* c, int n, const TX* y, const TX* ybar, const TX* lc,
                                   const TX* uc, int m, double* d, double* cd, double* e,
                                   double* pe)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      double v = (double)xbar[i] - (double)x[i];
      if (isfinite((double)l[i])) v = fmax(v, 0.0);
      if (isfinite((double)u[i])) v = fmin(v, 0.0);
      d[i]  = v;
      cd[i] = (double)c[i] * v;
    } else {
      const int r = i - n;
      double v    = (double)ybar[r] - (double)y[r];
      if (!isfinite((double)lc[r])) v = fmin(v, 0.0);
      if (!isfinite((double)uc[r])) v = fmax(v, 0.0);
      e[r]  = v;
      pe[r] = fmax(v, 0.0) * finite_or_zero((double)lc[r]) + fmin(v, 0.0) * finite_or_zero((double)uc[r]);
    }
  }
}

// Row i of A applied to d: violation of the primal ray, (max(-Ad, 0) [lc finite] +
// max(Ad, 0) [uc finite]) dr_i with Ad scaled by 1 / |d|_inf.
template <typename TX>
struct ray_primal_epi {
  static constexpr int kRed = 0;
  const TX* lc;
  const TX* uc;
  const double* dr;
  double inv_norm;
  double* out;
  struct pre_t {};
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int) const { return pre_t{}; }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t&, red_t<0>&) const
  {
    const double ad = acc * inv_norm;
    out[i]          = (fmax(-ad, 0.0) * (isfinite((double)lc[i]) ? 1.0 : 0.0) +
              fmax(ad, 0.0) * (isfinite((double)uc[i]) ? 1.0 : 0.0)) *
             dr[i];
  }
};

// Row j of A^T applied to e (g = (A^T e)_j): dual-slack objective term and dual-ray violation.
template <typename TX>
struct ray_dual_epi {
  static constexpr int kRed = 0;
  const TX* l;
  const TX* u;
  const double* dc;
  double* slack_term;
  double* violation;
  struct pre_t {};
  __device__ bool skip() const { return false; }
  __device__ __forceinline__ pre_t load(int) const { return pre_t{}; }
  __device__ __forceinline__ void operator()(int j, double g, const pre_t&, red_t<0>&) const
  {
    const double lj = (double)l[j], uj = (double)u[j];
    slack_term[j] = fmax(-g, 0.0) * finite_or_zero(lj) + fmin(-g, 0.0) * finite_or_zero(uj);
    violation[j]  = (fmax(-g, 0.0) * (isfinite(lj) ? 0.0 : 1.0) -
                    fmin(-g, 0.0) * (isfinite(uj) ? 0.0 : 1.0)) *
                   dc[j];
  }
};

// Per-block sum (MAX = false) or maximum of |a| (MAX = true) into partials[blockIdx.x].
template <bool MAX>
__global__ void __launch_bounds__(kBlock) block_stat_kernel(const double* a, int n, double* partials)
{
  __shared__ double sm[kBlock];
  double v = 0.0;
  for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock)
    v = MAX ? fmax(v, fabs(a[i])) : v + a[i];
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int h = kBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      sm[threadIdx.x] = MAX ? fmax(sm[threadIdx.x], sm[threadIdx.x + h])
                            : sm[threadIdx.x] + sm[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) partials[blockIdx.x] = sm[0];
}

// Elementwise helpers
template <typename TX>
__global__ void clamp_kernel(TX* x, const TX* l, const TX* u, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = (TX)fmin(fmax((double)x[i], (double)l[i]), (double)u[i]);
}

template <typename TA, typename TB>
__global__ void copy_convert_kernel(TB* dst, const TA* src, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    dst[i] = (TB)src[i];
}

}  // namespace cuopt_b200
