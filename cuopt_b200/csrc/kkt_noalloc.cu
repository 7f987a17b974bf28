// KKT error evaluation of a given LP point without any device allocation.
//
// Computes, for (x, y, reduced costs) of an LP held in device memory in the user's CSR order, the
// same quantities the solver reports for its own solution (the reference's
// convergence_information_t::compute_convergence_information, cpp/src/pdlp/termination_strategy/
// convergence_information.cu:327-489, restated by evaluate_unscaled in pdlp_engine.cu):
//   l2 primal residual  |A x - clamp(A x, lc, uc)|_2
//   l2 dual residual    |c - A^T y - rc|_2
//   primal / dual objective, gap, and the three relative errors.
//
// Who needs it: callers that must check a candidate point while they may not allocate device
// memory — a process whose memory pool is already fully reserved by a larger solve or by another
// framework's caching allocator (where a foreign cudaMalloc fails or fragments the pool), and
// latency-bound loops (heuristics testing many candidate points) where cudaMalloc / cudaFree would
// add an implicit device synchronisation on every call.  The solver's own evaluation builds a
// relabelled matrix layout and per-solve buffers; this variant reads the user's CSR directly and
// keeps its scratch in fixed-size device globals instead:
//   g_na_aty      A^T y accumulator, kNaMaxCols doubles (4 MiB): bounds num_variables;
//                 must be zero before the row pass (cleared by a memset on every call);
//   g_na_partials per-block partial sums of the two passes, written in full before they are read;
//   g_na_bad      count of malformed entries (column indices outside [0, n), rows whose offsets
//                 decrease or start below 0); must be zero before the row pass (cleared on every
//                 call).
// Because the scratch is one static copy per device, calls that overlap in time on the same
// device (different streams or host threads without ordering between them) race on it and give
// wrong results; callers must order them.  A^T y is accumulated with double-precision atomics, so
// the dual residual and the quantities derived from it may differ in the last bits between calls.
// The scratch belongs to this library's device code, which the CUDA runtime loads on a device at
// the first call that needs it (lazily, by default): that first call is when the static arrays take
// their device memory.
#include <math_constants.h>

#include <cstdio>

#include <cuopt_b200.h>

#include "common.cuh"

namespace cuopt_b200 {
namespace {

constexpr int kBlock         = 256;
constexpr int kWarpsPerBlock = kBlock / kWarp;
constexpr int kNaMaxCols     = 1 << 19;  // 524,288 columns
constexpr int kNaBlocks  = 592;      // 148 SMs x 4 resident blocks; fixed so partials fit
constexpr int kNaRowRed  = 3;        // row pass: |r_p|^2, dual row term, |b|^2
constexpr int kNaColRed  = 4;        // column pass: |r_d|^2, c.x, rc.x, |c|^2

static __device__ __align__(256) double g_na_aty[kNaMaxCols];
static __device__ __align__(256) double g_na_partials[kNaBlocks * (kNaRowRed + kNaColRed)];
static __device__ __align__(256) unsigned int g_na_bad;

struct na_scratch {
  double* aty;
  double* partials;
  unsigned int* bad;
};

__device__ __forceinline__ double fin0(double v) { return isfinite(v) ? v : 0.0; }

// Block sum of K per-thread values (fixed order); thread q < K writes partials[blockIdx.x*K + q].
template <int K>
__device__ __forceinline__ void block_sum_store(const double (&v)[K], double* partials)
{
  __shared__ double sm[kWarpsPerBlock][K];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const double w = warp_sum(v[q]);
    if (lane == 0) sm[warp][q] = w;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kWarpsPerBlock; ++w) t += sm[w][threadIdx.x];
    partials[(size_t)blockIdx.x * K + threadIdx.x] = t;
  }
}

// Warp per constraint row: A x and the row's residual / dual-objective / |b| terms, and the
// scatter of y_i A[i, :] into the A^T y accumulator.
__global__ void __launch_bounds__(kBlock)
  na_rows_kernel(int m, int n, const int* __restrict__ off, const int* __restrict__ idx,
                 const double* __restrict__ val, const double* __restrict__ x,
                 const double* __restrict__ y, const double* __restrict__ lo,
                 const double* __restrict__ up, double sgn, na_scratch s)
{
  double r[kNaRowRed] = {};
  const int lane = threadIdx.x & 31;
  const int nw   = gridDim.x * kWarpsPerBlock;
  for (int i = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5); i < m; i += nw) {
    const int b = off[i], e = off[i + 1];
    if (b < 0 || e < b) {  // malformed offsets: counted, the row is skipped
      if (lane == 0) atomicAdd(s.bad, 1u);
      continue;
    }
    const double yi = y[i];
    double ax       = 0.0;
    for (int k = b + lane; k < e; k += kWarp) {
      const int j = idx[k];
      if ((unsigned)j >= (unsigned)n) {
        atomicAdd(s.bad, 1u);
        continue;
      }
      const double a = val[k];
      ax += a * x[j];
      atomicAdd(s.aty + j, a * yi);
    }
    ax = warp_sum(ax);
    if (lane == 0) {
      const double l = lo[i], u = up[i];
      const double rp   = ax - fmax(l, fmin(ax, u));
      const double yint = sgn * yi;  // the dual in minimisation form
      r[0] += rp * rp;
      r[1] += fmax(yint, 0.0) * fin0(l) + fmin(yint, 0.0) * fin0(u);
      r[2] += ((isfinite(l) && l != u) ? l * l : 0.0) + (isfinite(u) ? u * u : 0.0);
    }
  }
  block_sum_store<kNaRowRed>(r, s.partials);
}

// Thread per variable: dual residual and objective terms.
__global__ void __launch_bounds__(kBlock)
  na_cols_kernel(int n, const double* __restrict__ c, const double* __restrict__ x,
                 const double* __restrict__ rc, na_scratch s)
{
  double r[kNaColRed] = {};
  for (int j = blockIdx.x * kBlock + threadIdx.x; j < n; j += gridDim.x * kBlock) {
    const double cj = c[j], xj = x[j], sj = rc[j];
    const double rd = (cj - s.aty[j]) - sj;
    r[0] += rd * rd;
    r[1] += cj * xj;
    r[2] += sj * xj;
    r[3] += cj * cj;
  }
  block_sum_store<kNaColRed>(r, s.partials + kNaBlocks * kNaRowRed);
}

// One block: ordered, compensated sums over the block partials, then the reported quantities.
__global__ void __launch_bounds__(kBlock)
  na_finish_kernel(double sgn, double offset, na_scratch s, double* __restrict__ out)
{
  __shared__ double sm[kBlock];
  __shared__ double tot[kNaRowRed + kNaColRed];
  for (int q = 0; q < kNaRowRed + kNaColRed; ++q) {
    const bool row_q    = q < kNaRowRed;
    const int K         = row_q ? kNaRowRed : kNaColRed;
    const double* base  = row_q ? s.partials : s.partials + kNaBlocks * kNaRowRed;
    const int qq        = row_q ? q : q - kNaRowRed;
    ksum acc;
    for (int b = threadIdx.x; b < kNaBlocks; b += kBlock) acc.add(base[(size_t)b * K + qq]);
    sm[threadIdx.x] = acc.value();
    __syncthreads();
    for (int h = kBlock / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) sm[threadIdx.x] += sm[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) tot[q] = sm[0];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double rp2 = tot[0], drow = tot[1], b2 = tot[2];
    const double rd2 = tot[3], cx = tot[4], sx = tot[5], c2 = tot[6];
    const double l2p = sqrt(rp2), l2d = sqrt(rd2);
    const double primal = cx + offset;
    const double dual   = sgn * (drow + sgn * sx) + offset;
    const double gap    = fabs(primal - dual);
    const unsigned bad  = *s.bad;
    const double vals[8] = {l2p, l2d, primal, dual, gap, l2p / (1.0 + sqrt(b2)),
                            l2d / (1.0 + sqrt(c2)), gap / (1.0 + fabs(primal) + fabs(dual))};
    for (int q = 0; q < 8; ++q) out[q] = bad ? CUDART_NAN : vals[q];
    out[8] = (double)bad;
  }
}

// Device addresses of the static scratch on the current device.  Looked up on every call (a host
// query that allocates nothing), so that a device reset or a new primary context, after which the
// module is loaded again at new addresses, never leaves a stale address behind.
bool scratch_for_current_device(na_scratch& out, int& dev)
{
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  na_scratch s{};
  if (cudaGetSymbolAddress((void**)&s.aty, g_na_aty) != cudaSuccess) return false;
  if (cudaGetSymbolAddress((void**)&s.partials, g_na_partials) != cudaSuccess) return false;
  if (cudaGetSymbolAddress((void**)&s.bad, g_na_bad) != cudaSuccess) return false;
  out = s;
  return true;
}

}  // namespace
}  // namespace cuopt_b200

extern "C" cuopt_int_t cuOptComputeKKTErrorsNoAlloc(
  cuopt_int_t m, cuopt_int_t n, cuopt_int_t sense, cuopt_float_t offset, const cuopt_float_t* d_c,
  const cuopt_int_t* d_off, const cuopt_int_t* d_idx, const cuopt_float_t* d_val,
  const cuopt_float_t* d_lo, const cuopt_float_t* d_up, const cuopt_float_t* d_x,
  const cuopt_float_t* d_y, const cuopt_float_t* d_rc, void* stream, cuopt_float_t* d_out)
{
  using namespace cuopt_b200;
  if (!d_c || !d_off || !d_idx || !d_val || !d_lo || !d_up || !d_x || !d_y || !d_rc || !d_out)
    return CUOPT_INVALID_ARGUMENT;
  if (m <= 0 || n <= 0) return CUOPT_INVALID_ARGUMENT;
  if (sense != CUOPT_MINIMIZE && sense != CUOPT_MAXIMIZE) return CUOPT_INVALID_ARGUMENT;
  if (n > kNaMaxCols) {
    std::fprintf(stderr,
                 "cuOptComputeKKTErrorsNoAlloc: num_variables = %d exceeds the static scratch "
                 "capacity of %d variables\n",
                 (int)n, kNaMaxCols);
    return CUOPT_INVALID_ARGUMENT;
  }
  na_scratch s{};
  int dev = 0;
  if (!scratch_for_current_device(s, dev)) {
    std::fprintf(stderr, "cuOptComputeKKTErrorsNoAlloc: scratch lookup failed on device %d\n", dev);
    return CUOPT_RUNTIME_ERROR;
  }
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const double sgn      = sense == CUOPT_MAXIMIZE ? -1.0 : 1.0;
  if (cudaMemsetAsync(s.aty, 0, (size_t)n * sizeof(double), st) != cudaSuccess ||
      cudaMemsetAsync(s.bad, 0, sizeof(unsigned int), st) != cudaSuccess)
    return CUOPT_RUNTIME_ERROR;
  na_rows_kernel<<<kNaBlocks, kBlock, 0, st>>>(m, n, d_off, d_idx, d_val, d_x, d_y, d_lo, d_up, sgn,
                                               s);
  na_cols_kernel<<<kNaBlocks, kBlock, 0, st>>>(n, d_c, d_x, d_rc, s);
  na_finish_kernel<<<1, kBlock, 0, st>>>(sgn, offset, s, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "cuOptComputeKKTErrorsNoAlloc: %s\n", cudaGetErrorString(e));
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}
