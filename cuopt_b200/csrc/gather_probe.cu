// Measurement hook: the random-gather request ceiling of one B200.
//
// The fused PDHG sweeps read the matrix as a coalesced stream and gather one iterate element per
// stored non-zero at a random column.  On uniformly random sparsity every gather is its own L1
// request and L2 sector, so the sweeps are bound by the rate at which the SMs can issue such
// requests, not by HBM.  This probe measures that rate on the sweep's own access pattern with
// nothing else in the kernel: warps stream int4 index chunks with evict-first loads (as the
// sliced-ELL sweeps do) and gather the four elements each chunk names from a vector that stays in
// L2, CHUNKS chunks in flight per thread.  The returned rate (gathers per second) is the
// denominator of the sweeps' gather roofline.
#include <cuopt_b200.h>

#include <cstdio>

#include "common.cuh"

namespace cuopt_b200 {
namespace {

constexpr int kProbeBlock = 256;

// Deterministic pseudo-random indices in [0, n) (splitmix64 of the position).
__global__ void probe_fill_kernel(int* idx, int64_t count, int n, uint64_t seed)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count;
       i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t z = seed + 0x9E3779B97F4A7C15ull * (uint64_t)(i + 1);
    z          = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z          = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    idx[i] = (int)(z % (uint64_t)n);
  }
}

template <typename T>
__global__ void probe_fill_vec_kernel(T* v, int n)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    v[i] = (T)(1.0 + 1e-7 * (i & 1023));
}

// Warp w of the grid owns chunk rows w, w + W, ...; a chunk row is 32 lanes x 4 indices
// (512 contiguous bytes), the sliced-ELL chunk shape.  Each thread keeps CHUNKS chunks in flight.
template <typename T, int CHUNKS>
__global__ void __launch_bounds__(kProbeBlock)
  probe_gather_kernel(const int* __restrict__ idx, int64_t rows, const T* __restrict__ g,
                      double* __restrict__ sink)
{
  const int lane   = threadIdx.x & 31;
  const int64_t w  = (blockIdx.x * (int64_t)kProbeBlock + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kProbeBlock) >> 5;
  double acc       = 0.0;
  for (int64_t r = w * CHUNKS; r < rows; r += nw * CHUNKS) {
    int4 ix[CHUNKS];
#pragma unroll
    for (int c = 0; c < CHUNKS; ++c)
      ix[c] = r + c < rows ? __ldcs(reinterpret_cast<const int4*>(idx + ((r + c) * 32 + lane) * 4))
                           : make_int4(0, 0, 0, 0);
    T v[CHUNKS][4];
#pragma unroll
    for (int c = 0; c < CHUNKS; ++c) {
      v[c][0] = g[ix[c].x];
      v[c][1] = g[ix[c].y];
      v[c][2] = g[ix[c].z];
      v[c][3] = g[ix[c].w];
    }
#pragma unroll
    for (int c = 0; c < CHUNKS; ++c)
      acc += (double)v[c][0] + (double)v[c][1] + (double)v[c][2] + (double)v[c][3];
  }
  acc = warp_sum(acc);
  if (lane == 0) sink[w] = acc;
}

// The scatter counterpart: each gathered index instead receives an atomic add (the result is not
// used, so it compiles to a fire-and-forget reduction).
template <typename T, int CHUNKS>
__global__ void __launch_bounds__(kProbeBlock)
  probe_scatter_kernel(const int* __restrict__ idx, int64_t rows, T* __restrict__ g,
                       double* __restrict__ sink)
{
  const int lane   = threadIdx.x & 31;
  const int64_t w  = (blockIdx.x * (int64_t)kProbeBlock + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * kProbeBlock) >> 5;
  for (int64_t r = w * CHUNKS; r < rows; r += nw * CHUNKS) {
    int4 ix[CHUNKS];
#pragma unroll
    for (int c = 0; c < CHUNKS; ++c)
      ix[c] = r + c < rows ? __ldcs(reinterpret_cast<const int4*>(idx + ((r + c) * 32 + lane) * 4))
                           : make_int4(0, 0, 0, 0);
#pragma unroll
    for (int c = 0; c < CHUNKS; ++c) {
      if (r + c >= rows) continue;
      atomicAdd(g + ix[c].x, (T)1);
      atomicAdd(g + ix[c].y, (T)1);
      atomicAdd(g + ix[c].z, (T)1);
      atomicAdd(g + ix[c].w, (T)1);
    }
  }
  (void)lane;
  (void)sink;
}

template <typename T, int CHUNKS>
float time_probe(const int* idx, int64_t rows, const T* g, double* sink, int grid, cudaStream_t s,
                 int repeats)
{
  cudaEvent_t a, b;
  B200_CUDA_CHECK(cudaEventCreate(&a));
  B200_CUDA_CHECK(cudaEventCreate(&b));
  for (int i = 0; i < 3; ++i)
    probe_gather_kernel<T, CHUNKS><<<grid, kProbeBlock, 0, s>>>(idx, rows, g, sink);
  B200_LAUNCH_CHECK();
  B200_CUDA_CHECK(cudaEventRecord(a, s));
  for (int i = 0; i < repeats; ++i)
    probe_gather_kernel<T, CHUNKS><<<grid, kProbeBlock, 0, s>>>(idx, rows, g, sink);
  B200_CUDA_CHECK(cudaEventRecord(b, s));
  B200_CUDA_CHECK(cudaEventSynchronize(b));
  float ms = 0.f;
  B200_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / repeats;
}

template <typename T, int CHUNKS>
float time_scatter(const int* idx, int64_t rows, T* g, double* sink, int grid, cudaStream_t s,
                   int repeats)
{
  cudaEvent_t a, b;
  B200_CUDA_CHECK(cudaEventCreate(&a));
  B200_CUDA_CHECK(cudaEventCreate(&b));
  for (int i = 0; i < 3; ++i)
    probe_scatter_kernel<T, CHUNKS><<<grid, kProbeBlock, 0, s>>>(idx, rows, g, sink);
  B200_LAUNCH_CHECK();
  B200_CUDA_CHECK(cudaEventRecord(a, s));
  for (int i = 0; i < repeats; ++i)
    probe_scatter_kernel<T, CHUNKS><<<grid, kProbeBlock, 0, s>>>(idx, rows, g, sink);
  B200_CUDA_CHECK(cudaEventRecord(b, s));
  B200_CUDA_CHECK(cudaEventSynchronize(b));
  float ms = 0.f;
  B200_CUDA_CHECK(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / repeats;
}

template <typename T>
double best_scatter_rate(const int* idx, int64_t rows, T* g, double* sink, int grid,
                         cudaStream_t s, int repeats, int* best_chunks)
{
  const double n = (double)rows * 128.0;
  double best    = 0.0;
  const float t[3] = {time_scatter<T, 1>(idx, rows, g, sink, grid, s, repeats),
                      time_scatter<T, 2>(idx, rows, g, sink, grid, s, repeats),
                      time_scatter<T, 4>(idx, rows, g, sink, grid, s, repeats)};
  for (int k = 0; k < 3; ++k) {
    const double rate = n / (t[k] * 1e-3);
    if (rate > best) {
      best         = rate;
      *best_chunks = 1 << k;
    }
  }
  return best;
}

template <typename T>
double best_rate(const int* idx, int64_t rows, const T* g, double* sink, int grid, cudaStream_t s,
                 int repeats, int* best_chunks)
{
  const double gathers = (double)rows * 128.0;
  double best          = 0.0;
  const float t[4]     = {time_probe<T, 1>(idx, rows, g, sink, grid, s, repeats),
                          time_probe<T, 2>(idx, rows, g, sink, grid, s, repeats),
                          time_probe<T, 4>(idx, rows, g, sink, grid, s, repeats),
                          time_probe<T, 8>(idx, rows, g, sink, grid, s, repeats)};
  for (int k = 0; k < 4; ++k) {
    const double rate = gathers / (t[k] * 1e-3);
    if (rate > best) {
      best         = rate;
      *best_chunks = 1 << k;
    }
  }
  return best;
}

}  // namespace
}  // namespace cuopt_b200

extern "C" cuopt_int_t cuOptProfileGatherRate(cuopt_int_t vector_length, int64_t gathers,
                                              cuopt_int_t element_bytes, void* stream,
                                              cuopt_float_t* gathers_per_second,
                                              cuopt_int_t* chunks_in_flight)
{
  using namespace cuopt_b200;
  if (vector_length <= 0 || gathers < 128 || !gathers_per_second || !chunks_in_flight ||
      (element_bytes != 4 && element_bytes != 8))
    return CUOPT_INVALID_ARGUMENT;
  try {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t rows = gathers / 128;
    const int grid     = sms * 8;
    alloc_scope scope(s);
    dbuf<int> idx((size_t)rows * 128);
    dbuf<double> sink((size_t)grid * (kProbeBlock / 32));
    probe_fill_kernel<<<sms * 8, kProbeBlock, 0, s>>>(idx.data(), rows * 128, vector_length,
                                                       0x5eedull);
    B200_LAUNCH_CHECK();
    if (element_bytes == 4) {
      dbuf<float> g(vector_length);
      probe_fill_vec_kernel<float><<<sms * 4, kProbeBlock, 0, s>>>(g.data(), vector_length);
      *gathers_per_second = best_rate<float>(idx.data(), rows, g.data(), sink.data(), grid, s, 10,
                                             chunks_in_flight);
    } else {
      dbuf<double> g(vector_length);
      probe_fill_vec_kernel<double><<<sms * 4, kProbeBlock, 0, s>>>(g.data(), vector_length);
      *gathers_per_second = best_rate<double>(idx.data(), rows, g.data(), sink.data(), grid, s, 10,
                                              chunks_in_flight);
    }
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptProfileGatherRate: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}

extern "C" cuopt_int_t cuOptProfileScatterRate(cuopt_int_t vector_length, int64_t scatters,
                                               cuopt_int_t element_bytes, void* stream,
                                               cuopt_float_t* scatters_per_second,
                                               cuopt_int_t* chunks_in_flight)
{
  using namespace cuopt_b200;
  if (vector_length <= 0 || scatters < 128 || !scatters_per_second || !chunks_in_flight ||
      (element_bytes != 4 && element_bytes != 8))
    return CUOPT_INVALID_ARGUMENT;
  try {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 148;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t rows = scatters / 128;
    const int grid     = sms * 8;
    alloc_scope scope(s);
    dbuf<int> idx((size_t)rows * 128);
    dbuf<double> sink((size_t)grid * (kProbeBlock / 32));
    probe_fill_kernel<<<sms * 8, kProbeBlock, 0, s>>>(idx.data(), rows * 128, vector_length,
                                                       0x5eedull);
    B200_LAUNCH_CHECK();
    if (element_bytes == 4) {
      dbuf<float> g(vector_length);
      g.zero(s);
      *scatters_per_second = best_scatter_rate<float>(idx.data(), rows, g.data(), sink.data(),
                                                      grid, s, 10, chunks_in_flight);
    } else {
      dbuf<double> g(vector_length);
      g.zero(s);
      *scatters_per_second = best_scatter_rate<double>(idx.data(), rows, g.data(), sink.data(),
                                                       grid, s, 10, chunks_in_flight);
    }
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptProfileScatterRate: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}
