// Shared device/host helpers for the cuopt_b200 PDLP library (sm_100a).
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <utility>

namespace cuopt_b200 {

// Error carried from the device side back to the C interface.
struct cuda_error : std::runtime_error {
  explicit cuda_error(const std::string& s) : std::runtime_error(s) {}
};

#define B200_CUDA_CHECK(expr)                                                                 \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess) {                                                                 \
      throw ::cuopt_b200::cuda_error(std::string("CUDA error ") + cudaGetErrorString(_e) +   \
                                     " at " + __FILE__ + ":" + std::to_string(__LINE__));    \
    }                                                                                        \
  } while (0)

#define B200_LAUNCH_CHECK() B200_CUDA_CHECK(cudaGetLastError())

constexpr int kWarp = 32;

// Stream on which device buffers are allocated and released (stream-ordered allocator).  Solver
// entry points set it for their duration with alloc_scope; buffers remember their stream and free
// themselves asynchronously on it, so a release is ordered after the kernels that used the memory.
inline cudaStream_t& alloc_stream_ref()
{
  static thread_local cudaStream_t s = nullptr;
  return s;
}
struct alloc_scope {
  cudaStream_t prev;
  explicit alloc_scope(cudaStream_t s) : prev(alloc_stream_ref()) { alloc_stream_ref() = s; }
  ~alloc_scope() { alloc_stream_ref() = prev; }
};

// Keeps freed device memory in the default pool between solves (configured once per device).
inline void configure_pool_once()
{
  static thread_local int configured_device = -1;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev == configured_device) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  configured_device = dev;
}

// A kernel's dynamic shared memory limit is a property of the function, shared by every host
// thread: set per launch, two solves on different threads could lower it under each other's
// launch.  It is therefore raised once per function and device to the device's opt-in maximum
// less the function's static shared memory; launches that ask for less are unaffected.
inline void allow_max_dynamic_smem(const void* fn)
{
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0, optin = 0;
  B200_CUDA_CHECK(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({fn, dev})) return;
  B200_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  B200_CUDA_CHECK(cudaFuncGetAttributes(&fa, fn));
  B200_CUDA_CHECK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       optin - (int)fa.sharedSizeBytes));
  done.insert({fn, dev});
}

// Dynamic shared memory a launch of fn may ask for on the current device.
inline size_t max_dynamic_smem(const void* fn)
{
  int dev = 0, optin = 0;
  B200_CUDA_CHECK(cudaGetDevice(&dev));
  B200_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa{};
  B200_CUDA_CHECK(cudaFuncGetAttributes(&fa, fn));
  return (size_t)optin - fa.sharedSizeBytes;
}

// Small pinned host scratch for scalar read-backs (per thread, allocated once).
inline double* pinned_scratch()
{
  static thread_local double* p = nullptr;
  if (!p) B200_CUDA_CHECK(cudaMallocHost(&p, 64 * sizeof(double)));
  return p;
}

// The engines capture CUDA graphs, which the legacy default stream does not allow, so they always
// work on a non-blocking stream of their own, ordered after / before the caller's stream by events.
struct joined_stream {
  cudaStream_t caller, own = nullptr;
  cudaEvent_t ev = nullptr;
  explicit joined_stream(cudaStream_t c) : caller(c)
  {
    B200_CUDA_CHECK(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
    B200_CUDA_CHECK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    B200_CUDA_CHECK(cudaEventRecord(ev, caller));
    B200_CUDA_CHECK(cudaStreamWaitEvent(own, ev, 0));
  }
  ~joined_stream()
  {
    if (cudaEventRecord(ev, own) == cudaSuccess) cudaStreamWaitEvent(caller, ev, 0);
    cudaEventDestroy(ev);
    cudaStreamDestroy(own);
  }
};

// Phase timing printed to stderr when the environment variable CUOPT_B200_TRACE is set.
inline void trace(const char* what)
{
  static const bool on = std::getenv("CUOPT_B200_TRACE") != nullptr;
  if (!on) return;
  static thread_local double last = 0;
  const double t = std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
  if (last > 0) std::fprintf(stderr, "[cuopt_b200] %-40s %8.3f ms\n", what, (t - last) * 1e3);
  last = t;
}

// trace() once the stream's work so far has finished (no synchronisation unless tracing).
inline void trace_sync(cudaStream_t s, const char* what)
{
  static const bool on = std::getenv("CUOPT_B200_TRACE") != nullptr;
  if (!on) return;
  cudaStreamSynchronize(s);
  trace(what);
}

// Device buffer owning `n` elements of T (stream-ordered allocation on alloc_stream_ref()).
template <typename T>
class dbuf {
 public:
  dbuf() = default;
  explicit dbuf(size_t n) { resize(n); }
  ~dbuf() { release(); }
  dbuf(const dbuf&)            = delete;
  dbuf& operator=(const dbuf&) = delete;
  dbuf(dbuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_)
  {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  dbuf& operator=(dbuf&& o) noexcept
  {
    if (this != &o) {
      release();
      p_   = o.p_;
      n_   = o.n_;
      s_   = o.s_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  void resize(size_t n)
  {
    release();
    s_ = alloc_stream_ref();
    if (n) B200_CUDA_CHECK(cudaMallocAsync(&p_, n * sizeof(T), s_));
    n_ = n;
  }
  void release()
  {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    n_ = 0;
  }
  void zero(cudaStream_t s)
  {
    if (n_) B200_CUDA_CHECK(cudaMemsetAsync(p_, 0, n_ * sizeof(T), s));
  }
  void upload(const T* h, size_t n, cudaStream_t s)
  {
    if (n) B200_CUDA_CHECK(cudaMemcpyAsync(p_, h, n * sizeof(T), cudaMemcpyDefault, s));
  }
  void download(T* h, size_t n, cudaStream_t s) const
  {
    if (n) B200_CUDA_CHECK(cudaMemcpyAsync(h, p_, n * sizeof(T), cudaMemcpyDefault, s));
  }
  T* data() { return p_; }
  const T* data() const { return p_; }
  size_t size() const { return n_; }

 private:
  T* p_          = nullptr;
  size_t n_      = 0;
  cudaStream_t s_ = nullptr;
};

#ifdef __CUDACC__
__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Neumaier-compensated running sum (FP64 norms and objectives of the termination test).
struct ksum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v)
  {
    double t = s + v;
    if (fabs(s) >= fabs(v))
      c += (s - t) + v;
    else
      c += (v - t) + s;
    s = t;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

// Streaming (evict-first) loads for matrix data that is read once per sweep, so the L2 keeps the
// iterate vectors that the gathers reuse.
__device__ __forceinline__ double ld_stream(const double* p) { return __ldcs(p); }
__device__ __forceinline__ float ld_stream(const float* p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int* p) { return __ldcs(p); }

#endif  // __CUDACC__

#ifdef __CUDACC__
#define B200_HD __host__ __device__
#else
#define B200_HD
#endif

B200_HD inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// Sliced-ELL element address.  A slice holds 32 rows; row t of the slice owns lane t.  Elements are
// grouped in chunks of 4 consecutive row elements per lane, and the 32 lanes' chunks are adjacent:
// element k of lane t lives at base + ((k / 4) * 32 + t) * 4 + k % 4.  A warp therefore reads one
// chunk of every row with a single 128-bit load per lane (512 contiguous bytes for 32-bit data).
// Slice lengths are multiples of 4 and slice bases multiples of 4 elements (16-byte aligned).
constexpr int kChunk = 4;
B200_HD inline int64_t sell_pos(int64_t base, int k, int lane)
{
  return base + ((int64_t)(k >> 2) * 32 + lane) * kChunk + (k & 3);
}

}  // namespace cuopt_b200
