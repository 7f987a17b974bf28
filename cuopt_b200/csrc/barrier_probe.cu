// Measurement and test hook: the grid barrier of the persistent plain-iteration kernel on its own.
//
// persist_barrier (kernels.cuh) is the only wait in the persistent kernel.  This entry point runs
// it in a cooperative launch with no sweep around it, to measure what one barrier costs, and to
// check that a barrier which cannot complete (a target above the grid's arrivals, which no block
// will ever provide) ends at its deadline with a status that the host reads, instead of hanging.
#include <cuopt_b200.h>

#include <cstdio>

#include "common.cuh"
#include "kernels.cuh"

extern "C" cuopt_int_t cuOptProbeGridBarrier(cuopt_int_t blocks, cuopt_int_t rounds,
                                             cuopt_int_t unreachable, cuopt_float_t budget_ms,
                                             void* stream, cuopt_int_t* status,
                                             cuopt_float_t* elapsed_ms)
{
  using namespace cuopt_b200;
  if (blocks <= 0 || rounds <= 0 || rounds > 1000000 || !(budget_ms > 0.0) ||
      budget_ms > 10000.0 || !status || !elapsed_ms)
    return CUOPT_INVALID_ARGUMENT;
  try {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0, coop = 0, per_sm = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    const void* fn = (const void*)persist_barrier_probe_kernel;
    B200_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kBlock, 0));
    if (!coop || blocks > per_sm * sms) return CUOPT_INVALID_ARGUMENT;
    alloc_scope scope(s);
    dbuf<persist_ctl> ctl(1);
    dbuf<unsigned long long> el(1);
    ctl.zero(s);
    el.zero(s);
    persist_ctl* c               = ctl.data();
    int r                        = rounds;
    unsigned extra               = unreachable ? 1u : 0u;
    unsigned long long budget    = (unsigned long long)(budget_ms * 1e6);
    unsigned long long* elapsed  = el.data();
    void* args[] = {(void*)&c, (void*)&r, (void*)&extra, (void*)&budget, (void*)&elapsed};
    B200_CUDA_CHECK(cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kBlock), args, 0, s));
    B200_LAUNCH_CHECK();
    persist_ctl hc{};
    unsigned long long he = 0;
    B200_CUDA_CHECK(cudaMemcpyAsync(&hc, c, sizeof(hc), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaMemcpyAsync(&he, elapsed, sizeof(he), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    *status     = hc.status;
    *elapsed_ms = (double)he * 1e-6;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptProbeGridBarrier: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}

namespace cuopt_b200 {
namespace {
// `rounds` cluster barriers (barrier.cluster arrive.release / wait.acquire) in one cluster; block 0
// records the elapsed nanoseconds.
__global__ void cluster_barrier_probe_kernel(int rounds, unsigned long long* elapsed)
{
  const unsigned long long t0 = global_ns();
  for (int r = 0; r < rounds; ++r) cluster_barrier();
  if (cluster_rank() == 0 && threadIdx.x == 0) *elapsed = global_ns() - t0;
}
}  // namespace
}  // namespace cuopt_b200

extern "C" cuopt_int_t cuOptProbeClusterBarrier(cuopt_int_t blocks, cuopt_int_t threads,
                                                cuopt_int_t rounds, void* stream,
                                                cuopt_float_t* elapsed_ms)
{
  using namespace cuopt_b200;
  if (blocks <= 0 || blocks > 16 || threads <= 0 || threads > 1024 || threads % 32 != 0 ||
      rounds <= 0 || rounds > 1000000 || !elapsed_ms)
    return CUOPT_INVALID_ARGUMENT;
  try {
    const cudaStream_t s = static_cast<cudaStream_t>(stream);
    const void* fn       = (const void*)cluster_barrier_probe_kernel;
    if (blocks > 8 &&
        cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
      (void)cudaGetLastError();
      return CUOPT_INVALID_ARGUMENT;
    }
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    cfg.gridDim              = dim3(blocks);
    cfg.blockDim             = dim3(threads);
    cfg.stream               = s;
    attr[0].id               = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = blocks;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs                = attr;
    cfg.numAttrs             = 1;
    int clusters             = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) != cudaSuccess || clusters == 0) {
      (void)cudaGetLastError();
      return CUOPT_INVALID_ARGUMENT;
    }
    alloc_scope scope(s);
    dbuf<unsigned long long> el(1);
    el.zero(s);
    B200_CUDA_CHECK(cudaLaunchKernelEx(&cfg, cluster_barrier_probe_kernel, (int)rounds, el.data()));
    unsigned long long he = 0;
    B200_CUDA_CHECK(cudaMemcpyAsync(&he, el.data(), sizeof(he), cudaMemcpyDeviceToHost, s));
    B200_CUDA_CHECK(cudaStreamSynchronize(s));
    *elapsed_ms = (double)he * 1e-6;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptProbeClusterBarrier: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}
