// Host <-> device transfer helpers for host-resident problem data.
//
// Pageable cudaMemcpy runs through the driver's own small staging buffer and reaches only a few
// GB/s.  staged_upload copies through two pinned buffers of its own instead: host threads fill one
// buffer while the DMA engine drains the other, so large uploads run at host-memcpy speed.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <mutex>
#include <thread>
#include <vector>

#include "common.cuh"

namespace cuopt_b200 {

// memcpy split over up to 16 host threads for large copies.
inline void parallel_memcpy(void* dst, const void* src, size_t bytes)
{
  constexpr size_t kChunk = size_t(2) << 20;  // at least this much per thread
  const unsigned hw       = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const unsigned parts    = (unsigned)std::min<size_t>(hw, bytes / kChunk);
  if (parts <= 1) {
    std::memcpy(dst, src, bytes);
    return;
  }
  auto part = [=](unsigned t) {
    const size_t lo = bytes * t / parts, hi = bytes * (t + 1) / parts;
    std::memcpy(static_cast<char*>(dst) + lo, static_cast<const char*>(src) + lo, hi - lo);
  };
  std::vector<std::thread> pool;
  unsigned started = 0;
  try {
    for (; started < parts; ++started) pool.emplace_back(part, started);
  } catch (...) {  // no thread to spare: the rest is copied here
  }
  for (unsigned t = started; t < parts; ++t) part(t);
  for (auto& th : pool) th.join();
}

// fn(lo, hi) over [0, count) split into contiguous ranges on up to 16 host threads (the calling
// thread takes the last range; at least `grain` items per range, so small counts run on the
// calling thread alone).  An exception thrown by fn on any thread is rethrown to the caller once
// every range has ended (the first one, if several threw).
template <class F>
void parallel_ranges(int count, F&& fn, int grain = 16)
{
  const int hw    = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const int parts = std::max(1, std::min(hw, count / std::max(1, grain)));
  if (parts <= 1) {
    fn(0, count);
    return;
  }
  std::mutex mu;
  std::exception_ptr failure;
  auto run = [&](int t) {
    try {
      fn((int)((int64_t)count * t / parts), (int)((int64_t)count * (t + 1) / parts));
    } catch (...) {
      std::lock_guard<std::mutex> lock(mu);
      if (!failure) failure = std::current_exception();
    }
  };
  std::vector<std::thread> pool;
  int started = 0;
  try {
    for (; started < parts - 1; ++started) pool.emplace_back(run, started);
  } catch (...) {  // no thread to spare: the rest runs here
  }
  for (int t = started; t < parts; ++t) run(t);
  for (auto& th : pool) th.join();
  if (failure) std::rethrow_exception(failure);
}

// Copies the pieces one after another into dst, split over up to 16 host threads by bytes (a
// thread's range may cover many small pieces or part of a large one).
struct host_piece {
  const void* src;
  size_t bytes;
};
inline void parallel_gather(char* dst, const host_piece* pieces, size_t count, size_t total)
{
  constexpr size_t kPerThread = size_t(2) << 20;
  const unsigned hw    = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  const unsigned parts = (unsigned)std::max<size_t>(1, std::min<size_t>(hw, total / kPerThread));
  auto copy_range = [&](size_t lo, size_t hi) {  // bytes [lo, hi) of the concatenation
    size_t at = 0;
    for (size_t i = 0; i < count && at < hi; ++i) {
      const size_t b = pieces[i].bytes, s0 = std::max(lo, at), s1 = std::min(hi, at + b);
      if (s0 < s1)
        std::memcpy(dst + s0, static_cast<const char*>(pieces[i].src) + (s0 - at), s1 - s0);
      at += b;
    }
  };
  if (parts <= 1) {
    copy_range(0, total);
    return;
  }
  std::vector<std::thread> pool;
  unsigned started = 0;
  try {
    for (; started < parts; ++started)
      pool.emplace_back(copy_range, total * started / parts, total * (started + 1) / parts);
  } catch (...) {  // no thread to spare: the rest is copied here
  }
  for (unsigned t = started; t < parts; ++t) copy_range(total * t / parts, total * (t + 1) / parts);
  for (auto& th : pool) th.join();
}

// Two pinned staging buffers per host thread (allocated once), shared by staged_upload and
// staged_download.
constexpr size_t kStageBytes = size_t(32) << 20;
struct staging_buffers {
  char* buf[2]        = {nullptr, nullptr};
  cudaEvent_t done[2] = {nullptr, nullptr};
};
inline staging_buffers& staging()
{
  static thread_local staging_buffers b;
  for (int i = 0; i < 2; ++i) {
    if (!b.buf[i]) B200_CUDA_CHECK(cudaMallocHost(&b.buf[i], kStageBytes));
    if (!b.done[i]) B200_CUDA_CHECK(cudaEventCreateWithFlags(&b.done[i], cudaEventDisableTiming));
  }
  return b;
}

// Uploads host arrays to device memory through the pinned staging buffers.  put() may return before the copy has reached the device; finish() (or the
// destructor) waits for every copy issued.
class staged_upload {
 public:
  explicit staged_upload(cudaStream_t s) : s_(s) { staging(); }
  ~staged_upload()
  {
    try {
      finish();
    } catch (...) {
    }
  }
  staged_upload(const staged_upload&)            = delete;
  staged_upload& operator=(const staged_upload&) = delete;

  template <typename T>
  void put(T* dst, const T* src, size_t count)
  {
    put_bytes(dst, src, count * sizeof(T));
  }

  void put_bytes(void* dst, const void* src, size_t bytes)
  {
    auto* d       = static_cast<char*>(dst);
    const auto* h = static_cast<const char*>(src);
    while (bytes > 0) {
      if (used_ == kStage) flush();
      const size_t n = std::min(bytes, kStage - used_);
      parallel_memcpy(state().buf[cur_] + used_, h, n);
      pending_.push_back({d, used_, n});
      used_ += n;
      d += n;
      h += n;
      bytes -= n;
    }
  }

  // Uploads the pieces, in order, to consecutive device memory from dst (inside one allocation),
  // filling the staging buffers with all host threads.
  void put_gather(void* dst, const std::vector<host_piece>& pieces)
  {
    auto* d = static_cast<char*>(dst);
    std::vector<host_piece> window;
    size_t i = 0, skip = 0;  // next piece, bytes of it already sent
    while (i < pieces.size()) {
      if (used_ == kStage) flush();
      const size_t space = kStage - used_;
      size_t filled      = 0;
      window.clear();
      while (i < pieces.size() && filled < space) {
        const size_t rest = pieces[i].bytes - skip;
        const size_t take = std::min(rest, space - filled);
        if (take > 0)
          window.push_back({static_cast<const char*>(pieces[i].src) + skip, take});
        filled += take;
        if (take == rest) {
          ++i;
          skip = 0;
        } else {
          skip += take;
        }
      }
      if (filled == 0) continue;
      parallel_gather(state().buf[cur_] + used_, window.data(), window.size(), filled);
      pending_.push_back({d, used_, filled});
      used_ += filled;
      d += filled;
    }
  }

  void finish()
  {
    flush();
    auto& st = state();
    for (int i = 0; i < 2; ++i)
      if (armed_[i]) B200_CUDA_CHECK(cudaEventSynchronize(st.done[i]));
    armed_[0] = armed_[1] = false;
  }

 private:
  static constexpr size_t kStage = kStageBytes;
  struct piece {
    char* dst;
    size_t off, bytes;
  };
  static staging_buffers& state() { return staging(); }
  // Issues the copies of the current buffer and switches to the other one (waiting until the
  // DMA engine has drained it).
  void flush()
  {
    if (pending_.empty()) return;
    auto& st = state();
    for (const piece& p : pending_)
      B200_CUDA_CHECK(cudaMemcpyAsync(p.dst, st.buf[cur_] + p.off, p.bytes,
                                      cudaMemcpyHostToDevice, s_));
    B200_CUDA_CHECK(cudaEventRecord(st.done[cur_], s_));
    armed_[cur_] = true;
    pending_.clear();
    cur_  = 1 - cur_;
    used_ = 0;
    if (armed_[cur_]) {
      B200_CUDA_CHECK(cudaEventSynchronize(st.done[cur_]));
      armed_[cur_] = false;
    }
  }

  cudaStream_t s_;
  int cur_         = 0;
  size_t used_     = 0;
  bool armed_[2]   = {false, false};
  std::vector<piece> pending_;
};

// Copies `bytes` of device memory to host memory through the pinned staging buffers, after the
// work already queued on `s`: the DMA engine fills one buffer while host threads empty the other,
// in pieces of kPiece bytes so the two overlap.  Returns when the host copy is complete.
inline void staged_download(void* dst, const void* src, size_t bytes, cudaStream_t s)
{
  constexpr size_t kPiece = size_t(8) << 20;
  if (bytes == 0) return;
  auto& st      = staging();
  auto* d       = static_cast<char*>(dst);
  const auto* h = static_cast<const char*>(src);
  size_t off    = 0;
  int cur       = 0;
  size_t n      = std::min(bytes, kPiece);
  B200_CUDA_CHECK(cudaMemcpyAsync(st.buf[cur], h, n, cudaMemcpyDeviceToHost, s));
  B200_CUDA_CHECK(cudaEventRecord(st.done[cur], s));
  for (;;) {
    const size_t next = off + n;
    const size_t nn   = std::min(bytes - next, kPiece);
    if (nn > 0) {
      B200_CUDA_CHECK(cudaMemcpyAsync(st.buf[1 - cur], h + next, nn, cudaMemcpyDeviceToHost, s));
      B200_CUDA_CHECK(cudaEventRecord(st.done[1 - cur], s));
    }
    B200_CUDA_CHECK(cudaEventSynchronize(st.done[cur]));
    parallel_memcpy(d + off, st.buf[cur], n);
    if (nn == 0) break;
    off = next;
    n   = nn;
    cur = 1 - cur;
  }
}

}  // namespace cuopt_b200
