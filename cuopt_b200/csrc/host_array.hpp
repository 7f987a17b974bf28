// Host arrays without zero-fill, on transparent huge pages when large.
#pragma once

#include <sys/mman.h>

#include <cstddef>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

namespace cuopt_b200 {

// Large host blocks (2 MiB aligned, advised as transparent huge pages) with a bounded cache of
// freed ones: a block of the same rounded size is handed out again with its pages already
// faulted in, instead of being returned to the system and zeroed again on first touch (a
// problem, its solution and a batch's arrays are typically allocated at the same sizes solve
// after solve).  At most kCacheBytes are kept.
class huge_blocks {
 public:
  static constexpr std::size_t kAlign = std::size_t(2) << 20, kCacheBytes = std::size_t(1) << 30;
  static void* get(std::size_t rounded)
  {
    {
      auto& c = cache();
      std::lock_guard<std::mutex> lock(c.mu);
      for (std::size_t i = 0; i < c.blocks.size(); ++i)
        if (c.blocks[i].second == rounded) {
          void* p = c.blocks[i].first;
          c.blocks[i] = c.blocks.back();
          c.blocks.pop_back();
          c.bytes -= rounded;
          return p;
        }
    }
    void* p = std::aligned_alloc(kAlign, rounded);
    if (!p) throw std::bad_alloc();
    madvise(p, rounded, MADV_HUGEPAGE);
    return p;
  }
  static void put(void* p, std::size_t rounded)
  {
    auto& c = cache();
    {
      std::lock_guard<std::mutex> lock(c.mu);
      if (c.bytes + rounded <= kCacheBytes) {
        c.blocks.emplace_back(p, rounded);
        c.bytes += rounded;
        return;
      }
    }
    std::free(p);
  }

 private:
  struct state {
    std::mutex mu;
    std::vector<std::pair<void*, std::size_t>> blocks;
    std::size_t bytes = 0;
  };
  static state& cache()
  {
    static state* s = new state;  // never destroyed: arrays may be released during exit
    return *s;
  }
};

// std::vector whose resize leaves new elements uninitialised: the problem arrays are always
// overwritten right after they are sized, and zero-filling 10^8 elements first (single-threaded)
// would cost as much as the copy itself.  Arrays of 4 MiB or more come from huge_blocks.
template <typename T>
struct default_init_allocator : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = default_init_allocator<U>;
  };
  using std::allocator<T>::allocator;
  static constexpr std::size_t kHugeMin = std::size_t(4) << 20, kHuge = std::size_t(2) << 20;
  T* allocate(std::size_t n)
  {
    const std::size_t bytes = n * sizeof(T);
    if (bytes < kHugeMin) return std::allocator<T>::allocate(n);
    return static_cast<T*>(huge_blocks::get((bytes + kHuge - 1) / kHuge * kHuge));
  }
  void deallocate(T* p, std::size_t n)
  {
    const std::size_t bytes = n * sizeof(T);
    if (bytes < kHugeMin)
      std::allocator<T>::deallocate(p, n);
    else
      huge_blocks::put(p, (bytes + kHuge - 1) / kHuge * kHuge);
  }
  template <typename U>
  void construct(U* p) noexcept
  {
    ::new (static_cast<void*>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U* p, Args&&... args)
  {
    ::new (static_cast<void*>(p)) U(std::forward<Args>(args)...);
  }
};
template <typename T>
using host_array = std::vector<T, default_init_allocator<T>>;

}  // namespace cuopt_b200
