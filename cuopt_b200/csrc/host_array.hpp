// Host arrays without zero-fill, on transparent huge pages when large.
#pragma once

#include <sys/mman.h>

#include <cstddef>
#include <cstdlib>
#include <memory>
#include <new>
#include <utility>
#include <vector>

namespace cuopt_b200 {

// std::vector whose resize leaves new elements uninitialised: the problem arrays are always
// overwritten right after they are sized, and zero-filling 10^8 elements first (single-threaded)
// would cost as much as the copy itself.  Arrays of 4 MiB or more are 2 MiB aligned and advised
// as transparent huge pages, which halves the page-fault cost of filling fresh memory.
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
    const std::size_t rounded = (bytes + kHuge - 1) / kHuge * kHuge;
    void* p                   = std::aligned_alloc(kHuge, rounded);
    if (!p) throw std::bad_alloc();
    madvise(p, rounded, MADV_HUGEPAGE);
    return static_cast<T*>(p);
  }
  void deallocate(T* p, std::size_t n)
  {
    if (n * sizeof(T) < kHugeMin)
      std::allocator<T>::deallocate(p, n);
    else
      std::free(p);
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
