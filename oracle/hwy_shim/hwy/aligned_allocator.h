// hwy/aligned_allocator.h -- project-written stand-in for the two allocation
// names of the Google Highway 1.2.0 API that the reference's batched engine uses
// (hwy::AllocateAligned<T>(n) and hwy::AlignedFreeUniquePtr<T[]>).
//
// TEST INFRASTRUCTURE ONLY (oracle/): see hwy/highway.h in this directory for
// why the shim exists. Arrays are aligned to 128 bytes (a multiple of every
// vector width hwy/highway.h selects) and their size is rounded up to a whole
// number of 128-byte lines, so full-vector Load/Store at any lane-multiple
// offset inside the array stays inside the allocation.
#pragma once

#include <cstddef>
#include <cstdlib>
#include <memory>
#include <new>

namespace hwy {

inline constexpr std::size_t kShimAlignment = 128;

struct AlignedFreer {
  void operator()(void* p) const noexcept { std::free(p); }
};

template <class T>
using AlignedFreeUniquePtr = std::unique_ptr<T, AlignedFreer>;

template <class T>
AlignedFreeUniquePtr<T[]> AllocateAligned(std::size_t items) {
  std::size_t bytes = items * sizeof(T);
  bytes = (bytes + kShimAlignment - 1) / kShimAlignment * kShimAlignment;
  if (bytes == 0) bytes = kShimAlignment;
  void* p = std::aligned_alloc(kShimAlignment, bytes);
  if (p == nullptr) throw std::bad_alloc();
  return AlignedFreeUniquePtr<T[]>(static_cast<T*>(p));
}

}  // namespace hwy
