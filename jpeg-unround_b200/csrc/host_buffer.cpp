// The cache of pinned blocks behind HostBuffer. Idle blocks are kept up to kIdleLimit bytes in
// all; a request takes the smallest idle block that holds it and is at most twice its size, or
// pins a new one (rounded up to 2 MiB). The cache is never destroyed: the blocks outlive static
// destruction, when the CUDA runtime may be gone, and the process's exit returns them.
#include "host_buffer.hpp"

#include <cstdlib>
#include <map>
#include <mutex>
#include <new>
#include <utility>

#include <cuda_runtime.h>

namespace urb {

namespace {

constexpr std::size_t kIdleLimit = std::size_t{4} << 30;
constexpr std::size_t kGrain = std::size_t{2} << 20;

struct Cache {
  std::mutex lock;
  std::multimap<std::size_t, void*> idle;  // bytes -> block
  std::size_t idle_bytes = 0;

  // A pinned block of at least `bytes` (its size into `got`), or null.
  void* take(std::size_t bytes, std::size_t& got) {
    {
      std::lock_guard<std::mutex> hold(lock);
      auto it = idle.lower_bound(bytes);
      if (it != idle.end() && it->first <= 2 * bytes) {
        void* block = it->second;
        got = it->first;
        idle_bytes -= it->first;
        idle.erase(it);
        return block;
      }
    }
    got = (bytes + kGrain - 1) / kGrain * kGrain;
    void* block = nullptr;
    if (cudaHostAlloc(&block, got, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();  // the failure is not the caller's error
      return nullptr;
    }
    return block;
  }

  void give(void* block, std::size_t bytes) {
    {
      std::lock_guard<std::mutex> hold(lock);
      if (idle_bytes + bytes <= kIdleLimit) {
        idle.emplace(bytes, block);
        idle_bytes += bytes;
        return;
      }
    }
    cudaFreeHost(block);
  }
};

Cache& cache() {
  static Cache* made = new Cache;
  return *made;
}

}  // namespace

HostBuffer::HostBuffer(HostBuffer&& other) noexcept
    : data_(std::exchange(other.data_, nullptr)),
      size_(std::exchange(other.size_, 0)),
      bytes_(std::exchange(other.bytes_, 0)),
      pinned_(std::exchange(other.pinned_, false)) {}

HostBuffer& HostBuffer::operator=(HostBuffer&& other) noexcept {
  if (this != &other) {
    release();
    data_ = std::exchange(other.data_, nullptr);
    size_ = std::exchange(other.size_, 0);
    bytes_ = std::exchange(other.bytes_, 0);
    pinned_ = std::exchange(other.pinned_, false);
  }
  return *this;
}

HostBuffer::~HostBuffer() { release(); }

void HostBuffer::release() {
  if (data_ != nullptr) {
    if (pinned_) {
      cache().give(data_, bytes_);
    } else {
      std::free(data_);
    }
  }
  data_ = nullptr;
  size_ = bytes_ = 0;
  pinned_ = false;
}

void HostBuffer::resize(std::size_t count) {
  const std::size_t bytes = count * sizeof(double);
  if (count == size_) return;
  if (bytes <= bytes_ && bytes * 2 >= bytes_) {
    size_ = count;
    return;
  }
  release();
  if (count == 0) return;
  std::size_t got = 0;
  void* block = cache().take(bytes, got);
  if (block != nullptr) {
    pinned_ = true;
  } else {
    block = std::malloc(bytes);
    if (block == nullptr) throw std::bad_alloc();
    got = bytes;
  }
  data_ = static_cast<double*>(block);
  size_ = count;
  bytes_ = got;
}

}  // namespace urb
