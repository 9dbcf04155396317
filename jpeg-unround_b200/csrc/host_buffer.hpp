// Host arrays of a result (the binary64 canvas, coefficients, planes and picture) in pinned
// memory from a process-wide cache of pinned blocks: the copies from the device run at the
// link's speed into pages that are already resident, and a caller that solves again reuses the
// blocks a freed result gave back instead of faulting in fresh pages. Where pinning fails the
// array is pageable memory.
#pragma once

#include <cstddef>

namespace urb {

class HostBuffer {
 public:
  HostBuffer() = default;
  HostBuffer(const HostBuffer&) = delete;
  HostBuffer& operator=(const HostBuffer&) = delete;
  HostBuffer(HostBuffer&& other) noexcept;
  HostBuffer& operator=(HostBuffer&& other) noexcept;
  ~HostBuffer();

  // `count` doubles; the contents are not kept.
  void resize(std::size_t count);
  [[nodiscard]] double* data() { return data_; }
  [[nodiscard]] const double* data() const { return data_; }
  [[nodiscard]] std::size_t size() const { return size_; }
  [[nodiscard]] bool empty() const { return size_ == 0; }

 private:
  void release();
  double* data_ = nullptr;
  std::size_t size_ = 0;
  std::size_t bytes_ = 0;  // of the block
  bool pinned_ = false;
};

}  // namespace urb
