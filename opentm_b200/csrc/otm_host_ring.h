// otm_host_ring.h -- offset bookkeeping of the serving form's pinned host ring (plain C++).
//
// Allocations are made in submit order and released in any order; space is reclaimed from the
// oldest live allocation forward, so with first come, first served admission the region behaves
// as a ring. The class only hands out offsets into a region of `capacity` units; the caller
// owns the memory.
#pragma once

#include <cstddef>
#include <cstdint>
#include <deque>

namespace otm {

class RingOffsets {
 public:
  explicit RingOffsets(size_t capacity = 0, size_t align = 1) : cap_(capacity), align_(align ? align : 1) {}
  size_t capacity() const { return cap_; }
  size_t live() const { return live_.size(); }
  // n units at *off (aligned to `align`), or false when the ring has no contiguous room.
  bool alloc(size_t n, size_t* off, int64_t* seq) {
    n = (n + align_ - 1) / align_ * align_;
    if (n == 0) n = align_;
    size_t o;
    if (live_.empty()) {
      head_ = 0;
      if (n > cap_) return false;
      o = 0;
    } else {
      const size_t tail = live_.front().off;
      if (head_ > tail) {  // free space [head, cap) and [0, tail)
        if (n <= cap_ - head_)
          o = head_;
        else if (n <= tail)
          o = 0;
        else
          return false;
      } else {  // wrapped: free space [head, tail)
        if (n <= tail - head_)
          o = head_;
        else
          return false;
      }
    }
    head_ = o + n;
    live_.push_back(Span{o, false});
    *off = o;
    *seq = front_seq_ + int64_t(live_.size()) - 1;
    return true;
  }
  void release(int64_t seq) {
    const int64_t i = seq - front_seq_;
    if (i < 0 || i >= int64_t(live_.size())) return;
    live_[size_t(i)].freed = true;
    while (!live_.empty() && live_.front().freed) {
      live_.pop_front();
      front_seq_++;
    }
  }

 private:
  struct Span {
    size_t off;
    bool freed;
  };
  size_t cap_, align_, head_ = 0;
  std::deque<Span> live_;
  int64_t front_seq_ = 0;
};

}  // namespace otm
