// Minimal fixed-capacity ring buffer standing in for boost::circular_buffer
// (Boost is not vendored with the reference and not installed here). The
// reference uses it only to remember which face/node spans are in the
// current stencil window (zone_FD/src/src/differ.cpp:33,67): push_back drops
// the oldest element once the buffer is full, operator[](0) is the oldest,
// size() counts the held elements. No arithmetic passes through it.
#pragma once
#include <cstddef>
#include <vector>
namespace boost {
template <class T> class circular_buffer {
public:
    explicit circular_buffer(std::size_t capacity) : cap_(capacity), head_(0), size_(0) { buf_.resize(capacity); }
    void push_back(const T &v) {
        if (cap_ == 0) return;
        if (size_ < cap_) { buf_[(head_ + size_) % cap_] = v; ++size_; }
        else { buf_[head_] = v; head_ = (head_ + 1) % cap_; }
    }
    T &operator[](std::size_t i) { return buf_[(head_ + i) % cap_]; }
    const T &operator[](std::size_t i) const { return buf_[(head_ + i) % cap_]; }
    std::size_t size() const { return size_; }
    std::size_t capacity() const { return cap_; }
private:
    std::vector<T> buf_;
    std::size_t cap_, head_, size_;
};
} // namespace boost
