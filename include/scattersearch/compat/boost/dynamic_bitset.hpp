// Stand-in for boost::dynamic_bitset<> for drivers written against the
// reference's include/annsearch.h (which includes <boost/dynamic_bitset.hpp>
// for the caller-owned `flags` argument of its search methods).  Boost is
// not required: this is a small self-contained bitset with the members those
// drivers and the reference's searches use -- construction from (size,
// value), copy and move, operator[] (readable and assignable), test, set,
// reset, flip, count, any, none, size, resize.  The GPU search keeps its
// visited set on the device, so the drop-in ANNSearch only resets `flags`.
//
// Like the header it stands in for, it also brings in <cassert>, <algorithm>
// and <cstring>, which the reference's drivers use without including them
// (tests/search.cpp:31 calls assert).
#ifndef SCATTERSEARCH_COMPAT_BOOST_DYNAMIC_BITSET_HPP
#define SCATTERSEARCH_COMPAT_BOOST_DYNAMIC_BITSET_HPP

#include <algorithm>
#include <cassert>
#include <climits>
#include <cstddef>
#include <cstring>
#include <memory>
#include <vector>

namespace boost {

template <typename Block = unsigned long, typename Allocator = std::allocator<Block>>
class dynamic_bitset {
 public:
  typedef Block block_type;
  typedef std::size_t size_type;
  static constexpr size_type bits_per_block = sizeof(Block) * CHAR_BIT;

  // Assignable view of one bit, returned by the non-const operator[].
  class reference {
   public:
    reference(Block &b, Block mask) : b_(b), m_(mask) {}
    reference &operator=(bool x) {
      if (x) b_ |= m_;
      else b_ &= ~m_;
      return *this;
    }
    reference &operator=(const reference &o) { return *this = static_cast<bool>(o); }
    reference &operator|=(bool x) { return x ? (*this = true) : *this; }
    reference &operator&=(bool x) { return x ? *this : (*this = false); }
    operator bool() const { return (b_ & m_) != 0; }
    bool operator~() const { return (b_ & m_) == 0; }
    reference &flip() { b_ ^= m_; return *this; }

   private:
    Block &b_;
    Block m_;
  };

  dynamic_bitset() = default;
  // num_bits bits; the low bits of `value` set the first bits (boost's rule).
  explicit dynamic_bitset(size_type num_bits, unsigned long value = 0,
                          const Allocator &alloc = Allocator())
      : blocks_(blocks_for(num_bits), Block(0), alloc), size_(num_bits) {
    for (size_type i = 0; i < num_bits && i < sizeof(unsigned long) * CHAR_BIT; ++i)
      if ((value >> i) & 1ul) set(i);
  }
  dynamic_bitset(const dynamic_bitset &) = default;
  dynamic_bitset(dynamic_bitset &&) noexcept = default;
  dynamic_bitset &operator=(const dynamic_bitset &) = default;
  dynamic_bitset &operator=(dynamic_bitset &&) noexcept = default;

  size_type size() const { return size_; }
  size_type num_blocks() const { return blocks_.size(); }
  bool empty() const { return size_ == 0; }

  reference operator[](size_type pos) {
    assert(pos < size_);
    return reference(blocks_[pos / bits_per_block], mask(pos));
  }
  bool operator[](size_type pos) const { return test(pos); }
  bool test(size_type pos) const {
    assert(pos < size_);
    return (blocks_[pos / bits_per_block] & mask(pos)) != 0;
  }

  dynamic_bitset &set() {
    std::fill(blocks_.begin(), blocks_.end(), ~Block(0));
    clear_tail();
    return *this;
  }
  dynamic_bitset &set(size_type pos, bool val = true) {
    (*this)[pos] = val;
    return *this;
  }
  dynamic_bitset &reset() {
    std::fill(blocks_.begin(), blocks_.end(), Block(0));
    return *this;
  }
  dynamic_bitset &reset(size_type pos) { return set(pos, false); }
  dynamic_bitset &flip() {
    for (auto &b : blocks_) b = ~b;
    clear_tail();
    return *this;
  }
  dynamic_bitset &flip(size_type pos) {
    (*this)[pos].flip();
    return *this;
  }

  size_type count() const {
    size_type c = 0;
    for (Block b : blocks_)
      for (; b; b &= b - 1) ++c;
    return c;
  }
  bool any() const {
    for (Block b : blocks_)
      if (b) return true;
    return false;
  }
  bool none() const { return !any(); }

  void resize(size_type num_bits, bool value = false) {
    const size_type old = size_;
    blocks_.resize(blocks_for(num_bits), value ? ~Block(0) : Block(0));
    size_ = num_bits;
    if (value)
      for (size_type i = old; i < num_bits && i < blocks_for(old) * bits_per_block; ++i) set(i);
    clear_tail();
  }
  void clear() {
    blocks_.clear();
    size_ = 0;
  }

  friend bool operator==(const dynamic_bitset &a, const dynamic_bitset &b) {
    return a.size_ == b.size_ && a.blocks_ == b.blocks_;
  }
  friend bool operator!=(const dynamic_bitset &a, const dynamic_bitset &b) { return !(a == b); }

 private:
  static size_type blocks_for(size_type bits) {
    return (bits + bits_per_block - 1) / bits_per_block;
  }
  static Block mask(size_type pos) { return Block(1) << (pos % bits_per_block); }
  void clear_tail() {
    const size_type extra = size_ % bits_per_block;
    if (extra && !blocks_.empty()) blocks_.back() &= (Block(1) << extra) - 1;
  }

  std::vector<Block, Allocator> blocks_;
  size_type size_ = 0;
};

}  // namespace boost

#endif
