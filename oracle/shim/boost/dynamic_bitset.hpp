// Minimal stand-in for boost::dynamic_bitset, written for this project so the
// reference library (which includes <boost/dynamic_bitset.hpp>) compiles in a
// container without Boost.  TEST INFRASTRUCTURE ONLY: it is used solely to
// build the reference search as a parity oracle under oracle/_ref/.
//
// Surface the reference needs: a (num_bits, value) constructor, operator[]
// returning an assignable proxy, test(), set(), reset() and size()
// (src/annsearch.cpp:229-231, :258, :1596-1598; tests/search.cpp:71).
// The reference also relies on headers that Boost pulls in transitively:
// <algorithm> for std::sort (annsearch.cpp:215), <cassert> (tests/search.cpp:31)
// and <cstring> for memset (annsearch.cpp:854).
#ifndef SS_ORACLE_BOOST_DYNAMIC_BITSET_SHIM
#define SS_ORACLE_BOOST_DYNAMIC_BITSET_SHIM

#include <algorithm>
#include <cassert>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

namespace boost {

template <typename Block = unsigned long, typename Allocator = std::allocator<Block>>
class dynamic_bitset {
 public:
  using size_type = std::size_t;

  class reference {
   public:
    reference(std::uint64_t* word, std::uint64_t mask) : word_(word), mask_(mask) {}
    operator bool() const { return (*word_ & mask_) != 0; }
    bool operator~() const { return (*word_ & mask_) == 0; }
    reference& operator=(bool v) {
      if (v) *word_ |= mask_; else *word_ &= ~mask_;
      return *this;
    }
    reference& operator=(const reference& other) { return *this = static_cast<bool>(other); }

   private:
    std::uint64_t* word_;
    std::uint64_t mask_;
  };

  dynamic_bitset() : nbits_(0) {}
  explicit dynamic_bitset(size_type num_bits, unsigned long value = 0)
      : words_((num_bits + 63) / 64, 0), nbits_(num_bits) {
    if (!words_.empty()) words_[0] = static_cast<std::uint64_t>(value);
    trim();
  }

  reference operator[](size_type pos) { return reference(&words_[pos >> 6], bit(pos)); }
  bool operator[](size_type pos) const { return (words_[pos >> 6] & bit(pos)) != 0; }
  bool test(size_type pos) const { return (*this)[pos]; }
  dynamic_bitset& set(size_type pos, bool v = true) {
    (*this)[pos] = v;
    return *this;
  }
  dynamic_bitset& reset() {
    std::fill(words_.begin(), words_.end(), 0);
    return *this;
  }
  dynamic_bitset& reset(size_type pos) { return set(pos, false); }
  size_type size() const { return nbits_; }
  void resize(size_type num_bits, bool value = false) {
    words_.resize((num_bits + 63) / 64, value ? ~std::uint64_t(0) : 0);
    nbits_ = num_bits;
    trim();
  }

 private:
  static std::uint64_t bit(size_type pos) { return std::uint64_t(1) << (pos & 63); }
  void trim() {
    if (nbits_ & 63) words_.back() &= (std::uint64_t(1) << (nbits_ & 63)) - 1;
  }
  std::vector<std::uint64_t> words_;
  size_type nbits_;
};

}  // namespace boost

#endif
