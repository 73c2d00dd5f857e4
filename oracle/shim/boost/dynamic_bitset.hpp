// Test infrastructure (oracle only): a minimal stand-in for the part of
// Boost.DynamicBitset that the reference uses (src/Graph.hpp:5; call sites
// src/Graph.cpp:1710-1760, 1948-2032, 2269-2299), so the reference compiles
// in a container without Boost.  Boost is a third-party dependency the
// reference does not vendor or pin; this header restates the documented
// semantics of the members used: construction with a size, set(i), reset(),
// operator[] (read and assign), any(), count(), num_blocks(), size(),
// find_first(), find_next(i) (first set bit strictly after i) and npos.
#pragma once
#include <cstddef>
#include <cstdint>
#include <vector>

namespace boost {

template <typename Block = unsigned long>
class dynamic_bitset {
   public:
    static constexpr std::size_t npos = static_cast<std::size_t>(-1);

    class reference {
       public:
        reference(std::vector<std::uint64_t>& w, std::size_t i) : w_(w), i_(i) {}
        reference& operator=(bool v) {
            if (v) w_[i_ >> 6] |= (std::uint64_t)1 << (i_ & 63);
            else w_[i_ >> 6] &= ~((std::uint64_t)1 << (i_ & 63));
            return *this;
        }
        operator bool() const { return (w_[i_ >> 6] >> (i_ & 63)) & 1u; }

       private:
        std::vector<std::uint64_t>& w_;
        std::size_t i_;
    };

    dynamic_bitset() = default;
    explicit dynamic_bitset(std::size_t nbits, unsigned long value = 0) : bits_(nbits), words_((nbits + 63) / 64, 0) {
        if (nbits && value) words_[0] = value;
    }

    dynamic_bitset& set(std::size_t i) {
        words_[i >> 6] |= (std::uint64_t)1 << (i & 63);
        return *this;
    }
    dynamic_bitset& reset() {
        for (auto& x : words_) x = 0;
        return *this;
    }
    reference operator[](std::size_t i) { return reference(words_, i); }
    bool operator[](std::size_t i) const { return (words_[i >> 6] >> (i & 63)) & 1u; }
    bool any() const {
        for (auto x : words_)
            if (x) return true;
        return false;
    }
    std::size_t count() const {
        std::size_t c = 0;
        for (auto x : words_) c += (std::size_t)__builtin_popcountll(x);
        return c;
    }
    std::size_t size() const { return bits_; }
    std::size_t num_blocks() const { return words_.size(); }
    std::size_t find_first() const { return scan_from(0); }
    std::size_t find_next(std::size_t i) const { return i + 1 >= bits_ ? npos : scan_from(i + 1); }

   private:
    std::size_t scan_from(std::size_t i) const {
        if (i >= bits_) return npos;
        std::size_t k = i >> 6;
        std::uint64_t x = words_[k] & (~(std::uint64_t)0 << (i & 63));
        for (;;) {
            if (x) {
                std::size_t r = (k << 6) + (std::size_t)__builtin_ctzll(x);
                return r < bits_ ? r : npos;
            }
            if (++k >= words_.size()) return npos;
            x = words_[k];
        }
    }

    std::size_t bits_ = 0;
    std::vector<std::uint64_t> words_;
};

}  // namespace boost
