// Project-written stand-in for quicky_utils::quicky_bitfield<T> (an external
// library of the reference, not vendored with it).  Test infrastructure: it lets
// the reference's own emp_strategy headers compile unmodified in oracle/_ref.
//
// Semantics, as the reference headers use them (include/emp_position_strategy.h:
// 183-208, include/emp_piece_db.h:830-884, include/emp_situation_binary_dumper.h:
// 103-117, include/emp_FSM_situation.h):
//   quicky_bitfield(n, ones)  n bits, all 0 or all 1 (bits past n stay 0)
//   set(v, k, off)            bits off..off+k-1 := low k bits of v
//   get(v&, k, off)           v := bits off..off+k-1
//   ffs()                     1-based index of the lowest set bit, 0 when none
//   apply_and(a, b) / apply_or(a, b)   *this := a & b / a | b, word by word
//   bitsize(), reset(), dump_in(ostream) (raw words, little endian)
// Bit i lives in word i / (8*sizeof(T)), bit i % (8*sizeof(T)).
//
// A write to a bit past the storage (the reference's identical-piece mask
// construction can index another kind's piece, include/emp_piece_db.h:874-875)
// is undefined behaviour in a plain array implementation.  Here it is dropped
// and counted in out_of_range_writes(), so the driver can report it.  A write
// inside the last word but past n (padding) is kept; padding bits are never 1 in
// a set the search walks, because every walked set is an AND with a table entry
// whose padding is 0.
#pragma once

// The external headers this replaces also brought in assert, iostream and
// iomanip for the reference headers that include them.
#include <algorithm>
#include <cassert>
#include <cstdint>
#include <cstring>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <vector>

namespace quicky_utils {

inline uint64_t& bitfield_out_of_range_counter()
{
    static uint64_t n = 0;
    return n;
}

template <typename T>
class quicky_bitfield {
  public:
    static constexpr unsigned kBits = 8 * sizeof(T);

    quicky_bitfield() : m_size(0) {}
    explicit quicky_bitfield(unsigned int p_size, bool p_ones = false)
        : m_size(p_size), m_words((p_size + kBits - 1) / kBits, T(0))
    {
        if (p_ones)
            for (unsigned int i = 0; i < p_size; ++i) m_words[i / kBits] |= T(1) << (i % kBits);
    }

    unsigned int bitsize() const { return m_size; }

    void reset() { std::fill(m_words.begin(), m_words.end(), T(0)); }

    template <typename V>
    void set(V p_value, unsigned int p_nb_bits, unsigned int p_offset)
    {
        for (unsigned int b = 0; b < p_nb_bits; ++b) {
            const unsigned int i = p_offset + b;
            if (i / kBits >= m_words.size()) {
                ++bitfield_out_of_range_counter();
                continue;
            }
            const T bit = T(1) << (i % kBits);
            if ((static_cast<uint64_t>(p_value) >> b) & 1u) m_words[i / kBits] |= bit;
            else m_words[i / kBits] &= ~bit;
        }
    }

    template <typename V>
    void get(V& p_value, unsigned int p_nb_bits, unsigned int p_offset) const
    {
        uint64_t v = 0;
        for (unsigned int b = 0; b < p_nb_bits; ++b) {
            const unsigned int i = p_offset + b;
            if (i / kBits < m_words.size() && ((m_words[i / kBits] >> (i % kBits)) & 1u)) v |= uint64_t(1) << b;
        }
        p_value = static_cast<V>(v);
    }

    unsigned int ffs() const
    {
        for (size_t w = 0; w < m_words.size(); ++w)
            if (m_words[w]) return static_cast<unsigned int>(w * kBits + __builtin_ctzll(m_words[w]) + 1);
        return 0;
    }

    void apply_and(const quicky_bitfield& a, const quicky_bitfield& b)
    {
        for (size_t w = 0; w < m_words.size(); ++w) m_words[w] = a.m_words[w] & b.m_words[w];
    }

    void apply_or(const quicky_bitfield& a, const quicky_bitfield& b)
    {
        for (size_t w = 0; w < m_words.size(); ++w) m_words[w] = a.m_words[w] | b.m_words[w];
    }

    void dump_in(std::ostream& os) const
    {
        os.write(reinterpret_cast<const char*>(m_words.data()), static_cast<std::streamsize>(m_words.size() * sizeof(T)));
    }

  private:
    unsigned int m_size;
    std::vector<T> m_words;
};

}  // namespace quicky_utils
