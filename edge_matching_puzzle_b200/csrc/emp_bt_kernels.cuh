// Device-side table access of the exhaustive backtracker (sm_100a).
//
// The search is the reference's emp_strategy::specific_run
// (include/emp_strategy.h:343-410): a depth-first walk over the levels of a
// position order; at each level the candidate set is
//     table[constraint] & availability of the position's kind
// (include/emp_position_strategy.h:172-186) and the transitions are tried in
// ascending bit order (ffs, :205-208).  A placement is a "node"; a placement
// at the last level is a solution.  With identical pieces, trying t also
// removes the bits of its identical mask (:189-202).
//
// Table blob layout: emp_model.h (DeviceTables).  Candidate bit t =
// kind_index*4 + orientation lives in 64-bit word t>>6, bit t&63.
#pragma once

#include "emp_layout.h"

#include <cstdint>

namespace emp {
namespace dev {

// header word indices of a puzzle blob
enum : uint32_t {
    H_N = 1, H_NCOL = 2, H_KW = 3, H_AOFF = 6, H_AWORDS = 9, H_SIDE = 10, H_PAIR = 13, H_DESC = 14, H_TINFO = 15,
    H_EXTRA = 18, H_INIT = 21, H_W = 22, H_H = 23, H_SIZE = 24, H_MAXKW = 25
};

__device__ __forceinline__ uint32_t ldg(const uint32_t* p) { return __ldg(p); }
__device__ __forceinline__ uint64_t ldg64(const uint32_t* p)
{
    return __ldg(reinterpret_cast<const unsigned long long*>(p));
}

struct LevelDesc {
    uint32_t d0, d1, d2, d3, d4, d5, d6, d7;
    // transition tables of the kinds of neighbours A, B and the extra ones (read when asked for)
    uint32_t d8 = 0, d9 = 0, d10 = 0, d11 = 0;
    __device__ __forceinline__ uint32_t kw() const { return d0 & 0xFFu; }
    __device__ __forceinline__ uint32_t kind() const { return (d0 >> 8) & 3u; }
    __device__ __forceinline__ uint32_t nextra() const { return (d0 >> 13) & 7u; }
    __device__ __forceinline__ uint32_t aoff() const { return d0 >> 16; }
    __device__ __forceinline__ uint32_t level_a() const { return d1 & 0xFFu; }
    __device__ __forceinline__ uint32_t level_b() const { return (d1 >> 8) & 0xFFu; }
    __device__ __forceinline__ uint32_t shift_a() const { return (d1 >> 16) & 0xFFu; }
    __device__ __forceinline__ uint32_t shift_b() const { return d1 >> 24; }
    __device__ __forceinline__ uint32_t stride_a() const { return d3 & 0xFFFFu; }
    __device__ __forceinline__ uint32_t stride_b() const { return d3 >> 16; }
    __device__ __forceinline__ uint32_t extra_side(uint32_t j) const { return (d7 >> (2 * j)) & 3u; }
    __device__ __forceinline__ uint32_t extra_level(uint32_t j) const { return (d7 >> (8 + 8 * j)) & 0xFFu; }
    // pair-table row of this level given the stack words of neighbours A and B
    __device__ __forceinline__ uint32_t row(uint32_t ea, uint32_t eb) const
    {
        return d2 + ((ea >> shift_a()) & 31u) * stride_a() + ((eb >> shift_b()) & 31u) * stride_b();
    }
};

__device__ __forceinline__ LevelDesc load_desc(const uint32_t* tb, uint32_t desc_off, uint32_t L, bool ext = false)
{
    const uint4* d = reinterpret_cast<const uint4*>(tb + desc_off + kDescWords * L);
    const uint4 a = __ldg(d), b = __ldg(d + 1);
    const uint4 c = ext ? __ldg(d + 2) : make_uint4(0, 0, 0, 0);
    return LevelDesc{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
}

// colour that the neighbour placed at the level whose stack word is `e`
// shows towards my side `s` (its side (s+2)&3); 5 bits per side
__device__ __forceinline__ uint32_t facing_colour(uint32_t e, uint32_t s) { return (e >> (5 * ((s + 2) & 3u))) & 31u; }

}  // namespace dev
}  // namespace emp
