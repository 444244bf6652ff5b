// Device side of the exhaustive backtracker (sm_100a).
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
// Table blob layout: see emp_model.h (DeviceTables, header words 0..31).
#pragma once

#include <cstdint>

namespace emp {
namespace dev {

// header word indices of a puzzle blob
enum : uint32_t {
    H_N = 1, H_NCOL = 2, H_KW = 3, H_AOFF = 6, H_AWORDS = 9, H_SIDE = 10, H_BASE = 13,
    H_DESC = 14, H_TINFO = 15, H_EXTRA = 18, H_INIT = 21, H_W = 22, H_H = 23, H_SIZE = 24,
    H_DEPTH = 25
};

__device__ __forceinline__ uint32_t ldg(const uint32_t* p) { return __ldg(p); }

// level descriptor fields (emp_model.cpp build_device_tables)
struct LevelDesc {
    uint32_t kind, nplaced, kw, aoff, base, w0, w1;
};

__device__ __forceinline__ LevelDesc load_desc(const uint32_t* tb, uint32_t L)
{
    const uint32_t* d = tb + ldg(tb + H_DESC) + 4 * L;
    LevelDesc r;
    r.w0 = ldg(d);
    r.w1 = ldg(d + 1);
    r.base = ldg(d + 2);
    r.aoff = ldg(d + 3) & 0xFFFFu;
    r.kind = r.w0 & 3u;
    r.nplaced = (r.w0 >> 2) & 7u;
    r.kw = (r.w0 >> 16) & 0xFFu;
    return r;
}

__device__ __forceinline__ uint32_t desc_side(const LevelDesc& d, uint32_t j) { return (d.w0 >> (5 + 2 * j)) & 3u; }
__device__ __forceinline__ uint32_t desc_nb(const LevelDesc& d, uint32_t j) { return (d.w1 >> (8 * j)) & 0xFFu; }

}  // namespace dev
}  // namespace emp
