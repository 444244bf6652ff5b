// Host-side puzzle model of edge_matching_puzzle_b200.
//
// It rebuilds, from a w x h piece list, what the reference derives in its piece
// database (include/emp_piece_db.h) and in emp_strategy's neighbour wiring
// (include/emp_strategy.h:159-265), and lays it out for the GPU:
//
//  * kinds (0 centre, 1 border, 2 corner = number of frame sides,
//    include/emp_piece.h:122-131), kind indices in file order, auto-similarity
//    (include/emp_piece.h:144-157) and the allowed orientation subset
//    {o : o % 2^similarity == 0} used by the constraint table
//    (include/emp_piece_db.h:1267-1273);
//  * the identical-piece relation and masks with the reference's exact
//    comparison rules (include/emp_piece.h:193-220, emp_piece_db.h:528-540,
//    830-884);
//  * per-side colour masks replacing the reference's 2^(4*cs) constraint table:
//    table[code] == AND over constrained sides s of side_mask[kind][s][colour]
//    (a code constrains exactly the sides whose slot is non-zero and the
//    table's kind is the count of frame slots, emp_piece_db.h:1281-1309), so the
//    candidate set of a level is base[level] & side masks of its placed
//    neighbours & availability;
//  * a level plan for a position order (row-major "basic" or spiral).
//
// Candidate bit t = (kind_index << 2) | orientation, one nibble per piece.  The
// host model keeps 32-bit words (word t >> 5, bit t & 31: 8 pieces per word); the
// device tables (DeviceTables below) store the same bits in 64-bit words (word
// t >> 6, bit t & 63: 16 pieces per word), so a kernel covers a level's candidate
// set in few, fully unrolled word operations.
#pragma once

#include "emp_layout.h"

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace emp {

constexpr uint32_t kMaxPieces = 256;
constexpr uint32_t kMaxColourId = 31;   // colours are packed on 5 bits on the GPU
constexpr uint32_t kMaxLevels = 256;

enum Kind : uint32_t { kCenter = 0, kBorder = 1, kCorner = 2 };

struct PuzzleModel {
    uint32_t width = 0, height = 0, n = 0;
    std::vector<std::array<uint8_t, 4>> colours;  // per piece index: N,E,S,W
    std::vector<uint8_t> kind, similarity;
    std::vector<uint32_t> kind_index;
    std::array<std::vector<uint32_t>, 3> members;   // piece index per (kind, kind index)
    uint32_t max_colour = 0, border_id = 0;         // border_id = max colour + 1
    std::array<uint32_t, 3> kind_words{};           // 32-bit words per kind bitfield
    bool has_identical = false;
    bool identical_out_of_range = false;
    // identical masks per kind: [4*nk][kind_words] (all ones except cleared bits)
    std::array<std::vector<uint32_t>, 3> idmask;

    uint32_t nb_kind(uint32_t k) const { return static_cast<uint32_t>(members[k].size()); }
    // colour of side s (0..3) of piece index p in orientation o (emp_piece.h:173-178)
    uint32_t colour(uint32_t p, uint32_t s, uint32_t o) const { return colours[p][(s + o) & 3]; }
    bool allowed(uint32_t p, uint32_t o) const { return (o % (1u << similarity[p])) == 0; }
};

// Builds the model; returns false with a message on malformed input.
bool build_model(uint32_t width, uint32_t height, const uint8_t* colours, PuzzleModel& m,
                 std::string& error);

// Positions in visiting order: y*w+x.
std::vector<uint32_t> order_basic(uint32_t w, uint32_t h);
std::vector<uint32_t> order_spiral(uint32_t w, uint32_t h);

// Per level of a position order.
struct LevelPlan {
    uint32_t position = 0;
    uint32_t kind = 0;
    uint32_t nplaced = 0;              // neighbours placed at lower levels
    std::array<uint8_t, 4> side{};     // my side facing the placed neighbour
    std::array<uint8_t, 4> nb_level{}; // level of that neighbour
    std::vector<uint32_t> base;        // frame-side masks & allowed orientations
};

// Flattened tables consumed by the GPU kernels (one blob per puzzle), 32-bit
// words; every 64-bit table starts on an even word and the blob size is a
// multiple of 4 words so blobs can be concatenated keeping 16-byte alignment.
//
// header (kHeaderWords words):
//   0 magic, 1 n, 2 ncol (= border_id + 1), 3..5 kw[k] (64-bit words per kind),
//   6..8 aoff[k] (64-bit word offset of kind k in the availability array),
//   9 avail words (64-bit), 10..12 side[k], 13 pair section, 14 desc,
//   15..17 tinfo[k], 18..20 extra[k], 21 initial availability, 22 width,
//   23 height, 24 blob words, 25 max kw, 26 words of the hot prefix
// sections in order: header, pair tables, desc, tinfo, side, extra, initial
// availability; the hot prefix [0, side[0]) is what the DFS reads at every step
// desc (kDescWords = 16 words per level; the first two placed neighbours A and B
// index the level's pair table, further placed neighbours AND their side masks):
//   d0 kw | kind<<8 | nextra<<13 | aoff<<16
//   d1 levelA | levelB<<8 | shiftA<<16 | shiftB<<24 (bit offset of the
//      neighbour's facing colour in its stack word)
//   d2 pair table (word offset): rows [cA][cB][kw] (2 placed), [cA][kw] (1), [kw] (0);
//      entries = frame-side masks & allowed orientations & placed-side masks
//   d3 strideA | strideB<<16 (words per colour step of A and B; 0 when absent)
//   d4 side[kind], d5 tinfo[kind], d6 extra[kind],
//   d7 extra placed sides: side3 | side4<<2 | level3<<8 | level4<<16
//   d8..d11 tinfo[kind] of the levels of neighbours A, B, 3 and 4 (level 0's kind
//      when absent), for a stack that keeps transitions without their colours
//   d12..d15 0
// side[k]: 64-bit [side][colour][kw[k]] masks (colour ncol-1 = frame)
// tinfo[k]: per transition t, colours of the oriented piece (5 bits per side)
//           | has_extra<<20 (its identical mask clears other candidates)
// extra[k]: 64-bit [4*nk][kw[k]] identical masks
struct DeviceTables {
    std::vector<uint32_t> blob;
    uint32_t n = 0, ncol = 0, max_kw = 0;
    std::array<uint32_t, 3> kw{};       // 64-bit words per kind
    std::array<uint32_t, 3> aoff{};     // availability offset of each kind (64-bit words)
    uint32_t avail_words = 0;           // 64-bit words
    std::array<uint32_t, 3> side_off{}, tinfo_off{}, extra_off{};
    uint32_t desc_off = 0, pair_off = 0, init_off = 0;
};

bool build_plan(const PuzzleModel& m, const std::vector<uint32_t>& order,
                std::vector<LevelPlan>& plan, std::string& error);

// Lays the tables out; the header of the blob (first kHeaderWords words) holds
// the offsets so a kernel can read everything from one pointer.
constexpr uint32_t kHeaderWords = 32;
void build_device_tables(const PuzzleModel& m, const std::vector<LevelPlan>& plan,
                         DeviceTables& t);

// Seeded generator (splitmix64 stream; see edge_matching_puzzle_b200/puzzle.py).
void generate_puzzle(uint32_t w, uint32_t h, uint32_t border_colours, uint32_t interior_colours,
                     uint64_t seed, uint8_t* out_colours);

}  // namespace emp
