// Exhaustive backtracker kernels for sm_100a.
//
// Work decomposition (the reference runs one warp on one tree, never split,
// src/CUDA_backtracker.cu:190-214; this build splits the tree):
//   1. prefix expansion, level by level up to the split depth d: one thread per
//      parent prefix walks the candidate set of its next level in the
//      reference's order, applying identical-piece masks exactly as
//      emp_position_strategy::select_piece does; a count pass, an exclusive
//      scan and an emit pass keep the prefixes in the reference's DFS order;
//   2. a persistent DFS kernel: every thread owns one subtree at a time, pops
//      subtree ids from a global queue (one atomic per warp, distributed with
//      ballot/shuffle) and walks it with its stack in shared memory.
//
// Per-thread DFS state is thread-interleaved so that a warp touching "its" entries
// hits 32 distinct banks: 64-bit availability words of the three kinds in shared
// memory and a stack with one entry per level (placements below).  A level's
// candidate words are computed in full, unrolled over a compile-time word count:
// data-dependent loops over words cost more in idle lanes than they save.
// The identical-piece case needs the exact remaining-candidate set of a level
// once a transition with a non-trivial mask has been tried there; such a level
// keeps its set in a per-thread global scratch row (spill) until it is left.
#include "emp_bt.h"
#include "emp_bt_kernels.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

namespace emp {

using namespace dev;

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kMaxExpandDepth = 64;
constexpr uint32_t kMaxAvailWords = 24;   // 64-bit availability words, three kinds
constexpr uint32_t kMaxKindWords = 16;    // 64-bit words of one kind (256 pieces)

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Prefix expansion.  mode 0: count children; mode 1: write children.
__global__ void expand_kernel(BtLaunch P, const uint16_t* __restrict__ parents,
                              const uint32_t* __restrict__ parent_puzzle, uint64_t n_parents,
                              uint32_t level, uint32_t* __restrict__ counts,
                              const uint64_t* __restrict__ offsets, uint16_t* __restrict__ children,
                              uint32_t* __restrict__ child_puzzle, unsigned long long* __restrict__ level_nodes,
                              unsigned long long* __restrict__ level_sols, int mode,
                              const uint8_t* __restrict__ frozen)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_parents;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t pz = parent_puzzle ? parent_puzzle[i] : 0u;
        if (frozen && frozen[pz]) {
            // this puzzle has enough subtrees: carry the prefix over, padded
            if (mode) {
                const uint16_t* pre = parents + i * level;
                uint16_t* c = children + offsets[i] * (level + 1);
                for (uint32_t l = 0; l < level; ++l) c[l] = pre[l];
                c[level] = 0xFFFFu;
                if (child_puzzle) child_puzzle[offsets[i]] = pz;
            } else {
                counts[i] = 1;
            }
            continue;
        }
        const uint32_t* tb = P.tables + P.puzzle_offset[pz];
        const uint32_t n = ldg(tb + H_N), ncol = ldg(tb + H_NCOL), desc_off = ldg(tb + H_DESC);
        uint64_t av[kMaxAvailWords];
        uint32_t stk[kMaxExpandDepth];
        const uint32_t aw = ldg(tb + H_AWORDS), init = ldg(tb + H_INIT);
        for (uint32_t w = 0; w < aw; ++w) av[w] = ldg64(tb + init + 2 * w);
        const uint16_t* pre = parents + i * level;
        for (uint32_t l = 0; l < level; ++l) {
            const LevelDesc d = load_desc(tb, desc_off, l);
            const uint32_t t = pre[l];
            av[d.aoff() + (t >> 6)] &= ~(0xFull << (t & 60u));
            stk[l] = ldg(tb + d.d5 + t) & 0xFFFFFu;
        }
        uint32_t cnt = 0;
        if (level < n) {
            const LevelDesc d = load_desc(tb, desc_off, level);
            const uint32_t kw = d.kw();
            const uint32_t row = d.row(stk[d.level_a()], stk[d.level_b()]);
            uint64_t R[kMaxKindWords];
            for (uint32_t w = 0; w < kw; ++w) R[w] = ldg64(tb + row + 2 * w) & av[d.aoff() + w];
            for (uint32_t j = 0; j < d.nextra(); ++j) {
                const uint32_t sd = d.extra_side(j);
                const uint32_t c = facing_colour(stk[d.extra_level(j)], sd);
                const uint32_t* sm = tb + d.d4 + ((sd * ncol + c) * kw) * 2;
                for (uint32_t w = 0; w < kw; ++w) R[w] &= ldg64(sm + 2 * w);
            }
            uint64_t out = mode ? offsets[i] : 0;
            for (uint32_t w = 0; w < kw; ++w) {
                while (R[w]) {
                    const uint32_t t = w * 64 + __ffsll(R[w]) - 1;
                    if (mode) {
                        uint16_t* c = children + out * (level + 1);
                        for (uint32_t l = 0; l < level; ++l) c[l] = pre[l];
                        c[level] = static_cast<uint16_t>(t);
                        if (child_puzzle) child_puzzle[out] = pz;
                        ++out;
                    }
                    ++cnt;
                    if (level == 0) {  // position 0 keeps its first transition (emp_strategy.h:389)
                        w = kw;
                        break;
                    }
                    if ((ldg(tb + d.d5 + t) >> 20) & 1u) {
                        const uint32_t* ex = tb + d.d6 + t * kw * 2;
                        for (uint32_t ww = 0; ww < kw; ++ww) R[ww] &= ldg64(ex + 2 * ww);
                    } else {
                        R[w] &= ~(1ull << (t & 63));
                    }
                }
            }
        }
        if (!mode) {
            counts[i] = cnt;
            if (cnt) {
                atomicAdd(&level_nodes[pz], (unsigned long long)cnt);
                if (level == n - 1) atomicAdd(&level_sols[pz], (unsigned long long)cnt);
            }
        }
    }
}

// Exclusive scan of u32 counts into u64 offsets: per-block sums, then one
// block scans the block sums, then each block scans its slice.
constexpr uint32_t kScanBlock = 1024;

__device__ uint64_t block_exclusive_scan(uint64_t v, uint64_t* sh, uint64_t& total)
{
    const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    uint64_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
        uint64_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint64_t s = lane < (blockDim.x >> 5) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            uint64_t y = __shfl_up_sync(kFull, s, o);
            if (lane >= (uint32_t)o) s += y;
        }
        sh[lane] = s;
    }
    __syncthreads();
    const uint64_t before = wid ? sh[wid - 1] : 0;
    total = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + x - v;
}

__global__ void scan_block_sums(const uint32_t* __restrict__ in, uint64_t n, uint64_t* __restrict__ sums)
{
    __shared__ uint64_t sh[32];
    const uint64_t i = blockIdx.x * (uint64_t)kScanBlock + threadIdx.x;
    uint64_t total;
    block_exclusive_scan(i < n ? in[i] : 0, sh, total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

__global__ void scan_sums_serial(uint64_t* __restrict__ sums, uint64_t nblocks, uint64_t* __restrict__ grand)
{
    __shared__ uint64_t sh[32];
    uint64_t carry = 0;
    for (uint64_t b0 = 0; b0 < nblocks; b0 += kScanBlock) {
        const uint64_t i = b0 + threadIdx.x;
        const uint64_t v = i < nblocks ? sums[i] : 0;
        uint64_t total;
        const uint64_t ex = block_exclusive_scan(v, sh, total);
        if (i < nblocks) sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) *grand = carry;
}

__global__ void scan_apply(const uint32_t* __restrict__ in, uint64_t n, const uint64_t* __restrict__ sums,
                           uint64_t* __restrict__ out)
{
    __shared__ uint64_t sh[32];
    const uint64_t i = blockIdx.x * (uint64_t)kScanBlock + threadIdx.x;
    uint64_t total;
    const uint64_t ex = block_exclusive_scan(i < n ? in[i] : 0, sh, total);
    if (i < n) out[i] = sums[blockIdx.x] + ex;
}


// ---------------------------------------------------------------------------
// Persistent subtree DFS over work records.
//
// A work record is "prefix t[0..len-1], resume bit `start` at level len"
// (plus the exact remaining set of level len when it is spilled).  The initial
// records are the split-depth prefixes with start 0.  Once a round's queue is
// empty, a thread that spent more than `item_budget` steps on its record hands
// the remaining work back as one record per level that still has candidates
// (the current level from its resume bit, every shallower level from its next
// sibling) for the next round, so a huge subtree spreads over the GPU in a few
// rounds.
//
// record words: [0,1] subtree id (for per-subtree counts), [2] len | start<<16,
// [3] puzzle | spilled<<16 | empty<<17, [4..] transitions (u16 pairs), then
// the remaining set of level len (max_kw 64-bit words as u32 pairs).
//
// Per-thread state, thread-interleaved with a compile-time block size T (a warp
// touching its own entries hits distinct banks and every address is base +
// immediate):
//   av[w*T + tid]  = 64-bit availability words of the three kinds (shared memory)
//   the DFS stack, one entry per level, in one of three placements (StackMode):
//     kStackShared32: shared memory, more<<31 | t<<21 | spilled<<20 | colours of
//                     the placed piece (5 bits per side)
//     kStackShared16: shared memory, more<<15 | spilled<<14 | t: half the bytes, so
//                     more threads fit on an SM; a neighbour's colours are read from
//                     the transition table of its kind instead
//     kStackGlobal32: the 32-bit form in global memory (cached in L1), which leaves
//                     shared memory to the tables and the availability words
//   more: candidates remained after t when it was placed.
struct ThreadItem {
    uint64_t orig;
    const uint32_t* tb;
    uint32_t pz, n, desc_off, L, base, start, spilled;
    bool pop;  // the current level is known to be exhausted: go up without scanning
    uint64_t nodes, sols, steps;
    bool active;
};

// Table access: SM = the plan's single puzzle has its hot tables (header,
// pair tables, level descriptors, transition info) staged in shared memory at
// the start of the block's dynamic shared memory; otherwise every read goes
// through the read-only data path from the global blob.
extern __shared__ __align__(16) uint32_t g_smem[];

template <bool SM>
struct Tab;

template <>
struct Tab<true> {
    static __device__ __forceinline__ uint32_t u32(const ThreadItem&, uint32_t off) { return g_smem[off]; }
    static __device__ __forceinline__ uint64_t u64(const ThreadItem&, uint32_t off)
    {
        return reinterpret_cast<const unsigned long long*>(g_smem)[off >> 1];
    }
    static __device__ __forceinline__ LevelDesc desc(const ThreadItem& s, uint32_t L, bool ext)
    {
        const uint4* d = reinterpret_cast<const uint4*>(g_smem + s.desc_off + kDescWords * L);
        const uint4 a = d[0], b = d[1];
        const uint4 c = ext ? d[2] : make_uint4(0, 0, 0, 0);
        return LevelDesc{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z, c.w};
    }
};

template <>
struct Tab<false> {
    static __device__ __forceinline__ uint32_t u32(const ThreadItem& s, uint32_t off) { return ldg(s.tb + off); }
    static __device__ __forceinline__ uint64_t u64(const ThreadItem& s, uint32_t off) { return ldg64(s.tb + off); }
    static __device__ __forceinline__ LevelDesc desc(const ThreadItem& s, uint32_t L, bool ext)
    {
        return load_desc(s.tb, s.desc_off, L, ext);
    }
};

// The thread's DFS stack (see above).  colour(): the colour that the piece placed
// at level l shows at bit offset `shift` of its colour word (5 bits per side);
// `tinfo` is the transition table of that level's kind (kStackShared16 only).
template <int MODE, int T>
struct Stk;

template <int T>
struct Stk<kStackShared32, T> {
    uint32_t* p;
    __device__ __forceinline__ uint32_t t(uint32_t l) const { return (p[l * T] >> 21) & 0x3FFu; }
    __device__ __forceinline__ bool more(uint32_t l) const { return (p[l * T] >> 31) != 0; }
    __device__ __forceinline__ uint32_t spilled(uint32_t l) const { return (p[l * T] >> 20) & 1u; }
    __device__ __forceinline__ void put(uint32_t l, uint32_t t, bool more, uint32_t spilled, uint32_t ti)
    {
        p[l * T] = (static_cast<uint32_t>(more) << 31) | (t << 21) | (spilled << 20) | (ti & 0xFFFFFu);
    }
    template <bool SM>
    __device__ __forceinline__ uint32_t colour(const ThreadItem&, uint32_t l, uint32_t shift, uint32_t) const
    {
        return (p[l * T] >> shift) & 31u;
    }
    static constexpr bool kNeedsKindTables = false;
};

template <int T>
struct Stk<kStackGlobal32, T> : Stk<kStackShared32, T> {
};

template <int T>
struct Stk<kStackShared16, T> {
    uint16_t* p;
    __device__ __forceinline__ uint32_t t(uint32_t l) const { return p[l * T] & 0x3FFu; }
    __device__ __forceinline__ bool more(uint32_t l) const { return (p[l * T] >> 15) != 0; }
    __device__ __forceinline__ uint32_t spilled(uint32_t l) const { return (p[l * T] >> 14) & 1u; }
    __device__ __forceinline__ void put(uint32_t l, uint32_t t, bool more, uint32_t spilled, uint32_t)
    {
        p[l * T] = static_cast<uint16_t>((static_cast<uint32_t>(more) << 15) | (spilled << 14) | t);
    }
    template <bool SM>
    __device__ __forceinline__ uint32_t colour(const ThreadItem& s, uint32_t l, uint32_t shift, uint32_t tinfo) const
    {
        return (Tab<SM>::u32(s, tinfo + t(l)) >> shift) & 31u;
    }
    static constexpr bool kNeedsKindTables = true;
};

// 64-bit shift left whose amount saturates at 64 (PTX clamps shift amounts)
__device__ __forceinline__ uint64_t shl_sat(uint64_t v, uint32_t n)
{
    uint64_t r;
    asm("shl.b64 %0, %1, %2;" : "=l"(r) : "l"(v), "r"(n));
    return r;
}

__device__ __forceinline__ uint32_t rec_t(const uint32_t* rec, uint32_t l)
{
    return (rec[4 + (l >> 1)] >> (16 * (l & 1))) & 0xFFFFu;
}

template <bool SM, int T, class S>
__device__ __forceinline__ void load_record(const BtLaunch& P, ThreadItem& s, const uint32_t* rec, S& stk,
                                            uint64_t* av, uint64_t* spill)
{
    using TB = Tab<SM>;
    s.orig = static_cast<uint64_t>(rec[0]) | (static_cast<uint64_t>(rec[1]) << 32);
    const uint32_t len = rec[2] & 0xFFFFu;
    s.start = rec[2] >> 16;
    s.pz = rec[3] & 0xFFFFu;
    s.spilled = (rec[3] >> 16) & 1u;
    s.tb = P.tables + P.puzzle_offset[s.pz];
    s.n = TB::u32(s, H_N);
    s.desc_off = TB::u32(s, H_DESC);
    const uint32_t aw = TB::u32(s, H_AWORDS), init = TB::u32(s, H_INIT);
    for (uint32_t w = 0; w < aw; ++w) av[w * T] = ldg64(s.tb + init + 2 * w);
    for (uint32_t l = 0; l < len; ++l) {
        const uint32_t d0 = TB::u32(s, s.desc_off + kDescWords * l);
        const uint32_t d5 = TB::u32(s, s.desc_off + kDescWords * l + 5);
        const uint32_t t = rec_t(rec, l);
        av[((d0 >> 16) + (t >> 6)) * T] &= ~(0xFull << (t & 60u));
        stk.put(l, t, false, 0u, S::kNeedsKindTables ? 0u : TB::u32(s, d5 + t));
    }
    if (s.spilled) {
        const uint32_t* R = rec + P.rec_r_off;
        for (uint32_t w = 0; w < P.max_kw; ++w)
            spill[len * P.max_kw + w] = static_cast<uint64_t>(R[2 * w]) | (static_cast<uint64_t>(R[2 * w + 1]) << 32);
    }
    s.L = len;
    s.base = len;
    s.pop = false;
    s.nodes = 0;
    s.sols = 0;
    s.steps = 0;
    s.active = true;
}

// Candidate words of level L (not yet masked by the resume bit): the level's
// pair-table row (frame sides & the first two placed neighbours) & availability
// & the side masks of further placed neighbours, or the spilled remaining set.
template <int KW, bool SM, int T, class S>
__device__ __forceinline__ void level_candidates(const BtLaunch& P, const ThreadItem& s, const LevelDesc& d,
                                                 uint32_t L, bool spilled, const S& stk, const uint64_t* av,
                                                 const uint64_t* spill, uint64_t* x)
{
    const uint32_t kw = d.kw();
    if (spilled) {
        const uint64_t* sp = spill + L * P.max_kw;
#pragma unroll
        for (int w = 0; w < KW; ++w) x[w] = (uint32_t)w < kw ? sp[w] : 0ull;
        return;
    }
    const uint32_t ca = stk.template colour<SM>(s, d.level_a(), d.shift_a(), d.d8);
    const uint32_t cb = stk.template colour<SM>(s, d.level_b(), d.shift_b(), d.d9);
    const uint32_t row = d.d2 + ca * d.stride_a() + cb * d.stride_b();
    const uint64_t* a = av + d.aoff() * T;
#pragma unroll
    for (int w = 0; w < KW; ++w) x[w] = (uint32_t)w < kw ? Tab<SM>::u64(s, row + 2 * w) & a[w * T] : 0ull;
    if (d.nextra()) {
        const uint32_t ncol = Tab<SM>::u32(s, H_NCOL);
        for (uint32_t j = 0; j < d.nextra(); ++j) {
            const uint32_t sd = d.extra_side(j);
            const uint32_t c = stk.template colour<SM>(s, d.extra_level(j), 5 * ((sd + 2) & 3u), j ? d.d11 : d.d10);
            const uint32_t* sm = s.tb + d.d4 + ((sd * ncol + c) * kw) * 2;
#pragma unroll
            for (int w = 0; w < KW; ++w)
                if ((uint32_t)w < kw) x[w] &= ldg64(sm + 2 * w);
        }
    }
}

// Masks the words below bit `start`, finds the first candidate t and whether
// more candidates follow it.  Returns false when there is none.
template <int KW>
__device__ __forceinline__ bool first_candidate(uint64_t* x, uint32_t start, uint32_t* t, bool* more)
{
    bool found = false;
    uint32_t fw = 0;
    uint64_t fx = 0;
#pragma unroll
    for (int w = 0; w < KW; ++w) {
        const int sh = static_cast<int>(start) - 64 * w;
        x[w] &= shl_sat(~0ull, static_cast<uint32_t>(sh > 0 ? sh : 0));
        if (!found && x[w]) {
            found = true;
            fw = w;
            fx = x[w];
        }
    }
    uint64_t rest = fx & (fx - 1);  // first word without t
#pragma unroll
    for (int w = 0; w < KW; ++w)
        if ((uint32_t)w > fw) rest |= x[w];
    *more = rest != 0;
    *t = fw * 64 + __ffsll(fx) - 1;
    return found;
}

// Goes up one level: gives back the piece placed there and resumes after it.
template <bool SM, int T, class S>
__device__ __forceinline__ void pop_level(ThreadItem& s, const S& stk, uint64_t* av)
{
    --s.L;
    const uint32_t t = stk.t(s.L);
    s.spilled = stk.spilled(s.L);
    s.pop = !stk.more(s.L);
    const uint32_t aoff = Tab<SM>::u32(s, s.desc_off + kDescWords * s.L) >> 16;
    av[(aoff + (t >> 6)) * T] |= 0xFull << (t & 60u);
    s.start = t + 1;
}

// One step of emp_strategy::specific_run (include/emp_strategy.h:352-401)
// inside the thread's record: place the next candidate of the current level, or go
// up one level (without scanning when the level is known to be exhausted).  One pop
// per step: a lane that went up several levels in one step would keep the others of
// its warp idle.  Returns false once the record is exhausted.
template <int KW, bool SM, int T, class S>
__device__ __forceinline__ bool dfs_step(const BtLaunch& P, ThreadItem& s, S& stk, uint64_t* av, uint64_t* spill,
                                         bool* solved)
{
    if (!s.pop) {
        const LevelDesc d = Tab<SM>::desc(s, s.L, S::kNeedsKindTables);
        uint64_t x[KW];
        level_candidates<KW, SM, T>(P, s, d, s.L, s.spilled != 0, stk, av, spill, x);
        uint32_t t;
        bool more;
        if (first_candidate<KW>(x, s.start, &t, &more)) {
            const uint32_t ti = Tab<SM>::u32(s, d.d5 + t);
            if ((ti >> 20) & 1u) {
                // select_piece with an identical mask that clears other candidates
                // (emp_position_strategy.h:197-200): the level keeps its exact
                // remaining set from now on
                const uint32_t kw = d.kw();
                if (!s.spilled) level_candidates<KW, SM, T>(P, s, d, s.L, false, stk, av, spill, x);
                const uint32_t* ex = s.tb + d.d6 + t * kw * 2;
                uint64_t* sp = spill + s.L * P.max_kw;
                uint64_t rest = 0;
#pragma unroll
                for (int w = 0; w < KW; ++w)
                    if ((uint32_t)w < kw) {
                        sp[w] = x[w] & ldg64(ex + 2 * w);
                        const int sh = static_cast<int>(t + 1) - 64 * w;
                        rest |= sp[w] & shl_sat(~0ull, static_cast<uint32_t>(sh > 0 ? sh : 0));
                    }
                more = rest != 0;
                s.spilled = 1;
            }
            uint64_t& aw = av[(d.aoff() + (t >> 6)) * T];
            const uint64_t nib = 0xFull << (t & 60u);
            aw &= ~nib;
            stk.put(s.L, t, more, s.spilled, ti);
            ++s.nodes;
            if (s.L == s.n - 1) {
                // solution: count it, give the piece back, try the next candidate
                ++s.sols;
                *solved = true;
                aw |= nib;
                s.start = t + 1;
                s.pop = !more;
            } else {
                ++s.L;
                s.start = 0;
                s.spilled = 0;
            }
            return true;
        }
    }
    // nothing left at this level: go up
    if (s.L == s.base) return false;
    pop_level<SM, T>(s, stk, av);
    return true;
}

// Keeps the lexicographically smallest solution path of each puzzle: in the
// reference's visiting order (ascending candidate bit at every level) that is
// its first solution.  The lock is held for a few hundred cycles; the wait for
// it is bounded in time (first_lock_wait_ns of %globaltimer) and a thread that
// gives up flags the record as missed, which the host reports as EMP_FIRST_LOST.
template <class S>
__device__ void record_solution(const BtLaunch& P, const ThreadItem& s, const S& stk)
{
    FirstRecord* r = P.first_records + s.pz;
    atomicMin(&P.first_item[s.pz], (unsigned long long)s.orig);
    if (s.orig > *(volatile unsigned long long*)&P.first_item[s.pz]) return;
    const uint64_t give_up = global_ns() + P.first_lock_wait_ns;
    while (atomicCAS(&r->lock, 0u, 1u) != 0u) {
        if (global_ns() > give_up) {
            atomicExch(&r->missed, 1u);
            atomicOr(P.status, EMP_DEV_FIRST_LOST);
            return;
        }
        __nanosleep(64);
    }
    __threadfence();
    bool better = !r->has;
    if (!better) {
        for (uint32_t l = 0; l < s.n; ++l) {
            const uint32_t mine = stk.t(l), theirs = r->t[l];
            if (mine != theirs) {
                better = mine < theirs;
                break;
            }
        }
    }
    if (better) {
        for (uint32_t l = 0; l < s.n; ++l) r->t[l] = static_cast<uint16_t>(stk.t(l));
        r->has = 1;
    }
    __threadfence();
    atomicExch(&r->lock, 0u);
}

__device__ __forceinline__ void account(const BtLaunch& P, const ThreadItem& s)
{
    if (s.nodes) atomicAdd(&P.totals[2 * s.pz], (unsigned long long)s.nodes);
    if (s.sols) atomicAdd(&P.totals[2 * s.pz + 1], (unsigned long long)s.sols);
    if (P.item_nodes) {
        if (s.nodes) atomicAdd(&P.item_nodes[s.orig], (unsigned long long)s.nodes);
        if (s.sols) atomicAdd(&P.item_sols[s.orig], (unsigned long long)s.sols);
    }
}

// Remaining candidates of level l (current level: from s.start unless it is
// known exhausted; shallower levels: after their placed transition, when the
// `more` bit says some remain), with `av` holding level l's entry availability.
template <int KW, bool SM, int T, class S>
__device__ __forceinline__ bool level_has_work(const BtLaunch& P, const ThreadItem& s, uint32_t l, const S& stk,
                                               const uint64_t* av, const uint64_t* spill, uint32_t* start_out,
                                               uint32_t* spilled_out)
{
    uint32_t start, spilled;
    bool maybe;
    if (l == s.L) {
        start = s.start;
        spilled = s.spilled;
        maybe = !s.pop;
    } else {
        start = stk.t(l) + 1;
        spilled = stk.spilled(l);
        maybe = stk.more(l);
    }
    *start_out = start;
    *spilled_out = spilled;
    if (!maybe) return false;
    const LevelDesc d = Tab<SM>::desc(s, l, S::kNeedsKindTables);
    uint64_t x[KW];
    level_candidates<KW, SM, T>(P, s, d, l, spilled != 0, stk, av, spill, x);
    uint32_t t;
    bool more;
    return first_candidate<KW>(x, start, &t, &more);
}

template <bool SM, int T, class S>
__device__ __forceinline__ void toggle_piece(const ThreadItem& s, uint32_t l, const S& stk, uint64_t* av,
                                             bool give_back)
{
    const uint32_t aoff = Tab<SM>::u32(s, s.desc_off + kDescWords * l) >> 16;
    const uint32_t t = stk.t(l);
    if (give_back) av[(aoff + (t >> 6)) * T] |= 0xFull << (t & 60u);
    else av[(aoff + (t >> 6)) * T] &= ~(0xFull << (t & 60u));
}

// Hands the remaining work of the thread's record to the next round: one
// record per level that still holds candidates.  Pass 1 walks the levels from
// the current one up, giving each level's piece back to get that level's entry
// availability, and counts; pass 2 walks back down, writing records and taking
// the pieces again, which leaves the state as it was.  Returns false when the
// output queue is full (the thread then keeps the work).
template <int KW, bool SM, int T, class S>
__device__ bool split_record(const BtLaunch& P, ThreadItem& s, const S& stk, uint64_t* av, const uint64_t* spill)
{
    uint32_t cnt = 0, start, spilled;
    for (uint32_t l = s.L + 1; l-- > s.base;) {
        if (l < s.L) toggle_piece<SM, T>(s, l, stk, av, true);
        cnt += level_has_work<KW, SM, T>(P, s, l, stk, av, spill, &start, &spilled);
    }
    const unsigned long long slot = cnt ? atomicAdd(P.out_tail, (unsigned long long)cnt) : 0ull;
    const bool fits = slot + cnt <= P.out_capacity;
    unsigned long long k = slot;
    for (uint32_t l = s.base; l <= s.L; ++l) {
        if (level_has_work<KW, SM, T>(P, s, l, stk, av, spill, &start, &spilled)) {
            if (fits) {
                uint32_t* rec = P.out_rec + k * P.rec_words;
                rec[0] = static_cast<uint32_t>(s.orig);
                rec[1] = static_cast<uint32_t>(s.orig >> 32);
                rec[2] = l | (start << 16);
                rec[3] = s.pz | (spilled << 16);
                for (uint32_t j = 0; j < l; j += 2) {
                    const uint32_t lo = stk.t(j);
                    const uint32_t hi = j + 1 < l ? stk.t(j + 1) : 0u;
                    rec[4 + (j >> 1)] = lo | (hi << 16);
                }
                if (spilled)
                    for (uint32_t w = 0; w < P.max_kw; ++w) {
                        const uint64_t v = spill[l * P.max_kw + w];
                        rec[P.rec_r_off + 2 * w] = static_cast<uint32_t>(v);
                        rec[P.rec_r_off + 2 * w + 1] = static_cast<uint32_t>(v >> 32);
                    }
            } else if (k < P.out_capacity) {
                P.out_rec[k * P.rec_words + 3] = 1u << 17;  // reserved slot that fits: mark empty
            }
            ++k;
        }
        if (l < s.L) toggle_piece<SM, T>(s, l, stk, av, false);
    }
    return fits;
}

template <int KW, bool SM, int T, int MODE, int kStepsPerFetch>
__global__ void __launch_bounds__(T) dfs_kernel(BtLaunch P)
{
    const uint32_t tid = threadIdx.x, lane = tid & 31;
    if (SM) {
        // stage the single puzzle's hot tables (words [0, smem_tab_words))
        const uint4* src = reinterpret_cast<const uint4*>(P.tables + P.puzzle_offset[0]);
        uint4* dst = reinterpret_cast<uint4*>(g_smem);
        for (uint32_t i = tid; i < P.smem_tab_words / 4; i += T) dst[i] = __ldg(src + i);
        __syncthreads();
    }
    // this thread's columns of the interleaved state: availability words, then
    // (shared placements) the stack
    uint64_t* av = reinterpret_cast<uint64_t*>(g_smem + P.smem_tab_words) + tid;
    Stk<MODE, T> stk;
    if (MODE == kStackGlobal32) {
        *reinterpret_cast<uint32_t**>(&stk.p) = P.stack + (size_t)blockIdx.x * T * P.max_levels + tid;
    } else if (MODE == kStackShared32) {
        *reinterpret_cast<uint32_t**>(&stk.p) = g_smem + P.smem_tab_words + 2 * P.max_avail_words * T + tid;
    } else {
        // warps 2j and 2j+1 share 32 words per level: lane l of the even warp takes the
        // low half of word l, of the odd warp the high half, so the 32 lanes of a warp
        // read 32 banks whatever levels they are at
        *reinterpret_cast<uint16_t**>(&stk.p) =
            reinterpret_cast<uint16_t*>(g_smem + P.smem_tab_words + 2 * P.max_avail_words * T) +
            ((tid & ~63u) | ((tid & 31u) << 1) | ((tid >> 5) & 1u));
    }
    uint64_t* spill = P.spill + (size_t)(blockIdx.x * T + tid) * P.max_levels * P.max_kw;
    ThreadItem s;
    s.active = false;
    bool alive = true;
    bool drained = false;      // warp-uniform: the input queue of this round is empty
    uint32_t iteration = 0;    // warp-uniform loop counter
    uint32_t since_check = 0;  // steps since the last look at the global flags
    // the run's deadline (set by reset_kernel) and this round's record count
    const uint64_t deadline = *(volatile unsigned long long*)&P.ctl->deadline;
    const uint64_t n_in = P.n_in_from_ctl ? *(volatile unsigned long long*)&P.ctl->n_in : P.n_in;
    const uint32_t lt_mask = (1u << lane) - 1u;

    for (;; ++iteration) {
        // ---- work fetch: one atomic per warp, ranks from the ballot ----
        const bool need = alive && !s.active;
        const unsigned needmask = __ballot_sync(kFull, need);
        if (needmask) {
            const uint32_t leader = __ffs(needmask) - 1;
            unsigned long long base = 0;
            if (lane == leader) base = atomicAdd(P.cursor, (unsigned long long)__popc(needmask));
            base = __shfl_sync(kFull, base, leader);
            if (base + __popc(needmask) >= n_in) drained = true;
            if (need) {
                const uint64_t my = base + __popc(needmask & lt_mask);
                if (my < n_in) {
                    const uint32_t* rec = P.in_rec + my * P.rec_words;
                    const uint32_t flags = rec[3];
                    if (!((flags >> 17) & 1u)) {
                        if (*(volatile int*)P.abort_flag) {
                            P.incomplete[flags & 0xFFFFu] = 1u;  // stopped: the record stays unsearched
                        } else {
                            load_record<SM, T>(P, s, rec, stk, av, spill);
                            if (P.stop_at_first && s.orig > *(volatile unsigned long long*)&P.first_item[s.pz])
                                s.active = false;  // a lower subtree of this puzzle holds a solution
                        }
                    }
                } else {
                    alive = false;
                }
            }
        } else if (!drained && (iteration & 31u) == 31u) {
            // every warp learns within 32 rounds of steps that the queue ran dry
            unsigned long long c = 0;
            if (lane == 0) c = *(volatile unsigned long long*)P.cursor;
            c = __shfl_sync(kFull, c, 0);
            drained = c >= n_in;
        }
        if (!__any_sync(kFull, alive)) break;

        // ---- DFS steps: a warp-uniform trip count, lanes without work idle,
        // every step ends reconverged ----
        for (int step = 0; step < kStepsPerFetch; ++step) {
            if (s.active) {
                bool solved = false;
                if (dfs_step<KW, SM, T>(P, s, stk, av, spill, &solved)) {
                    if (solved) {
                        record_solution(P, s, stk);
                        if (P.sols) {
                            const unsigned long long slot = atomicAdd(P.sol_count, 1ull);
                            if (slot < P.sol_capacity) {
                                SolutionRecord* r = P.sols + slot;
                                r->orig = s.orig;
                                r->local = s.nodes;
                                for (uint32_t l = 0; l < s.n; ++l)
                                    r->t[l] = static_cast<uint16_t>(stk.t(l));
                            }
                        }
                        if (P.stop_at_any) {
                            // first solution of the run: note the time and stop every thread
                            atomicCAS(&P.ctl->first_found_ns, 0ull, static_cast<unsigned long long>(global_ns()));
                            atomicExch(P.abort_flag, 1);
                        }
                    }
                } else {
                    account(P, s);
                    s.active = false;
                }
            }
            __syncwarp();
        }
        if (!s.active) continue;
        s.steps += kStepsPerFetch;
        since_check += kStepsPerFetch;

        // ---- once the queue is empty, hand work back for the next round ----
        if (drained && P.item_budget && s.steps >= P.item_budget) {
            if (split_record<KW, SM, T>(P, s, stk, av, spill)) {
                account(P, s);
                s.active = false;
                alive = false;
                continue;
            }
            s.steps = 0;
        }
        // ---- deadline, cancellation and stop-at-first, every 4096 steps ----
        if (since_check >= 4096) {
            since_check = 0;
            bool stop = *(volatile int*)P.abort_flag != 0;
            if (deadline && global_ns() > deadline) {
                stop = true;
                atomicOr(P.status, EMP_DEV_TIMEOUT);
            }
            const bool superseded =
                P.stop_at_first && s.orig > *(volatile unsigned long long*)&P.first_item[s.pz];
            if (superseded || stop) {
                account(P, s);
                s.active = false;
                if (stop) {
                    // the lane stays alive: it goes on taking records only to mark
                    // their puzzles incomplete, so every dropped piece of work is known
                    P.incomplete[s.pz] = 1u;
                    atomicExch(P.abort_flag, 1);
                    atomicOr(P.status, EMP_DEV_ABORTED);
                } else {
                    atomicOr(P.status, EMP_DEV_SUPERSEDED);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Warp-cooperative DFS (stack placement kStackWarp): one record per warp.  The
// warp's stack (32-bit entries as above) sits in shared memory; lane w holds
// word w of each kind's availability in registers and evaluates candidate word
// w of a level, so a try is one ballot over the words and one find-first-set
// in the first non-empty lane (the reference's warp method,
// src/CUDA_backtracker.cu:86-120, over the exhaustive search's candidate sets).
// Kinds up to 32 words (2048 transitions).  Every branch below is warp-uniform:
// the state `s` is the same in all lanes, and values read from memory that
// other warps change (the queue cursor, flags, first-solution records, the
// clock) are taken from lane 0.

struct WarpAv {
    uint64_t k0 = 0, k1 = 0, k2 = 0;  // word `lane` of kinds 0, 1, 2
    __device__ __forceinline__ uint64_t get(uint32_t kind) const { return kind == 0 ? k0 : (kind == 1 ? k1 : k2); }
    __device__ __forceinline__ void flip(uint32_t kind, uint64_t nib, bool give_back)
    {
        // selects, not a reference to the chosen member, so the words stay in registers
        const uint64_t m0 = kind == 0 ? nib : 0ull, m1 = kind == 1 ? nib : 0ull, m2 = kind == 2 ? nib : 0ull;
        if (give_back) {
            k0 |= m0;
            k1 |= m1;
            k2 |= m2;
        } else {
            k0 &= ~m0;
            k1 &= ~m1;
            k2 &= ~m2;
        }
    }
};

using WarpStk = Stk<kStackShared32, 1>;

// this lane's candidate word of level l (not masked by the resume bit)
template <bool SM>
__device__ __forceinline__ uint64_t warp_candidates(const BtLaunch& P, const ThreadItem& s, const LevelDesc& d,
                                                    uint32_t l, bool spilled, const WarpStk& stk, const WarpAv& av,
                                                    const uint64_t* spill, uint32_t lane)
{
    const uint32_t kw = d.kw();
    if (lane >= kw) return 0ull;
    if (spilled) return spill[l * P.max_kw + lane];
    const uint32_t ca = stk.template colour<SM>(s, d.level_a(), d.shift_a(), 0u);
    const uint32_t cb = stk.template colour<SM>(s, d.level_b(), d.shift_b(), 0u);
    uint64_t x = Tab<SM>::u64(s, d.d2 + ca * d.stride_a() + cb * d.stride_b() + 2 * lane) & av.get(d.kind());
    if (d.nextra()) {
        const uint32_t ncol = Tab<SM>::u32(s, H_NCOL);
        for (uint32_t j = 0; j < d.nextra(); ++j) {
            const uint32_t sd = d.extra_side(j);
            const uint32_t c = stk.template colour<SM>(s, d.extra_level(j), 5 * ((sd + 2) & 3u), 0u);
            x &= ldg64(s.tb + d.d4 + ((sd * ncol + c) * kw) * 2 + 2 * lane);
        }
    }
    return x;
}

__device__ __forceinline__ uint64_t from_bit(uint32_t start, uint32_t lane)
{
    const int sh = static_cast<int>(start) - 64 * static_cast<int>(lane);
    return shl_sat(~0ull, static_cast<uint32_t>(sh > 0 ? sh : 0));
}

template <bool SM>
__device__ __forceinline__ void warp_load_record(const BtLaunch& P, ThreadItem& s, const uint32_t* rec, WarpStk& stk,
                                                 WarpAv& av, uint64_t* spill, uint32_t lane)
{
    using TB = Tab<SM>;
    s.orig = static_cast<uint64_t>(rec[0]) | (static_cast<uint64_t>(rec[1]) << 32);
    const uint32_t len = rec[2] & 0xFFFFu;
    s.start = rec[2] >> 16;
    s.pz = rec[3] & 0xFFFFu;
    s.spilled = (rec[3] >> 16) & 1u;
    s.tb = P.tables + P.puzzle_offset[s.pz];
    s.n = TB::u32(s, H_N);
    s.desc_off = TB::u32(s, H_DESC);
    const uint32_t init = TB::u32(s, H_INIT);
    uint64_t w[3];
#pragma unroll
    for (uint32_t k = 0; k < 3; ++k)
        w[k] = lane < TB::u32(s, H_KW + k) ? ldg64(s.tb + init + 2 * (TB::u32(s, H_AOFF + k) + lane)) : 0ull;
    av.k0 = w[0];
    av.k1 = w[1];
    av.k2 = w[2];
    for (uint32_t l = 0; l < len; ++l) {
        const uint32_t kind = (TB::u32(s, s.desc_off + kDescWords * l) >> 8) & 3u;
        const uint32_t t = rec_t(rec, l);
        if (lane == (t >> 6)) av.flip(kind, 0xFull << (t & 60u), false);
    }
    for (uint32_t l = lane; l < len; l += 32) {
        const uint32_t t = rec_t(rec, l);
        stk.put(l, t, false, 0u, TB::u32(s, TB::u32(s, s.desc_off + kDescWords * l + 5) + t));
    }
    if (s.spilled && lane < P.max_kw) {
        const uint32_t* R = rec + P.rec_r_off;
        spill[len * P.max_kw + lane] =
            static_cast<uint64_t>(R[2 * lane]) | (static_cast<uint64_t>(R[2 * lane + 1]) << 32);
    }
    __syncwarp();
    s.L = len;
    s.base = len;
    s.pop = false;
    s.nodes = 0;
    s.sols = 0;
    s.steps = 0;
    s.active = true;
}

// One step of emp_strategy::specific_run (include/emp_strategy.h:352-401) by the
// whole warp: go up one level when the current one is exhausted, then place the
// next candidate of the current level (a dead end marks the level exhausted for
// the next step).  Returns false once the record is exhausted.
template <bool SM>
__device__ __forceinline__ bool warp_step(const BtLaunch& P, ThreadItem& s, WarpStk& stk, WarpAv& av,
                                          uint64_t* spill, uint32_t lane, bool* solved)
{
    if (s.pop) {
        if (s.L == s.base) return false;
        --s.L;
        const uint32_t t = stk.t(s.L);
        s.spilled = stk.spilled(s.L);
        s.pop = !stk.more(s.L);
        const uint32_t kind = (Tab<SM>::u32(s, s.desc_off + kDescWords * s.L) >> 8) & 3u;
        if (lane == (t >> 6)) av.flip(kind, 0xFull << (t & 60u), true);
        s.start = t + 1;
        if (s.pop) return true;
    }
    const LevelDesc d = Tab<SM>::desc(s, s.L, false);
    const uint64_t xu = warp_candidates<SM>(P, s, d, s.L, s.spilled != 0, stk, av, spill, lane);
    const uint64_t x = xu & from_bit(s.start, lane);
    const unsigned bal = __ballot_sync(kFull, x != 0ull);
    if (!bal) {
        s.pop = true;  // dead end: go up at the next step
        return true;
    }
    const uint32_t fw = __ffs(bal) - 1;
    const uint64_t xf = __shfl_sync(kFull, x, fw);
    const uint32_t t = fw * 64 + __ffsll(xf) - 1;
    const unsigned after = fw < 31 ? bal >> (fw + 1) : 0u;
    bool more = (xf & (xf - 1)) != 0ull || after != 0u;
    const uint32_t ti = Tab<SM>::u32(s, d.d5 + t);
    if ((ti >> 20) & 1u) {
        // select_piece with an identical mask (emp_position_strategy.h:197-200): the
        // level keeps its exact remaining set from now on
        const uint32_t kw = d.kw();
        uint64_t sp = 0;
        if (lane < kw) {
            sp = (s.spilled ? x : xu) & ldg64(s.tb + d.d6 + t * kw * 2 + 2 * lane);
            spill[s.L * P.max_kw + lane] = sp;
        }
        more = __ballot_sync(kFull, (sp & from_bit(t + 1, lane)) != 0ull) != 0u;
        s.spilled = 1;
    }
    const uint32_t kind = d.kind();
    const uint64_t nib = 0xFull << (t & 60u);
    if (lane == (t >> 6)) av.flip(kind, nib, false);
    if (lane == 0) stk.put(s.L, t, more, s.spilled, ti);
    __syncwarp();
    ++s.nodes;
    if (s.L == s.n - 1) {
        // solution: count it, give the piece back, try the next candidate
        ++s.sols;
        *solved = true;
        if (lane == (t >> 6)) av.flip(kind, nib, true);
        s.start = t + 1;
        s.pop = !more;
    } else {
        ++s.L;
        s.start = 0;
        s.spilled = 0;
    }
    return true;
}

// split_record for a warp: the same records, written by the lanes together
template <bool SM>
__device__ __forceinline__ bool warp_level_has_work(const BtLaunch& P, const ThreadItem& s, uint32_t l,
                                                    const WarpStk& stk, const WarpAv& av, const uint64_t* spill,
                                                    uint32_t lane, uint32_t* start_out, uint32_t* spilled_out)
{
    uint32_t start, spilled;
    bool maybe;
    if (l == s.L) {
        start = s.start;
        spilled = s.spilled;
        maybe = !s.pop;
    } else {
        start = stk.t(l) + 1;
        spilled = stk.spilled(l);
        maybe = stk.more(l);
    }
    *start_out = start;
    *spilled_out = spilled;
    if (!maybe) return false;
    const LevelDesc d = Tab<SM>::desc(s, l, false);
    const uint64_t x = warp_candidates<SM>(P, s, d, l, spilled != 0, stk, av, spill, lane) & from_bit(start, lane);
    return __ballot_sync(kFull, x != 0ull) != 0u;
}

template <bool SM>
__device__ __forceinline__ void warp_toggle_piece(const ThreadItem& s, uint32_t l, const WarpStk& stk, WarpAv& av,
                                                  uint32_t lane, bool give_back)
{
    const uint32_t kind = (Tab<SM>::u32(s, s.desc_off + kDescWords * l) >> 8) & 3u;
    const uint32_t t = stk.t(l);
    if (lane == (t >> 6)) av.flip(kind, 0xFull << (t & 60u), give_back);
}

template <bool SM>
__device__ bool warp_split_record(const BtLaunch& P, ThreadItem& s, const WarpStk& stk, WarpAv& av,
                                  const uint64_t* spill, uint32_t lane)
{
    uint32_t cnt = 0, start, spilled;
    for (uint32_t l = s.L + 1; l-- > s.base;) {
        if (l < s.L) warp_toggle_piece<SM>(s, l, stk, av, lane, true);
        cnt += warp_level_has_work<SM>(P, s, l, stk, av, spill, lane, &start, &spilled);
    }
    unsigned long long slot = 0;
    if (lane == 0 && cnt) slot = atomicAdd(P.out_tail, (unsigned long long)cnt);
    slot = __shfl_sync(kFull, slot, 0);
    const bool fits = slot + cnt <= P.out_capacity;
    unsigned long long k = slot;
    for (uint32_t l = s.base; l <= s.L; ++l) {
        if (warp_level_has_work<SM>(P, s, l, stk, av, spill, lane, &start, &spilled)) {
            if (fits) {
                uint32_t* rec = P.out_rec + k * P.rec_words;
                if (lane == 0) {
                    rec[0] = static_cast<uint32_t>(s.orig);
                    rec[1] = static_cast<uint32_t>(s.orig >> 32);
                    rec[2] = l | (start << 16);
                    rec[3] = s.pz | (spilled << 16);
                }
                for (uint32_t j = 2 * lane; j < l; j += 64) {
                    const uint32_t lo = stk.t(j);
                    const uint32_t hi = j + 1 < l ? stk.t(j + 1) : 0u;
                    rec[4 + (j >> 1)] = lo | (hi << 16);
                }
                if (spilled && lane < P.max_kw) {
                    const uint64_t v = spill[l * P.max_kw + lane];
                    rec[P.rec_r_off + 2 * lane] = static_cast<uint32_t>(v);
                    rec[P.rec_r_off + 2 * lane + 1] = static_cast<uint32_t>(v >> 32);
                }
            } else if (k < P.out_capacity && lane == 0) {
                P.out_rec[k * P.rec_words + 3] = 1u << 17;  // reserved slot that fits: mark empty
            }
            ++k;
        }
        if (l < s.L) warp_toggle_piece<SM>(s, l, stk, av, lane, false);
    }
    return fits;
}

template <bool SM, int T, int kStepsPerFetch>
__global__ void __launch_bounds__(T) dfs_warp_kernel(BtLaunch P)
{
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (SM) {
        const uint4* src = reinterpret_cast<const uint4*>(P.tables + P.puzzle_offset[0]);
        uint4* dst = reinterpret_cast<uint4*>(g_smem);
        for (uint32_t i = tid; i < P.smem_tab_words / 4; i += T) dst[i] = __ldg(src + i);
        __syncthreads();
    }
    WarpStk stk;
    stk.p = g_smem + P.smem_tab_words + warp * P.max_levels;
    const uint64_t gwarp = static_cast<uint64_t>(blockIdx.x) * (T / 32) + warp;
    uint64_t* spill = P.spill + gwarp * P.max_levels * P.max_kw;
    ThreadItem s;
    s.active = false;
    WarpAv av;
    bool drained = false;
    uint32_t since_check = 0;
    const uint64_t deadline = *(volatile unsigned long long*)&P.ctl->deadline;
    const uint64_t n_in = P.n_in_from_ctl ? *(volatile unsigned long long*)&P.ctl->n_in : P.n_in;

    for (;;) {
        if (!s.active) {
            // ---- work fetch: one record per warp ----
            unsigned long long my = 0;
            int abort = 0;
            if (lane == 0) {
                my = atomicAdd(P.cursor, 1ull);
                abort = *(volatile int*)P.abort_flag;
            }
            my = __shfl_sync(kFull, my, 0);
            abort = __shfl_sync(kFull, abort, 0);
            if (my >= n_in) break;
            drained = my + 1 >= n_in;
            const uint32_t* rec = P.in_rec + my * P.rec_words;
            const uint32_t flags = rec[3];
            if ((flags >> 17) & 1u) continue;  // an empty slot
            if (abort) {
                if (lane == 0) P.incomplete[flags & 0xFFFFu] = 1u;  // stopped: the record stays unsearched
                continue;
            }
            warp_load_record<SM>(P, s, rec, stk, av, spill, lane);
            if (P.stop_at_first) {
                unsigned long long f = 0;
                if (lane == 0) f = *(volatile unsigned long long*)&P.first_item[s.pz];
                if (s.orig > __shfl_sync(kFull, f, 0)) s.active = false;  // a lower subtree holds a solution
            }
            continue;
        }
        for (int step = 0; step < kStepsPerFetch; ++step) {
            bool solved = false;
            if (!warp_step<SM>(P, s, stk, av, spill, lane, &solved)) {
                if (lane == 0) account(P, s);
                s.active = false;
                break;
            }
            if (solved) {
                if (lane == 0) record_solution(P, s, stk);
                if (P.sols) {
                    unsigned long long slot = 0;
                    if (lane == 0) slot = atomicAdd(P.sol_count, 1ull);
                    slot = __shfl_sync(kFull, slot, 0);
                    if (slot < P.sol_capacity) {
                        SolutionRecord* r = P.sols + slot;
                        if (lane == 0) {
                            r->orig = s.orig;
                            r->local = s.nodes;
                        }
                        for (uint32_t l = lane; l < s.n; l += 32) r->t[l] = static_cast<uint16_t>(stk.t(l));
                    }
                }
                if (P.stop_at_any && lane == 0) {
                    atomicCAS(&P.ctl->first_found_ns, 0ull, static_cast<unsigned long long>(global_ns()));
                    atomicExch(P.abort_flag, 1);
                }
                __syncwarp();
            }
        }
        if (!s.active) continue;
        s.steps += kStepsPerFetch;
        since_check += kStepsPerFetch;

        // ---- once the queue is empty, hand work back for the next round ----
        if (!drained && (since_check & 1023u) == 0u) {
            unsigned long long c = 0;
            if (lane == 0) c = *(volatile unsigned long long*)P.cursor;
            drained = __shfl_sync(kFull, c, 0) >= n_in;
        }
        if (drained && P.item_budget && s.steps >= P.item_budget) {
            if (warp_split_record<SM>(P, s, stk, av, spill, lane)) {
                if (lane == 0) account(P, s);
                s.active = false;
                break;  // this warp's work went back to the queue; the queue is empty
            }
            s.steps = 0;
        }
        // ---- deadline, cancellation and stop-at-first, every 4096 steps ----
        if (since_check >= 4096) {
            since_check = 0;
            int flags = 0;
            if (lane == 0) {
                if (*(volatile int*)P.abort_flag != 0) flags |= 1;
                if (deadline && global_ns() > deadline) flags |= 2;
                if (P.stop_at_first && s.orig > *(volatile unsigned long long*)&P.first_item[s.pz]) flags |= 4;
            }
            flags = __shfl_sync(kFull, flags, 0);
            const bool stop = (flags & 3) != 0;
            if (stop || (flags & 4)) {
                if (lane == 0) {
                    account(P, s);
                    if (flags & 2) atomicOr(P.status, EMP_DEV_TIMEOUT);
                    if (stop) {
                        // the warp goes on taking records only to mark their puzzles
                        // incomplete, so every dropped piece of work is known
                        P.incomplete[s.pz] = 1u;
                        atomicExch(P.abort_flag, 1);
                        atomicOr(P.status, EMP_DEV_ABORTED);
                    } else {
                        atomicOr(P.status, EMP_DEV_SUPERSEDED);
                    }
                }
                s.active = false;
            }
        }
    }
}

__global__ void reset_kernel(BtLaunch P, uint32_t n_puzzles)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) {
        P.abort_flag[0] = 0;
        P.status[0] = 0;
        const unsigned long long now = global_ns();
        P.ctl->deadline = P.timeout_ns ? now + P.timeout_ns : 0ull;
        P.ctl->start_ns = now;
        P.ctl->first_found_ns = 0;
        // a run whose first round takes its record count from the device starts from
        // the count make_records left (graph runs, reused across selections)
        P.ctl->n_in = P.n_in_from_ctl ? P.ctl->n_init : 0ull;
        P.ctl->rounds = 0;
        P.ctl->records_in = P.n_in_from_ctl ? P.ctl->n_init : P.n_in;
        P.ctl->records_out = 0;
    }
    if (i < n_puzzles) {
        P.incomplete[i] = 0;
        P.totals[2 * i] = 0;
        P.totals[2 * i + 1] = 0;
        P.first_item[i] = ~0ull;
        P.first_records[i].lock = P.first_lock_init;
        P.first_records[i].missed = 0;
        P.first_records[i].has = 0;
    }
}

// Initial records from split-depth prefixes (a strided selection of them).
__global__ void make_records(const uint16_t* __restrict__ prefixes, const uint32_t* __restrict__ prefix_puzzle,
                             uint32_t depth, uint64_t first, uint64_t stride, uint64_t count, uint32_t rec_words,
                             uint32_t* __restrict__ rec, const uint32_t* __restrict__ puzzle_depth, BtRunCtl* ctl)
{
    if (ctl && blockIdx.x == 0 && threadIdx.x == 0) ctl->n_init = count;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < count;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j = first + i * stride;
        uint32_t* r = rec + i * rec_words;
        r[0] = static_cast<uint32_t>(i);
        r[1] = static_cast<uint32_t>(i >> 32);
        const uint32_t pz = prefix_puzzle[j];
        const uint32_t len = puzzle_depth ? puzzle_depth[pz] : depth;
        r[2] = len;
        r[3] = pz;
        const uint16_t* p = prefixes + j * depth;
        for (uint32_t l = 0; l < len; l += 2) r[4 + (l >> 1)] = p[l] | (l + 1 < len ? (uint32_t)p[l + 1] << 16 : 0u);
    }
}

// Graph runs: turns the records handed back by the round that just ended into
// the next round's input and decides whether the loop goes on.
__global__ void round_advance_kernel(BtLaunch P, cudaGraphConditionalHandle loop, uint32_t max_rounds)
{
    BtRunCtl* c = P.ctl;
    const unsigned long long tail = *P.out_tail;
    const unsigned long long n = tail < P.out_capacity ? tail : P.out_capacity;
    c->rounds += 1;
    c->records_out += n;
    c->records_in += n;
    c->n_in = n;
    *P.cursor = 0;
    *P.out_tail = 0;
    cudaGraphSetConditional(loop, (n && c->rounds < max_rounds) ? 1u : 0u);
}

// Graph runs: copies the round's input records (ctl->n_in of them) to the input queue.
__global__ void round_copy_kernel(BtLaunch P, uint4* __restrict__ dst, const uint4* __restrict__ src)
{
    const uint64_t words = *(volatile unsigned long long*)&P.ctl->n_in * P.rec_words;
    const uint64_t vec = words / 4;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < vec; i += (uint64_t)gridDim.x * blockDim.x)
        dst[i] = src[i];
    const uint64_t tail = vec * 4 + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (tail < words)
        reinterpret_cast<uint32_t*>(dst)[tail] = reinterpret_cast<const uint32_t*>(src)[tail];
}

// One block per solution: thread 0 binary-searches the level arrays, the block
// sums the counts of the subtrees before the solution's own.
__global__ void solution_index_kernel(const SolutionRecord* __restrict__ sols, const uint16_t* const* level_prefixes,
                                      const uint64_t* __restrict__ level_counts, uint32_t depth,
                                      const unsigned long long* __restrict__ item_nodes, unsigned long long* out)
{
    __shared__ unsigned long long part[256];
    const SolutionRecord& s = sols[blockIdx.x];
    unsigned long long acc = 0;
    for (unsigned long long j = threadIdx.x; j < s.orig; j += blockDim.x) acc += item_nodes[j];
    part[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t w = blockDim.x / 2; w; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        unsigned long long exp_before = 0;
        for (uint32_t L = 1; L <= depth; ++L) {
            // level arrays hold the prefixes of length L in lexicographic order:
            // count those at or before the solution's first L transitions
            const uint16_t* a = level_prefixes[L];
            uint64_t lo = 0, hi = level_counts[L];
            while (lo < hi) {
                const uint64_t mid = (lo + hi) / 2;
                int cmp = 0;
                for (uint32_t l = 0; l < L && !cmp; ++l) {
                    const uint16_t x = a[mid * L + l];
                    cmp = x < s.t[l] ? -1 : (x > s.t[l] ? 1 : 0);
                }
                if (cmp <= 0) lo = mid + 1;
                else hi = mid;
            }
            exp_before += lo;
        }
        out[blockIdx.x] = exp_before + part[0] + s.local;
    }
}

// Prefix (transitions) of selected subtree `i`, for the host.
__global__ void record_prefix(const uint32_t* __restrict__ rec, uint32_t rec_words, uint64_t i, uint16_t* out)
{
    const uint32_t* r = rec + i * rec_words;
    const uint32_t len = r[2] & 0xFFFFu;
    for (uint32_t l = threadIdx.x; l < 256; l += blockDim.x) out[l] = l < len ? static_cast<uint16_t>(rec_t(r, l)) : 0xFFFFu;
}

template <int KW, int T, int MODE>
const void* dfs_symbol(bool sm)
{
    return sm ? reinterpret_cast<const void*>(&dfs_kernel<KW, true, T, MODE, 32>)
              : reinterpret_cast<const void*>(&dfs_kernel<KW, false, T, MODE, 32>);
}

// Word counts with a kernel: a puzzle runs with the smallest one that holds its
// widest kind (8x8: 3 words, 12x12: 7 -> 8, 16x16: 13 -> 16).
template <int T, int MODE>
const void* dfs_symbol_kw(uint32_t max_kw, bool sm)
{
    if (max_kw <= 1) return dfs_symbol<1, T, MODE>(sm);
    if (max_kw <= 2) return dfs_symbol<2, T, MODE>(sm);
    if (max_kw <= 3) return dfs_symbol<3, T, MODE>(sm);
    if (max_kw <= 4) return dfs_symbol<4, T, MODE>(sm);
    if (max_kw <= 8) return dfs_symbol<8, T, MODE>(sm);
    if (max_kw <= 16) return dfs_symbol<16, T, MODE>(sm);
    return nullptr;
}

template <int T>
const void* dfs_symbol_mode(uint32_t max_kw, bool sm, int mode)
{
    switch (mode) {
        case kStackShared32: return dfs_symbol_kw<T, kStackShared32>(max_kw, sm);
        case kStackShared16: return dfs_symbol_kw<T, kStackShared16>(max_kw, sm);
        case kStackGlobal32: return dfs_symbol_kw<T, kStackGlobal32>(max_kw, sm);
        case kStackWarp:
            if (max_kw > 32) return nullptr;
            return sm ? reinterpret_cast<const void*>(&dfs_warp_kernel<true, T, 32>)
                      : reinterpret_cast<const void*>(&dfs_warp_kernel<false, T, 32>);
        default: return nullptr;
    }
}

const void* dfs_symbol_for(uint32_t max_kw, bool sm, uint32_t threads, int mode)
{
    switch (threads) {
        case 128: return dfs_symbol_mode<128>(max_kw, sm, mode);
        case 256: return dfs_symbol_mode<256>(max_kw, sm, mode);
        case 512: return dfs_symbol_mode<512>(max_kw, sm, mode);
        default: return nullptr;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// host launchers

cudaError_t launch_expand(const BtLaunch& P, const uint16_t* parents, const uint32_t* parent_puzzle,
                          uint64_t n_parents, uint32_t level, uint32_t* counts, const uint64_t* offsets,
                          uint16_t* children, uint32_t* child_puzzle, unsigned long long* level_nodes,
                          unsigned long long* level_sols, int mode, cudaStream_t stream)
{
    if (!n_parents) return cudaSuccess;
    const uint32_t threads = 128;
    const uint64_t blocks = std::min<uint64_t>((n_parents + threads - 1) / threads, 148ull * 64);
    expand_kernel<<<(unsigned)blocks, threads, 0, stream>>>(P, parents, parent_puzzle, n_parents, level, counts,
                                                            offsets, children, child_puzzle, level_nodes,
                                                            level_sols, mode, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_expand_frozen(const BtLaunch& P, const uint16_t* parents, const uint32_t* parent_puzzle,
                                 uint64_t n_parents, uint32_t level, uint32_t* counts, const uint64_t* offsets,
                                 uint16_t* children, uint32_t* child_puzzle, unsigned long long* level_nodes,
                                 unsigned long long* level_sols, int mode, const uint8_t* frozen,
                                 cudaStream_t stream)
{
    if (!n_parents) return cudaSuccess;
    const uint32_t threads = 128;
    const uint64_t blocks = std::min<uint64_t>((n_parents + threads - 1) / threads, 148ull * 64);
    expand_kernel<<<(unsigned)blocks, threads, 0, stream>>>(P, parents, parent_puzzle, n_parents, level, counts,
                                                            offsets, children, child_puzzle, level_nodes,
                                                            level_sols, mode, frozen);
    return cudaGetLastError();
}

cudaError_t launch_round_advance(const BtLaunch& P, cudaGraphConditionalHandle loop, uint32_t max_rounds,
                                 cudaStream_t stream)
{
    round_advance_kernel<<<1, 1, 0, stream>>>(P, loop, max_rounds);
    return cudaGetLastError();
}

cudaError_t launch_round_copy(const BtLaunch& P, uint32_t* dst, const uint32_t* src, cudaStream_t stream)
{
    // queues are allocated by cudaMalloc (256-byte aligned): 16-byte vector copies
    round_copy_kernel<<<148 * 4, 256, 0, stream>>>(P, reinterpret_cast<uint4*>(dst),
                                                   reinterpret_cast<const uint4*>(src));
    return cudaGetLastError();
}

cudaError_t launch_scan(const uint32_t* counts, uint64_t n, uint64_t* offsets, uint64_t* block_sums,
                        uint64_t* grand_total, cudaStream_t stream)
{
    if (!n) return cudaMemsetAsync(grand_total, 0, sizeof(uint64_t), stream);
    const uint64_t nb = (n + kScanBlock - 1) / kScanBlock;
    scan_block_sums<<<(unsigned)nb, kScanBlock, 0, stream>>>(counts, n, block_sums);
    scan_sums_serial<<<1, kScanBlock, 0, stream>>>(block_sums, nb, grand_total);
    scan_apply<<<(unsigned)nb, kScanBlock, 0, stream>>>(counts, n, block_sums, offsets);
    return cudaGetLastError();
}

uint64_t scan_block_sum_words(uint64_t n) { return (n + kScanBlock - 1) / kScanBlock + 1; }

size_t dfs_smem_bytes(uint32_t max_levels, uint32_t max_avail_words, uint32_t threads, uint32_t tab_words,
                      int stack_mode)
{
    if (stack_mode == kStackWarp)  // one stack per warp; availability in registers
        return static_cast<size_t>(tab_words) * sizeof(uint32_t) +
               static_cast<size_t>(threads / 32) * max_levels * sizeof(uint32_t);
    const size_t stack = stack_mode == kStackShared32 ? 4 : (stack_mode == kStackShared16 ? 2 : 0);
    return static_cast<size_t>(tab_words) * sizeof(uint32_t) +
           static_cast<size_t>(max_avail_words) * sizeof(uint64_t) * threads +
           ((static_cast<size_t>(max_levels) * stack * threads + 3) & ~size_t(3));
}

uint32_t record_words(uint32_t max_levels, uint32_t max_kw) { return 4 + (max_levels + 1) / 2 + 2 * max_kw; }

const void* dfs_kernel_symbol(uint32_t max_kw, bool smem_tables, uint32_t threads, int stack_mode)
{
    return dfs_symbol_for(max_kw, smem_tables, threads, stack_mode);
}

cudaError_t launch_dfs(const BtLaunch& P, uint32_t blocks, uint32_t threads, cudaStream_t stream)
{
    const void* fn = dfs_symbol_for(P.max_kw, P.smem_tab_words != 0, threads, P.stack_mode);
    if (!fn) return cudaErrorInvalidValue;
    const size_t smem = dfs_smem_bytes(P.max_levels, P.max_avail_words, threads, P.smem_tab_words, P.stack_mode);
    void* args[] = {const_cast<BtLaunch*>(&P)};
    return cudaLaunchKernel(fn, dim3(blocks), dim3(threads), args, smem, stream);
}

cudaError_t launch_bt_reset(const BtLaunch& P, uint32_t n_puzzles, cudaStream_t stream)
{
    reset_kernel<<<(n_puzzles + 255) / 256, 256, 0, stream>>>(P, n_puzzles);
    return cudaGetLastError();
}

cudaError_t launch_make_records(const uint16_t* prefixes, const uint32_t* prefix_puzzle, uint32_t depth,
                                uint64_t first, uint64_t stride, uint64_t count, uint32_t rec_words, uint32_t* rec,
                                cudaStream_t stream, const uint32_t* puzzle_depth, BtRunCtl* ctl)
{
    if (!count && !ctl) return cudaSuccess;
    const uint64_t blocks = std::max<uint64_t>(1, std::min<uint64_t>((count + 255) / 256, 148ull * 32));
    make_records<<<(unsigned)blocks, 256, 0, stream>>>(prefixes, prefix_puzzle, depth, first, stride, count,
                                                       rec_words, rec, puzzle_depth, ctl);
    return cudaGetLastError();
}

cudaError_t launch_solution_index(const SolutionRecord* sols, uint64_t nsol, const uint16_t* const* level_prefixes,
                                  const uint64_t* level_counts, uint32_t depth, const unsigned long long* item_nodes,
                                  unsigned long long* out, cudaStream_t stream)
{
    if (!nsol) return cudaSuccess;
    solution_index_kernel<<<static_cast<unsigned>(nsol), 256, 0, stream>>>(sols, level_prefixes, level_counts, depth,
                                                                           item_nodes, out);
    return cudaGetLastError();
}

cudaError_t launch_record_prefix(const uint32_t* rec, uint32_t rec_words, uint64_t i, uint16_t* out,
                                 cudaStream_t stream)
{
    record_prefix<<<1, 64, 0, stream>>>(rec, rec_words, i, out);
    return cudaGetLastError();
}

}  // namespace emp
