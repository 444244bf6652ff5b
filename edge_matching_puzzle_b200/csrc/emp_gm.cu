// Glutton max search for sm_100a.
//
// The method is the reference's CUDA_glutton_max kernel
// (include/CUDA_glutton_max.h:1522-1637): at every level
//   1. remove_invalid_transitions (:745-954): drop every candidate (position,
//      piece, orientation) whose trial placement empties a free position or
//      leaves an available piece with nowhere to go, until nothing changes;
//   2. get_best_candidate (:1010-1301): score every remaining candidate by its
//      trial (total remaining bits over positions and pieces, then
//      (max << 16) + min), keep the first maximum in (info, word, bit) order,
//      the last candidate at the last level;
//   3. apply_best_candidate (:1306-1476): clear its bit, build the next level,
//      push, apply the colour constraints of its sides;
// popping when a level fails (CUDA_glutton_max_stack.h:437-522).
//
// B200 design: one 1024-thread block per search keeps the level in shared
// memory together with per-level statistics -- nibble counts N[j][q] of piece
// q at free position j, bit totals A[j], per-piece sums S[q] and, per piece,
// the six smallest and six largest A[j]-N[j][q].  A trial then only scans the
// (at most four) colour-constrained neighbour positions word by word; every
// other position contributes A[j]-N[j][p] and the piece counts follow from
// S[q]-N[i][q] minus what the neighbours lost.  This gives the reference's
// (valid, total, min, max) exactly at a fraction of its cost.  Step 1 runs as
// Jacobi passes (all candidates against the same level, then all removals):
// validity only gets harder as bits disappear, so the passes reach the same
// greatest fixpoint as the reference's in-place sweep, and they empty a
// position exactly when the reference's sweep does.
#include "emp_gm.h"

#include <cuda_runtime.h>

namespace emp {

namespace {

constexpr int kThreads = 1024;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint64_t kBarrierWaitNs = 5000000000ull;  // 5 s: far beyond one validity pass

struct GmSmem {
    uint32_t X[256][32];       // infos of the current level
    uint32_t inval[256][32];   // candidates found invalid in this pass
    uint8_t N[256][256];       // N[j][q]: orientations of piece q left at info j
    uint32_t lo[256][6];       // per piece q: six smallest (A[j]-N[j][q]) << 16 | j, ~0 empty
    uint32_t hi[256][6];       // per piece q: six largest (A[j]-N[j][q]+1) << 16 | j, 0 empty
    uint32_t lo2[256][6];      // the same two lists over the second half of the infos,
    uint32_t hi2[256][6];      // merged into lo / hi at the end of each statistics pass
    uint16_t S2[256];
    uint32_t partA[32];        // per warp: bits of its infos, and whether one is empty
    uint32_t partE[32];
    uint32_t cc[32][4][32];    // colour constraints
    uint16_t A[256];           // bits of info j
    uint16_t S[256];           // sum over j of N[j][q]
    uint8_t pieces[256][4];
    uint32_t position_index[256];
    uint32_t info_index[256];
    uint32_t played[256];      // this block's copy of the played stack
    uint32_t avail[8];
    unsigned long long warp_key[32];
    uint32_t warp_order[32];
    uint32_t warp_trials[32];
    uint32_t sumA;
    uint32_t any_invalid;
    uint32_t any_empty;
    uint32_t next_info;
    uint32_t best_order;       // chosen candidate: info << 10 | word << 5 | bit; ~0 none
    uint32_t level, new_level, pop_index, stop, apply_failed;
};

__device__ __forceinline__ uint32_t tri_base(uint32_t S, uint32_t L)
{
    return (S * (S + 1) - (S - L) * (S - L + 1)) / 2;
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t warp_sum(uint32_t v)
{
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}
__device__ __forceinline__ uint32_t warp_min(uint32_t v)
{
    for (int o = 16; o; o >>= 1) v = min(v, __shfl_xor_sync(kFull, v, o));
    return v;
}
__device__ __forceinline__ uint32_t warp_max(uint32_t v)
{
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(kFull, v, o));
    return v;
}

// get_best_candidate's preference (include/CUDA_glutton_max.h:1196-1295): is candidate
// (k, o) better than (k0, o0)?  order ~0 is "none".  Orders are distinct, so this is a
// strict total order and any reduction tree finds the same best candidate.
__device__ __forceinline__ bool better_candidate(unsigned long long k, uint32_t o, unsigned long long k0, uint32_t o0,
                                                 bool last_level)
{
    if (o == ~0u) return false;
    if (o0 == ~0u) return true;
    return last_level ? o > o0 : (k > k0 || (k == k0 && o < o0));
}

// every lane ends with the warp's best (k, o)
__device__ __forceinline__ void warp_best(unsigned long long& k, uint32_t& o, bool last_level)
{
    for (int d = 16; d; d >>= 1) {
        const unsigned long long k2 = __shfl_xor_sync(kFull, k, d);
        const uint32_t o2 = __shfl_xor_sync(kFull, o, d);
        if (better_candidate(k2, o2, k, o, last_level)) {
            k = k2;
            o = o2;
        }
    }
}

__device__ __forceinline__ bool piece_available(const GmSmem& sm, uint32_t q)
{
    return (sm.avail[q >> 5] >> (q & 31)) & 1u;
}

// Six smallest (ASC) or largest of A[j]-N[j][q] over infos j in [j0, j1) for piece q,
// as sorted lists of distinct keys (the info index in the low bits).
template <bool ASC>
__device__ __forceinline__ void extreme_six(const GmSmem& sm, uint32_t q, uint32_t j0, uint32_t j1, uint32_t* best,
                                            uint32_t* sum)
{
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < 6; ++k) best[k] = ASC ? ~0u : 0u;
    for (uint32_t j = j0; j < j1; ++j) {
        const uint32_t n = sm.N[j][q];
        s += n;
        uint32_t v = ((sm.A[j] - n + (ASC ? 0u : 1u)) << 16) | j;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const uint32_t keep = ASC ? min(best[k], v) : max(best[k], v);
            v = ASC ? max(best[k], v) : min(best[k], v);
            best[k] = keep;
        }
    }
    *sum = s;
}

// the first six of two sorted six-lists (ascending for ASC, else descending)
template <bool ASC>
__device__ __forceinline__ void merge_six(uint32_t* a, const uint32_t* b)
{
    uint32_t out[6];
    int i = 0, k = 0;
#pragma unroll
    for (int o = 0; o < 6; ++o) {
        const uint32_t x = a[i < 6 ? i : 5], y = b[k < 6 ? k : 5];
        const bool take_a = k >= 6 || (i < 6 && (ASC ? x < y : x > y));
        out[o] = take_a ? x : y;
        i += take_a;
        k += !take_a;
    }
#pragma unroll
    for (int o = 0; o < 6; ++o) a[o] = out[o];
}

// Per-pass statistics of the current level (block-wide).  The per-piece scans run in
// four groups of 256 threads (six smallest / six largest, each over one half of the
// infos), merged afterwards; the lists are sets of distinct keys, so the halves and
// the merge give the lists of one scan over all infos.
__device__ void level_statistics(GmSmem& sm, uint32_t nb, uint32_t tid)
{
    const uint32_t lane = tid & 31, warp = tid >> 5;
    uint32_t asum = 0, aempty = 0;
    for (uint32_t j = warp; j < nb; j += kThreads / 32) {
        const uint32_t word = sm.X[j][lane];
        uint32_t packed0 = 0, packed1 = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            packed0 |= static_cast<uint32_t>(__popc((word >> (4 * k)) & 0xFu)) << (8 * k);
            packed1 |= static_cast<uint32_t>(__popc((word >> (4 * (k + 4))) & 0xFu)) << (8 * k);
        }
        reinterpret_cast<uint32_t*>(sm.N[j])[2 * lane] = packed0;
        reinterpret_cast<uint32_t*>(sm.N[j])[2 * lane + 1] = packed1;
        const uint32_t a = warp_sum(__popc(word));
        if (lane == 0) sm.A[j] = static_cast<uint16_t>(a);
        asum += a;
        aempty |= a == 0;
    }
    if (lane == 0) {
        sm.partA[warp] = asum;
        sm.partE[warp] = aempty;
    }
    __syncthreads();
    {
        const uint32_t q = tid & 255u, group = tid >> 8, half = nb / 2;
        const uint32_t j0 = (group & 1u) ? half : 0u, j1 = (group & 1u) ? nb : half;
        uint32_t best[6], s;
        if (group < 2) extreme_six<true>(sm, q, j0, j1, best, &s);
        else extreme_six<false>(sm, q, j0, j1, best, &s);
        uint32_t* dst = group == 0 ? sm.lo[q] : group == 1 ? sm.lo2[q] : group == 2 ? sm.hi[q] : sm.hi2[q];
#pragma unroll
        for (int k = 0; k < 6; ++k) dst[k] = best[k];
        if (group == 0) sm.S[q] = static_cast<uint16_t>(s);
        if (group == 1) sm.S2[q] = static_cast<uint16_t>(s);
    }
    __syncthreads();
    if (tid < 256) {
        merge_six<true>(sm.lo[tid], sm.lo2[tid]);
        sm.S[tid] = static_cast<uint16_t>(sm.S[tid] + sm.S2[tid]);
    } else if (tid < 512) {
        merge_six<false>(sm.hi[tid - 256], sm.hi2[tid - 256]);
    } else if (tid < 544) {
        const uint32_t a = warp_sum(sm.partA[lane]);
        const uint32_t empty = __any_sync(kFull, sm.partE[lane] != 0);
        if (lane == 0) {
            sm.sumA = a;
            sm.any_empty = empty;
        }
    }
    __syncthreads();
}

struct Trial {
    bool valid;
    uint32_t total, mn, mx;
};

// Trial placement of (info i, word wc, bit b) on the current level, warp-wide
// (lane w owns word w, i.e. pieces 8w..8w+7).  Mirrors the lambdas of
// remove_invalid_transitions and get_best_candidate.
__device__ Trial trial(const GmSmem& sm, uint32_t nb, uint32_t i, uint32_t wc, uint32_t b, uint32_t width,
                       uint32_t lane)
{
    Trial r{true, 0, ~0u, 0};
    const uint32_t p = 8 * wc + b / 4, o = b & 3u;
    const uint32_t pos = sm.position_index[i];
    const uint32_t pm = lane == wc ? ~(0xFu << (4 * (b / 4))) : kFull;
    const int off[4] = {-static_cast<int>(width), 1, static_cast<int>(width), -1};
    uint32_t nj[4], ncnt[4];
    uint32_t nn = 0;
    // apply_color_constraints (CUDA_glutton_max.h:531-612)
    for (uint32_t s = 0; s < 4; ++s) {
        const uint32_t col = sm.pieces[p][(s + o) & 3u];
        if (!col) continue;
        const uint32_t npos = static_cast<uint32_t>(static_cast<int>(pos) + off[s]);
        const uint32_t j = sm.info_index[npos];
        if (j >= nb) continue;  // position not free
        const uint32_t rw = sm.X[j][lane] & sm.cc[col - 1][s][lane] & pm;
        const uint32_t pc = warp_sum(__popc(rw));
        if (!pc) {
            r.valid = false;
            return r;
        }
        uint32_t packed = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) packed |= static_cast<uint32_t>(__popc((rw >> (4 * k)) & 0xFu)) << (3 * k);
        nj[nn] = j;
        ncnt[nn] = packed;
        ++nn;
        r.total += pc;
        r.mn = min(r.mn, pc);
        r.mx = max(r.mx, pc);
    }
    // every other free position keeps X[j] without piece p (apply_simple_mask)
    uint32_t sum_a = sm.sumA - sm.A[i];
    uint32_t sum_n = sm.S[p] - sm.N[i][p];
    for (uint32_t k = 0; k < nn; ++k) {
        sum_a -= sm.A[nj[k]];
        sum_n -= sm.N[nj[k]][p];
    }
    r.total += sum_a - sum_n;
    auto excluded = [&](uint32_t j) {
        bool e = j == i;
        for (uint32_t k = 0; k < nn; ++k) e |= j == nj[k];
        return e;
    };
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const uint32_t e = sm.lo[p][k];
        if (e == ~0u) break;
        if (!excluded(e & 0xFFFFu)) {
            const uint32_t v = e >> 16;
            if (v == 0) {
                r.valid = false;
                return r;
            }
            r.mn = min(r.mn, v);
            break;
        }
    }
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        const uint32_t e = sm.hi[p][k];
        if (e == 0u) break;
        if (!excluded(e & 0xFFFFu)) {
            r.mx = max(r.mx, (e >> 16) - 1u);
            break;
        }
    }
    // pieces: every available piece other than p needs a place left
    uint32_t psum = 0, pmin = ~0u, pmax = 0;
    bool bad = false;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t q = 8 * lane + k;
        if (q == p || !piece_available(sm, q)) continue;
        uint32_t c = static_cast<uint32_t>(sm.S[q]) - sm.N[i][q];
        for (uint32_t kk = 0; kk < nn; ++kk) c -= sm.N[nj[kk]][q] - ((ncnt[kk] >> (3 * k)) & 7u);
        bad |= c == 0;
        psum += c;
        pmin = min(pmin, c);
        pmax = max(pmax, c);
    }
    if (__any_sync(kFull, bad)) {
        r.valid = false;
        return r;
    }
    r.total += warp_sum(psum);
    r.mn = min(r.mn, warp_min(pmin));
    r.mx = max(r.mx, warp_max(pmax));
    return r;
}

__device__ void load_level(GmSmem& sm, const GmLaunch& P, uint32_t level, uint32_t tid)
{
    const uint32_t S = P.n, nb = S - level;
    const uint32_t* src = P.infos + static_cast<size_t>(tri_base(S, level)) * 32;
    for (uint32_t k = tid; k < nb * 32; k += kThreads) sm.X[k >> 5][k & 31] = src[k];
}

__device__ void store_level(const GmSmem& sm, const GmLaunch& P, uint32_t level, uint32_t tid)
{
    const uint32_t S = P.n, nb = S - level;
    uint32_t* dst = P.infos + static_cast<size_t>(tri_base(S, level)) * 32;
    for (uint32_t k = tid; k < nb * 32; k += kThreads) dst[k] = sm.X[k >> 5][k & 31];
}

// CUDA_glutton_max_stack::pop (thread 0); returns the restored info index.
// `owner` (the block that keeps the global search record) also updates it.
__device__ uint32_t pop_state(GmSmem& sm, GmState* st, uint32_t S, bool owner)
{
    const uint32_t level = sm.level;
    const uint32_t last = S - level;
    const uint32_t info = sm.position_index[last];
    const uint32_t played = sm.played[level - 1];
    const uint32_t pos = played & 0xFFu;
    sm.level = level - 1;
    const uint32_t piece = (played >> 8) & 0xFFu;
    sm.avail[piece >> 5] |= 1u << (piece & 31);
    sm.position_index[last] = pos;
    const uint32_t pos2 = sm.position_index[info];
    uint32_t t = sm.info_index[pos];
    sm.info_index[pos] = sm.info_index[pos2];
    sm.info_index[pos2] = t;
    t = sm.position_index[info];
    sm.position_index[info] = sm.position_index[last];
    sm.position_index[last] = t;
    if (owner) st->pops++;
    return info;
}

// CUDA_glutton_max_stack::push (thread 0).
__device__ void push_state(GmSmem& sm, GmState* st, uint32_t S, uint32_t info, uint32_t pos, uint32_t piece, uint32_t o,
                           bool owner)
{
    const uint32_t level = sm.level;
    sm.played[level] = (o << 16) | (piece << 8) | pos;
    sm.avail[piece >> 5] &= ~(1u << (piece & 31));
    const uint32_t nl = level + 1;
    sm.level = nl;
    if (owner) {
        st->played[level] = sm.played[level];
        if (nl > st->max) {
            for (uint32_t l = 0; l <= st->max && l < S; ++l) st->max_played[l] = sm.played[l];
            st->max = nl;
        }
        st->pushes++;
    }
    const uint32_t last = S - nl;
    const uint32_t last_pos = sm.position_index[last];
    sm.position_index[info] = info;
    uint32_t t = sm.info_index[pos];
    sm.info_index[pos] = sm.info_index[last_pos];
    sm.info_index[last_pos] = t;
    t = sm.position_index[info];
    sm.position_index[info] = sm.position_index[last];
    sm.position_index[last] = t;
}

// Grid barrier of the cooperative launch (all blocks are resident).  The wait is
// bounded: past the deadline the block flags an error and the barrier reports it.
__device__ bool grid_sync(GmGrid* g, uint32_t nblocks)
{
    __syncthreads();
    __shared__ uint32_t ok_s;
    if (threadIdx.x == 0) {
        uint32_t ok = 1;
        const uint32_t gen = *(volatile uint32_t*)&g->bar_gen;
        __threadfence();
        if (atomicAdd(&g->bar_count, 1u) == nblocks - 1) {
            g->bar_count = 0;
            __threadfence();
            atomicAdd(&g->bar_gen, 1u);
        } else {
            const uint64_t deadline = global_ns() + kBarrierWaitNs;
            while (*(volatile uint32_t*)&g->bar_gen == gen) {
                if (*(volatile int*)&g->error || global_ns() > deadline) {
                    atomicExch(&g->error, 1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// One glutton max search.  GRID = false: one block does everything.  GRID = true:
// every block of a cooperative launch keeps a copy of the level and makes the same
// decisions; the candidate trials of each validity pass are shared out over the warps
// of all blocks through global memory (triple-buffered per pass, one grid barrier per
// pass), and block 0 keeps the global search record.
template <bool GRID>
__global__ void __launch_bounds__(kThreads, 1) gm_kernel(GmLaunch P)
{
    extern __shared__ __align__(16) unsigned char gm_raw[];
    GmSmem& sm = *reinterpret_cast<GmSmem*>(gm_raw);
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t S = P.n;
    GmState* st = P.state;
    GmGrid* g = P.grid;
    const bool owner = !GRID || blockIdx.x == 0;
    const uint32_t nblocks = gridDim.x;
    uint32_t pass_no = 0;  // grid mode: passes so far (selects the exchange buffer)
    bool grid_failed = false;
    for (uint32_t k = tid; k < 256 * 4; k += kThreads) sm.pieces[k >> 2][k & 3] = P.pieces[k];
    for (uint32_t k = tid; k < P.ncolours * 4 * 32; k += kThreads) (&sm.cc[0][0][0])[k] = P.cc[k];
    for (uint32_t k = tid; k < 256; k += kThreads) {
        sm.position_index[k] = st->position_index[k];
        sm.info_index[k] = st->info_index[k];
        sm.played[k] = st->played[k];
    }
    if (tid < 8) sm.avail[tid] = st->avail[tid];
    if (tid == 0) {
        sm.level = st->level;
        sm.new_level = st->new_level;
        sm.pop_index = st->pop_index;
        sm.stop = 0;
    }
    __syncthreads();
    load_level(sm, P, sm.level, tid);
    __syncthreads();
    const uint64_t deadline = P.timeout_ns ? global_ns() + P.timeout_ns : 0;

    for (;;) {
        const uint32_t level = sm.level;
        if (level >= S) break;  // full board (level == S) or exhausted (wrapped below 0)
        if (owner && tid == 0) {
            const bool stop = (P.push_budget && st->pushes >= P.push_budget) ||
                              (P.placement_budget && st->trials + st->pushes >= P.placement_budget) ||
                              (deadline && global_ns() > deadline);
            sm.stop = stop;
            if (GRID) g->stop = stop;
        }
        if (GRID) {
            // every block follows block 0's decision
            if (!grid_sync(g, nblocks)) {
                grid_failed = true;
                break;
            }
            if (tid == 0) sm.stop = *(volatile uint32_t*)&g->stop;
        }
        __syncthreads();
        if (sm.stop) break;
        const uint32_t nb = S - level;
        // a popped level whose tried candidate was its last one pops again
        if (!sm.new_level) {
            const uint32_t any = __syncthreads_or(tid < 32 && sm.X[sm.pop_index][tid] != 0);
            if (!any) {
                __syncthreads();
                if (tid == 0) {
                    if (level == 0) sm.level = ~0u;
                    else sm.pop_index = pop_state(sm, st, S, owner);
                    sm.new_level = 0;
                }
                __syncthreads();
                if (sm.level < S) load_level(sm, P, sm.level, tid);
                __syncthreads();
                continue;
            }
        }
        if (owner && tid == 0) st->levels++;
        // ---- validity fixpoint and scores ----
        bool failed = false;
        for (;;) {
            level_statistics(sm, nb, tid);
            if (sm.any_empty) {
                failed = true;
                break;
            }
            const uint32_t buf = pass_no % 3;
            if (!GRID) {
                for (uint32_t k = tid; k < nb * 32; k += kThreads) sm.inval[k >> 5][k & 31] = 0;
            }
            if (tid == 0) {
                sm.any_invalid = 0;
                sm.next_info = 0;
                if (owner) st->passes++;
            }
            __syncthreads();
            unsigned long long best_key = 0;
            uint32_t best_order = ~0u, trials = 0;
            const bool last_level = level == S - 1;
            for (;;) {
                // work unit: one word (8 pieces x 4 orientations) of one free position's info
                uint32_t u = 0;
                if (lane == 0) u = GRID ? atomicAdd(&g->next_info[buf], 1u) : atomicAdd(&sm.next_info, 1u);
                u = __shfl_sync(kFull, u, 0);
                const uint32_t i = u >> 5;
                if (i >= nb) break;
                for (uint32_t w = u & 31u; w == (u & 31u); ++w) {
                    uint32_t word = sm.X[i][w];
                    while (word) {
                        const uint32_t b = __ffs(word) - 1;
                        word &= word - 1;
                        ++trials;
                        const Trial t = trial(sm, nb, i, w, b, P.width, lane);
                        const uint32_t order = (i << 10) | (w << 5) | b;
                        if (!t.valid) {
                            if (lane == 0) {
                                if (GRID) {
                                    atomicOr(&g->inval[buf][i][w], 1u << b);
                                    g->any_invalid[buf] = 1;
                                } else {
                                    atomicOr(&sm.inval[i][w], 1u << b);
                                    sm.any_invalid = 1;
                                }
                            }
                            continue;
                        }
                        const unsigned long long key =
                            (static_cast<unsigned long long>(t.total) << 32) | ((t.mx << 16) + t.mn);
                        const bool better = best_order == ~0u ||
                                            (last_level ? order > best_order
                                                        : (key > best_key || (key == best_key && order < best_order)));
                        if (better) {
                            best_key = key;
                            best_order = order;
                        }
                    }
                }
            }
            if (lane == 0) {
                sm.warp_key[warp] = best_key;
                sm.warp_order[warp] = best_order;
                sm.warp_trials[warp] = trials;
            }
            __syncthreads();
            // this block's best, reduced by warp 0 (a strict total order: any reduction
            // order gives the same result)
            if (warp == 0) {
                unsigned long long k0 = sm.warp_key[lane];
                uint32_t o0 = sm.warp_order[lane];
                warp_best(k0, o0, last_level);
                unsigned long long tr = sm.warp_trials[lane];
                for (int d = 16; d; d >>= 1) tr += __shfl_xor_sync(kFull, tr, d);
                if (lane == 0) {
                    if (GRID) {
                        atomicAdd(&st->trials, tr);
                        g->blk_key[buf][blockIdx.x] = k0;
                        g->blk_order[buf][blockIdx.x] = o0;
                    } else {
                        st->trials += tr;
                        sm.best_order = o0;
                    }
                }
            }
            if (GRID) {
                if (!grid_sync(g, nblocks)) {
                    grid_failed = true;
                    break;
                }
                // the buffer of the pass before last is free again: block 0 clears it
                if (blockIdx.x == 0) {
                    const uint32_t old = (pass_no + 2) % 3;
                    for (uint32_t k = tid; k < S * 32; k += kThreads) (&g->inval[old][0][0])[k] = 0;
                    if (tid == 0) {
                        g->any_invalid[old] = 0;
                        g->next_info[old] = 0;
                    }
                }
                if (warp == 0) {
                    // the blocks' bests, 32 at a time (the loads overlap instead of
                    // waiting on L2 one block after another)
                    unsigned long long k0 = 0;
                    uint32_t o0 = ~0u;
                    for (uint32_t b2 = lane; b2 < nblocks; b2 += 32) {
                        const uint32_t o = *(volatile uint32_t*)&g->blk_order[buf][b2];
                        const unsigned long long k = *(volatile unsigned long long*)&g->blk_key[buf][b2];
                        if (better_candidate(k, o, k0, o0, last_level)) {
                            k0 = k;
                            o0 = o;
                        }
                    }
                    warp_best(k0, o0, last_level);
                    if (lane == 0) {
                        sm.any_invalid = *(volatile uint32_t*)&g->any_invalid[buf];
                        sm.best_order = o0;
                    }
                }
                ++pass_no;
            }
            __syncthreads();
            if (!sm.any_invalid) break;
            if (GRID) {
                for (uint32_t k = tid; k < nb * 32; k += kThreads)
                    sm.X[k >> 5][k & 31] &= ~(*(volatile uint32_t*)&g->inval[buf][k >> 5][k & 31]);
            } else {
                for (uint32_t k = tid; k < nb * 32; k += kThreads) sm.X[k >> 5][k & 31] &= ~sm.inval[k >> 5][k & 31];
            }
            __syncthreads();
        }
        if (grid_failed) break;
        if (failed || sm.best_order == ~0u) {
            // remove_invalid_transitions failed or no candidate: pop
            __syncthreads();
            if (tid == 0) {
                if (level == 0) sm.level = ~0u;
                else sm.pop_index = pop_state(sm, st, S, owner);
                sm.new_level = 0;
            }
            __syncthreads();
            if (sm.level < S) load_level(sm, P, sm.level, tid);
            __syncthreads();
            continue;
        }
        // ---- apply_best_candidate ----
        const uint32_t bi = sm.best_order >> 10, bw = (sm.best_order >> 5) & 31u, bb = sm.best_order & 31u;
        const uint32_t piece = 8 * bw + bb / 4, o = bb & 3u;
        const uint32_t pos = sm.position_index[bi];
        if (tid == 0) sm.X[bi][bw] &= ~(1u << bb);
        __syncthreads();
        // the level keeps its remaining candidates for a later pop (in grid mode every
        // block writes the same values and reads back only its own writes)
        store_level(sm, P, level, tid);
        __threadfence_block();
        const uint32_t pm_word = ~(0xFu << (4 * (bb / 4)));
        // the next level moves the last info into the chosen slot; an empty
        // result there stops the reference's apply before its push
        const bool copy_last = bi < nb - 1 && level < S - 1;
        const uint32_t last_any =
            copy_last ? __syncthreads_or(tid < 32 && (sm.X[nb - 1][tid] & (tid == bw ? pm_word : kFull)) != 0) : 1u;
        if (!last_any) {
            if (tid == 0) sm.new_level = 1;
            __syncthreads();
            continue;
        }
        __syncthreads();
        // next level in place: X[j] &= pm for j < nb-1, X[bi] = X[nb-1] & pm
        for (uint32_t k = tid; k < (nb - 1) * 32; k += kThreads) {
            const uint32_t j = k >> 5, w = k & 31;
            const uint32_t m = w == bw ? pm_word : kFull;
            if (j == bi) sm.X[j][w] = sm.X[nb - 1][w] & m;
            else sm.X[j][w] &= m;
        }
        __syncthreads();
        if (tid == 0) push_state(sm, st, S, bi, pos, piece, o, owner);
        __syncthreads();
        // colour constraints of the placed piece on its free neighbours
        if (warp == 0) {
            const uint32_t nl = sm.level, nbn = S - nl;
            const int off[4] = {-static_cast<int>(P.width), 1, static_cast<int>(P.width), -1};
            bool invalid = false;
            for (uint32_t s2 = 0; s2 < 4 && !invalid; ++s2) {
                const uint32_t col = sm.pieces[piece][(s2 + o) & 3u];
                if (!col) continue;
                const uint32_t npos = static_cast<uint32_t>(static_cast<int>(pos) + off[s2]);
                const uint32_t j = sm.info_index[npos];
                if (j >= nbn) continue;
                const uint32_t r = sm.X[j][lane] & sm.cc[col - 1][s2][lane];
                if (!__any_sync(kFull, r)) {
                    invalid = true;
                    break;
                }
                sm.X[j][lane] = r;
            }
            if (lane == 0) sm.apply_failed = invalid;
        }
        __syncthreads();
        if (sm.apply_failed) {
            __syncthreads();
            if (tid == 0) pop_state(sm, st, S, owner);
            __syncthreads();
            load_level(sm, P, sm.level, tid);
        }
        if (tid == 0) sm.new_level = 1;
        __syncthreads();
    }
    // write the search state back (the owner block)
    __syncthreads();
    if (!owner) return;
    if (tid == 0) {
        const uint32_t level = sm.level;
        st->level = level;
        st->new_level = sm.new_level;
        st->pop_index = sm.pop_index;
        st->status = grid_failed ? 3 : (level == S ? 0 : (level > S ? 2 : 1));
    }
    if (sm.level < S) store_level(sm, P, sm.level, tid);
    for (uint32_t k = tid; k < 256; k += kThreads) {
        st->position_index[k] = sm.position_index[k];
        st->info_index[k] = sm.info_index[k];
    }
    if (tid < 8) st->avail[tid] = sm.avail[tid];
}

}  // namespace

size_t gm_smem_bytes() { return sizeof(GmSmem); }

cudaError_t launch_gm(const GmLaunch& P, cudaStream_t stream)
{
    const size_t smem = sizeof(GmSmem);
    cudaError_t e = cudaFuncSetAttribute(gm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    gm_kernel<false><<<1, kThreads, smem, stream>>>(P);
    return cudaGetLastError();
}

cudaError_t launch_gm_grid(const GmLaunch& P, uint32_t blocks, cudaStream_t stream)
{
    const size_t smem = sizeof(GmSmem);
    cudaError_t e = cudaFuncSetAttribute(gm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gm_kernel<true>, kThreads, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (per_sm < 1 || blocks > static_cast<uint32_t>(per_sm * sms) || blocks > kMaxGridBlocks || !blocks)
        return cudaErrorCooperativeLaunchTooLarge;
    GmLaunch copy = P;
    void* args[] = {&copy};
    return cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(&gm_kernel<true>), dim3(blocks), dim3(kThreads),
                                       args, smem, stream);
}

}  // namespace emp
