// Variable-space search of the reference's CUDA_backtracker feature, kept as a
// debug mode (its trace lines are what tests_CUDA/backtracker_3_3 checks).
//
// The reference runs one warp over "variables" (position, piece, orientation):
// src/CUDA_backtracker.cu:67-178 with the variables of
// emp_variable_generator::create_variables (include/emp_variable_generator.h:
// 335-525) and the transition vectors of system_equation_for_CUDA
// (include/system_equation_for_CUDA.h:70-173).  The exhaustive counting search of
// this library (emp_bt.cu) replaces it; this file reproduces its visiting order and
// first solution.
//
// Layout: a capability is 32 words, word 8*o + x/32, bit x%32 for (x, orientation
// o); x is a piece index for the first n capabilities (one per position, row-major)
// and a position for the next n (one per piece).  Each lane owns one word of every
// capability.  The stack holds n+1 levels of 2n capabilities in global memory;
// levels above 0 start zeroed and keep what earlier attempts wrote, as the
// reference's stack does.
#include "emp_b200.h"
#include "emp_common.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

using emp::DeviceBuffer;
using emp::fail;

namespace {

constexpr uint32_t kW = 32;
constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr uint32_t kMaxVsPieces = 64;

__device__ __forceinline__ uint64_t vs_now()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

struct VsLaunch {
    uint32_t n;
    const uint32_t* trans;     // [variables][2n][32]
    const int32_t* var_of;     // [n*1024]: variable number of a raw id, -1 when none
    uint32_t* lev;             // [n+1][2n][32]
    uint32_t* stack_var;       // [n]
    emp_vs_event* events;
    unsigned long long capacity;
    unsigned long long* n_events;
    uint32_t* found;           // 1: a solution, 2: stopped by the selection budget, 3: deadline
    unsigned long long max_selections;
    unsigned long long timeout_ns;
};

// One warp; lane l owns word l of every capability.
__global__ void __launch_bounds__(32) vs_kernel(VsLaunch P)
{
    const uint32_t lane = threadIdx.x, n = P.n;
    const size_t capw = size_t(2) * n * kW;
    const uint64_t deadline = vs_now() + P.timeout_ns;
    unsigned long long ne = 0, selections = 0;
    uint32_t step = 0, result = 0;
    do {
        uint32_t* avail = P.lev + capw * step + kW * step;
        const uint32_t word = avail[lane];
        const unsigned ballot = __ballot_sync(kFull, word != 0);
        if (!ballot) {
            --step;  // step 0 wraps and ends the loop, as the reference's unsigned step does
            continue;
        }
        const uint32_t elected = __ffs(ballot) - 1;
        const uint32_t w = __shfl_sync(kFull, word, elected);
        const uint32_t bit = __ffs(w) - 1;
        const uint32_t var = (step << 10) | (elected << 5) | bit;
        const uint32_t piece = (elected % 8) * 32 + bit;
        if (lane == 0) {
            if (ne < P.capacity) P.events[ne] = emp_vs_event{elected, var, step};
            P.stack_var[step] = var;
        }
        ++ne;
        if (lane == elected) avail[lane] = w & ~(1u << bit);
        if (step == n - 1) {
            result = 1;
            break;
        }
        ++selections;
        if ((P.max_selections && selections >= P.max_selections) || vs_now() > deadline) {
            result = P.max_selections && selections >= P.max_selections ? 2u : 3u;
            break;
        }
        const int32_t vi = P.var_of[var];
        const uint32_t* S = P.lev + capw * step;
        const uint32_t* T = P.trans + capw * static_cast<size_t>(vi >= 0 ? vi : 0);
        uint32_t* R = P.lev + capw * (step + 1);
        bool valid = vi >= 0;
        for (uint32_t q = step + 1; q < n && valid; ++q) {
            const uint32_t r = S[kW * q + lane] & T[kW * q + lane];
            if (__any_sync(kFull, r != 0)) R[kW * q + lane] = r;
            else valid = false;
        }
        // piece capabilities below, then above, the selected piece: the reference
        // passes the transition vector as the situation too (src/CUDA_backtracker.cu:
        // 155-164), so a piece's capability becomes the transition's own
        for (uint32_t q = 0; q < n && valid; ++q) {
            if (q == piece) continue;
            const uint32_t t = T[kW * (n + q) + lane];
            if (!__any_sync(kFull, t != 0)) continue;
            R[kW * (n + q) + lane] = t;
        }
        if (valid) {
            R[kW * (n + piece) + lane] = 0;
            ++step;
        }
        __syncwarp();
    } while (step < n);
    if (lane == 0) {
        *P.n_events = ne;
        *P.found = result;
    }
}

void vs_clear(uint32_t* cap, uint32_t x, uint32_t o) { cap[8 * o + x / 32] &= ~(1u << (x % 32)); }
void vs_set(uint32_t* cap, uint32_t x, uint32_t o) { cap[8 * o + x / 32] |= 1u << (x % 32); }

}  // namespace

extern "C" emp_status emp_bt_variable_space(emp_puzzle puzzle, int device, uint64_t max_selections,
                                            uint32_t timeout_ms, emp_vs_event* events, uint64_t capacity,
                                            uint64_t* n_events, uint32_t* board, uint32_t* found)
{
    emp::clear_error();
    if (!puzzle || !n_events || !board || !found || (capacity && !events))
        return fail(EMP_ERR_INVALID, "emp_bt_variable_space: null argument");
    const emp::PuzzleModel& m = puzzle->model;
    const uint32_t n = m.n, w = m.width, h = m.height;
    if (n > kMaxVsPieces)
        return fail(EMP_ERR_UNSUPPORTED, "emp_bt_variable_space: a debug mode for puzzles of at most 64 pieces");
    for (uint32_t i = 0; i < n; ++i)
        if (puzzle->order[i] != i)
            return fail(EMP_ERR_UNSUPPORTED, "emp_bt_variable_space: the reference's variable-space search is row-major");
    // variables per position: the pieces whose orientations fit the frame sides, in
    // the kind bitfield's order (kind_index*4 + o over allowed orientations)
    struct Var {
        uint32_t pos, piece, o;
    };
    std::vector<Var> vars;
    std::vector<uint32_t> first(n + 1, 0);
    for (uint32_t pos = 0; pos < n; ++pos) {
        first[pos] = static_cast<uint32_t>(vars.size());
        const uint32_t x = pos % w, y = pos / w;
        const bool frame[4] = {y == 0, x == w - 1, y == h - 1, x == 0};
        const bool xb = x == 0 || x == w - 1, yb = y == 0 || y == h - 1;
        const uint32_t k = (xb || yb) ? ((!xb || !yb) ? emp::kBorder : emp::kCorner) : emp::kCenter;
        for (uint32_t ki = 0; ki < m.nb_kind(k); ++ki) {
            const uint32_t p = m.members[k][ki];
            for (uint32_t o = 0; o < 4; ++o) {
                if (!m.allowed(p, o)) continue;
                bool ok = true;
                for (uint32_t s = 0; s < 4 && ok; ++s) ok = (m.colour(p, s, o) == 0) == frame[s];
                if (ok) vars.push_back({pos, p, o});
            }
        }
    }
    first[n] = static_cast<uint32_t>(vars.size());
    const size_t capw = size_t(2) * n * kW, nv = vars.size();
    std::vector<uint32_t> trans(capw * std::max<size_t>(nv, 1), ~0u);
    std::vector<int32_t> var_of(size_t(n) * 1024, -1);
    for (size_t v = 0; v < nv; ++v) var_of[vars[v].pos * 1024 + vars[v].o * 256 + vars[v].piece] = static_cast<int32_t>(v);
    for (size_t v = 0; v < nv; ++v) {
        uint32_t* T = trans.data() + capw * v;
        for (uint32_t u = first[vars[v].pos]; u < first[vars[v].pos + 1]; ++u) {
            vs_clear(T + kW * vars[v].pos, vars[u].piece, vars[u].o);
            vs_clear(T + kW * (n + vars[u].piece), vars[v].pos, vars[u].o);
        }
        for (size_t u = 0; u < nv; ++u) {
            if (vars[u].piece != vars[v].piece) continue;
            vs_clear(T + kW * (n + vars[v].piece), vars[u].pos, vars[u].o);
            vs_clear(T + kW * vars[u].pos, vars[v].piece, vars[u].o);
        }
    }
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x)
            for (int dir = 0; dir < 2; ++dir) {
                if ((dir == 0 && x + 1 >= w) || (dir == 1 && y + 1 >= h)) continue;
                const uint32_t p1 = y * w + x, p2 = dir == 0 ? p1 + 1 : p1 + w;
                const uint32_t side1 = dir == 0 ? 1u : 2u, side2 = dir == 0 ? 3u : 0u;
                for (uint32_t a = first[p1]; a < first[p1 + 1]; ++a)
                    for (uint32_t b = first[p2]; b < first[p2 + 1]; ++b) {
                        const Var &v1 = vars[a], &v2 = vars[b];
                        if (v1.piece == v2.piece || m.colour(v1.piece, side1, v1.o) == m.colour(v2.piece, side2, v2.o))
                            continue;
                        uint32_t *T1 = trans.data() + capw * a, *T2 = trans.data() + capw * b;
                        vs_clear(T1 + kW * p2, v2.piece, v2.o);
                        vs_clear(T1 + kW * (n + v2.piece), p2, v2.o);
                        vs_clear(T2 + kW * p1, v1.piece, v1.o);
                        vs_clear(T2 + kW * (n + v1.piece), p1, v1.o);
                    }
            }
    std::vector<uint32_t> lev0(capw, 0);
    for (const Var& v : vars) {
        vs_set(lev0.data() + kW * v.pos, v.piece, v.o);
        vs_set(lev0.data() + kW * (n + v.piece), v.pos, v.o);
    }
    int dev = 0;
    EMP_TRY(emp::select_device(device, &dev));
    DeviceBuffer d_trans, d_var, d_lev, d_stack, d_ev, d_cnt;
    CUDA_TRY(d_trans.alloc(sizeof(uint32_t) * trans.size()));
    CUDA_TRY(d_var.alloc(sizeof(int32_t) * var_of.size()));
    CUDA_TRY(d_lev.alloc(sizeof(uint32_t) * capw * (n + 1)));
    CUDA_TRY(d_stack.alloc(sizeof(uint32_t) * n));
    CUDA_TRY(d_ev.alloc(sizeof(emp_vs_event) * std::max<uint64_t>(capacity, 1)));
    CUDA_TRY(d_cnt.alloc(2 * sizeof(unsigned long long)));
    CUDA_TRY(cudaMemcpy(d_trans.p, trans.data(), sizeof(uint32_t) * trans.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_var.p, var_of.data(), sizeof(int32_t) * var_of.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(d_lev.p, 0, d_lev.bytes));
    CUDA_TRY(cudaMemcpy(d_lev.p, lev0.data(), sizeof(uint32_t) * capw, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(d_stack.p, 0, d_stack.bytes));
    CUDA_TRY(cudaMemset(d_cnt.p, 0, d_cnt.bytes));
    VsLaunch P;
    P.n = n;
    P.trans = d_trans.as<uint32_t>();
    P.var_of = d_var.as<int32_t>();
    P.lev = d_lev.as<uint32_t>();
    P.stack_var = d_stack.as<uint32_t>();
    P.events = d_ev.as<emp_vs_event>();
    P.capacity = capacity;
    P.n_events = d_cnt.as<unsigned long long>();
    P.found = reinterpret_cast<uint32_t*>(d_cnt.as<unsigned long long>() + 1);
    P.max_selections = max_selections;
    P.timeout_ns = 1000000ull * (timeout_ms ? timeout_ms : 60000u);
    vs_kernel<<<1, 32>>>(P);
    CUDA_TRY(cudaGetLastError());
    unsigned long long cnt[2] = {0, 0};
    CUDA_TRY(cudaMemcpy(cnt, d_cnt.p, sizeof(cnt), cudaMemcpyDeviceToHost));
    *n_events = cnt[0];
    const uint32_t res = static_cast<uint32_t>(cnt[1] & 0xFFFFFFFFu);
    *found = res == 1;
    if (capacity)
        CUDA_TRY(cudaMemcpy(events, d_ev.p, sizeof(emp_vs_event) * std::min<uint64_t>(capacity, cnt[0]),
                            cudaMemcpyDeviceToHost));
    std::vector<uint32_t> sv(n, 0);
    CUDA_TRY(cudaMemcpy(sv.data(), d_stack.p, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    for (uint32_t s = 0; s < n; ++s) {
        const uint32_t lane = (sv[s] >> 5) & 31u, bit = sv[s] & 31u;
        board[s] = res == 1 ? ((((lane % 8) * 32 + bit) << 2) | (lane / 8)) : 0xFFFFFFFFu;
    }
    if (res == 3) return fail(EMP_INCOMPLETE, "emp_bt_variable_space: the deadline stopped the search");
    if (res == 2) return fail(EMP_INCOMPLETE, "emp_bt_variable_space: the selection budget stopped the search");
    return EMP_OK;
}
