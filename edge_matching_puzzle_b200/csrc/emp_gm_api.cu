// C ABI of the glutton max search (emp_glutton_max).
#include "emp_b200.h"
#include "emp_common.h"
#include "emp_gm.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

using emp::DeviceBuffer;
using emp::fail;

namespace {

// Colour constraints (CUDA_common_glutton.h:111-146): mask[c-1][side] holds
// (piece, orientation) whose side opposite to `side` shows colour c.
std::vector<uint32_t> colour_constraints(const emp::PuzzleModel& m)
{
    std::vector<uint32_t> cc(static_cast<size_t>(m.border_id) * 4 * 32, 0);
    for (uint32_t c = 1; c <= m.max_colour; ++c)
        for (uint32_t s = 0; s < 4; ++s) {
            const uint32_t opp = (s + 2) & 3u;
            for (uint32_t i = 0; i < m.n; ++i)
                for (uint32_t o = 0; o < 4; ++o)
                    if (m.colour(i, opp, o) == c) cc[((c - 1) * 4 + s) * 32 + i / 8] |= 1u << (o + 4 * (i % 8));
        }
    return cc;
}

// Initial capability of every position (CUDA_common_glutton.h:150-211): corner
// and border pieces in their forced orientation, centre pieces in all four.
std::vector<uint32_t> initial_capability(const emp::PuzzleModel& m)
{
    std::vector<uint32_t> cap(static_cast<size_t>(m.n) * 32, 0);
    for (uint32_t pos = 0; pos < m.n; ++pos) {
        const uint32_t x = pos % m.width, y = pos / m.width;
        uint32_t* c = &cap[static_cast<size_t>(pos) * 32];
        const bool border = !x || !y || x == m.width - 1 || y == m.height - 1;
        const bool corner = (!x && !y) || (!x && y == m.height - 1) || (!y && x == m.width - 1) ||
                            (y == m.height - 1 && x == m.width - 1);
        if (corner) {
            const uint32_t ci = (!x && !y) ? 0 : (!y ? 1 : (x ? 2 : 3));
            const uint32_t b1 = ci, b2 = (ci + 3) & 3u;  // emp_FSM_info::get_corner_orientation
            for (uint32_t piece : m.members[emp::kCorner])
                for (uint32_t o = 0; o < 4; ++o)  // emp_piece_corner::compute_orientation
                    if (!m.colour(piece, b1, o) && !m.colour(piece, b2, o)) {
                        c[piece / 8] |= 1u << (o + 4 * (piece % 8));
                        break;
                    }
        } else if (border) {
            const uint32_t bo = !y ? 0 : (x == m.width - 1 ? 1 : (y == m.height - 1 ? 2 : 3));
            for (uint32_t piece : m.members[emp::kBorder]) {
                uint32_t pb = 0;
                for (uint32_t s = 0; s < 4; ++s)
                    if (!m.colours[piece][s]) {
                        pb = s;
                        break;
                    }
                const uint32_t o = (pb + 4 - bo) & 3u;  // emp_piece_border::compute_orientation
                c[piece / 8] |= 1u << (o + 4 * (piece % 8));
            }
        } else {
            for (uint32_t piece : m.members[emp::kCenter])
                for (uint32_t o = 0; o < 4; ++o) c[piece / 8] |= 1u << (o + 4 * (piece % 8));
        }
    }
    return cap;
}

void board_from_played(const emp::PuzzleModel& m, const uint32_t* played, uint32_t count, uint32_t* board)
{
    for (uint32_t i = 0; i < 256; ++i) board[i] = 0xFFFFFFFFu;
    for (uint32_t l = 0; l < count && l < m.n; ++l) {
        const uint32_t pi = played[l];
        if (pi == 0xFFFFFFFFu) continue;
        const uint32_t pos = pi & 0xFFu, piece = (pi >> 8) & 0xFFu, o = pi >> 16;
        if (pos < m.n) board[pos] = (piece << 2) | (o & 3u);
    }
}

}  // namespace

extern "C" emp_status emp_glutton_max(emp_puzzle puzzle, const emp_gm_config* config, emp_gm_result* result)
{
    emp::clear_error();
    if (!puzzle || !result) return fail(EMP_ERR_INVALID, "emp_glutton_max: null argument");
    emp_gm_config cfg{};
    cfg.device = -1;
    if (config) cfg = *config;
    const emp::PuzzleModel& m = puzzle->model;
    int dev = 0;
    EMP_TRY(emp::select_device(cfg.device, &dev));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
    if (emp::gm_smem_bytes() > static_cast<size_t>(prop.sharedMemPerBlockOptin))
        return fail(EMP_ERR_UNSUPPORTED, "glutton max level state does not fit shared memory");
    const uint32_t S = m.n;
    std::vector<uint8_t> pieces(256 * 4, 0);
    for (uint32_t i = 0; i < m.n; ++i)
        for (uint32_t s = 0; s < 4; ++s) pieces[4 * i + s] = m.colours[i][s];
    const std::vector<uint32_t> cc = colour_constraints(m);
    const std::vector<uint32_t> cap = initial_capability(m);
    emp::GmState st;
    std::memset(&st, 0, sizeof(st));
    st.new_level = 1;
    for (uint32_t i = 0; i < 256; ++i) {
        st.position_index[i] = i < S ? i : 0xFFFFFFFFu;
        st.info_index[i] = i < S ? i : 0xFFFFFFFFu;
        st.played[i] = 0xFFFFFFFFu;
        st.max_played[i] = 0xFFFFFFFFu;
    }
    for (uint32_t i = 0; i < m.n; ++i) st.avail[i >> 5] |= 1u << (i & 31);
    DeviceBuffer d_pieces, d_cc, d_infos, d_state, d_grid;
    const size_t tri = static_cast<size_t>(S) * (S + 1) / 2;
    uint32_t blocks = cfg.blocks;
    if (!blocks) blocks = static_cast<uint32_t>(prop.multiProcessorCount);
    blocks = std::min<uint32_t>(blocks, std::min<uint32_t>(emp::kMaxGridBlocks, prop.multiProcessorCount));
    if (blocks > 1) {
        CUDA_TRY(d_grid.alloc(sizeof(emp::GmGrid)));
        CUDA_TRY(cudaMemset(d_grid.p, 0, sizeof(emp::GmGrid)));
    }
    CUDA_TRY(d_pieces.alloc(pieces.size()));
    CUDA_TRY(d_cc.alloc(sizeof(uint32_t) * std::max<size_t>(cc.size(), 1)));
    CUDA_TRY(d_infos.alloc(sizeof(uint32_t) * 32 * tri));
    CUDA_TRY(d_state.alloc(sizeof(emp::GmState)));
    CUDA_TRY(cudaMemcpy(d_pieces.p, pieces.data(), pieces.size(), cudaMemcpyHostToDevice));
    if (!cc.empty()) CUDA_TRY(cudaMemcpy(d_cc.p, cc.data(), sizeof(uint32_t) * cc.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_infos.p, cap.data(), sizeof(uint32_t) * cap.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_state.p, &st, sizeof(st), cudaMemcpyHostToDevice));
    emp::GmLaunch P;
    P.pieces = d_pieces.as<uint8_t>();
    P.cc = d_cc.as<uint32_t>();
    P.infos = d_infos.as<uint32_t>();
    P.state = d_state.as<emp::GmState>();
    P.n = S;
    P.width = m.width;
    P.ncolours = m.border_id;
    P.push_budget = cfg.push_budget;
    P.placement_budget = cfg.placement_budget;
    P.grid = blocks > 1 ? d_grid.as<emp::GmGrid>() : nullptr;
    // without a caller limit the search still stops after an hour on the device
    const unsigned long long ms_limit = cfg.timeout_ms ? cfg.timeout_ms : 3600000ull;
    P.timeout_ns = ms_limit * 1000000ull;
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    CUDA_TRY(cudaEventRecord(e0));
    cudaError_t le = blocks > 1 ? emp::launch_gm_grid(P, blocks, nullptr) : emp::launch_gm(P, nullptr);
    if (le != cudaSuccess) {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return emp::cuda_fail(le, "glutton max launch");
    }
    CUDA_TRY(cudaEventRecord(e1));
    CUDA_TRY(cudaEventSynchronize(e1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    CUDA_TRY(cudaMemcpy(&st, d_state.p, sizeof(st), cudaMemcpyDeviceToHost));
    std::memset(result, 0, sizeof(*result));
    result->status = st.status;
    result->max_level = st.max;
    result->level = st.level <= S ? st.level : 0;
    board_from_played(m, st.max_played, st.max, result->best_board);
    board_from_played(m, st.played, result->level, result->final_board);
    result->trials = st.trials;
    result->pushes = st.pushes;
    result->pops = st.pops;
    result->passes = st.passes;
    result->levels = st.levels;
    result->kernel_ms = ms;
    if (st.status == 3) return fail(EMP_ERR_CUDA, "glutton max: a grid barrier of the multi-block search timed out");
    return st.status == 1 ? EMP_INCOMPLETE : EMP_OK;
}

// ---------------------------------------------------------------------------
// emp_glutton_max_noalloc: the same search with its device memory taken from a
// fixed array compiled into this library instead of cudaMalloc.
//
// Layout of the array (byte offsets, each section 256-byte aligned):
//   state   GmState
//   pieces  256 x 4 colours
//   cc      32 colours x 4 sides x 32 words
//   infos   triangular level stack for 256 positions: 256*257/2 infos x 32 words
// 4,232,448 bytes in all, enough for every puzzle the library accepts (at most
// 256 pieces; colour ids up to 30, which build_model enforces, so the colour check
// below is a second guard that a valid puzzle never trips).
namespace {

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
constexpr uint32_t kNoAllocMaxPieces = 256;
constexpr uint32_t kNoAllocMaxColours = 32;  // colour ids 1..31 plus the frame
constexpr size_t kOffState = 0;
constexpr size_t kOffPieces = align256(kOffState + sizeof(emp::GmState));
constexpr size_t kOffCc = align256(kOffPieces + 256 * 4);
constexpr size_t kOffInfos = align256(kOffCc + sizeof(uint32_t) * kNoAllocMaxColours * 4 * 32);
constexpr size_t kNoAllocBytes =
    align256(kOffInfos + sizeof(uint32_t) * 32 * (size_t(kNoAllocMaxPieces) * (kNoAllocMaxPieces + 1) / 2));
static_assert(kNoAllocBytes == 4232448, "scratch size stated above");
}  // namespace

static __device__ __align__(256) unsigned char g_gm_scratch[kNoAllocBytes];

extern "C" emp_status emp_glutton_max_noalloc(emp_puzzle puzzle, const emp_gm_config* config, emp_gm_result* result)
{
    emp::clear_error();
    if (!puzzle || !result) return fail(EMP_ERR_INVALID, "emp_glutton_max_noalloc: null argument");
    emp_gm_config cfg{};
    cfg.device = -1;
    if (config) cfg = *config;
    const emp::PuzzleModel& m = puzzle->model;
    if (m.n > kNoAllocMaxPieces)
        return fail(EMP_ERR_UNSUPPORTED, "emp_glutton_max_noalloc: " + std::to_string(m.n) +
                                             " pieces exceed the fixed scratch limit of " +
                                             std::to_string(kNoAllocMaxPieces));
    if (m.border_id > kNoAllocMaxColours)
        return fail(EMP_ERR_UNSUPPORTED, "emp_glutton_max_noalloc: " + std::to_string(m.border_id) +
                                             " colours exceed the fixed scratch limit of " +
                                             std::to_string(kNoAllocMaxColours));
    int dev = 0;
    EMP_TRY(emp::select_device(cfg.device, &dev));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, dev));
    if (emp::gm_smem_bytes() > static_cast<size_t>(prop.sharedMemPerBlockOptin))
        return fail(EMP_ERR_UNSUPPORTED, "glutton max level state does not fit shared memory");

    // The device address of the scratch array on the current device, looked up on
    // every call (no allocation; the first look-up on a device loads the array onto
    // it).  A cached address would go stale after cudaDeviceReset, which loads the
    // module again, possibly elsewhere.
    unsigned char* base = nullptr;
    {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_gm_scratch);
        if (e != cudaSuccess) return emp::cuda_fail(e, "emp_glutton_max_noalloc: scratch address look-up");
        base = static_cast<unsigned char*>(p);
    }

    const uint32_t S = m.n;
    std::vector<uint8_t> pieces(256 * 4, 0);
    for (uint32_t i = 0; i < m.n; ++i)
        for (uint32_t s = 0; s < 4; ++s) pieces[4 * i + s] = m.colours[i][s];
    const std::vector<uint32_t> cc = colour_constraints(m);
    const std::vector<uint32_t> cap = initial_capability(m);
    emp::GmState st;
    std::memset(&st, 0, sizeof(st));
    st.new_level = 1;
    for (uint32_t i = 0; i < 256; ++i) {
        st.position_index[i] = i < S ? i : 0xFFFFFFFFu;
        st.info_index[i] = i < S ? i : 0xFFFFFFFFu;
        st.played[i] = 0xFFFFFFFFu;
        st.max_played[i] = 0xFFFFFFFFu;
    }
    for (uint32_t i = 0; i < m.n; ++i) st.avail[i >> 5] |= 1u << (i & 31);
    // The array keeps whatever the previous call left.  Everything the kernel
    // reads before writing is overwritten here: the whole state, all piece
    // colours, the colour constraints of this puzzle's colours and the first
    // level of the info stack.  Deeper levels are written by the kernel before
    // they are read, exactly as with freshly allocated (uninitialised) memory.
    CUDA_TRY(cudaMemcpy(base + kOffState, &st, sizeof(st), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(base + kOffPieces, pieces.data(), pieces.size(), cudaMemcpyHostToDevice));
    if (!cc.empty()) CUDA_TRY(cudaMemcpy(base + kOffCc, cc.data(), sizeof(uint32_t) * cc.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(base + kOffInfos, cap.data(), sizeof(uint32_t) * cap.size(), cudaMemcpyHostToDevice));
    emp::GmLaunch P;
    P.pieces = reinterpret_cast<const uint8_t*>(base + kOffPieces);
    P.cc = reinterpret_cast<const uint32_t*>(base + kOffCc);
    P.infos = reinterpret_cast<uint32_t*>(base + kOffInfos);
    P.state = reinterpret_cast<emp::GmState*>(base + kOffState);
    P.n = S;
    P.width = m.width;
    P.ncolours = m.border_id;
    P.push_budget = cfg.push_budget;
    P.placement_budget = cfg.placement_budget;
    const unsigned long long ms_limit = cfg.timeout_ms ? cfg.timeout_ms : 3600000ull;
    P.timeout_ns = ms_limit * 1000000ull;
    // no CUDA events (they are driver objects to create and destroy): the time
    // reported is the host's wall time from launch to the result copy
    const auto t0 = std::chrono::steady_clock::now();
    cudaError_t le = emp::launch_gm(P, nullptr);
    if (le != cudaSuccess) return emp::cuda_fail(le, "glutton max launch");
    CUDA_TRY(cudaMemcpy(&st, base + kOffState, sizeof(st), cudaMemcpyDeviceToHost));
    const auto t1 = std::chrono::steady_clock::now();
    std::memset(result, 0, sizeof(*result));
    result->status = st.status;
    result->max_level = st.max;
    result->level = st.level <= S ? st.level : 0;
    board_from_played(m, st.max_played, st.max, result->best_board);
    board_from_played(m, st.played, result->level, result->final_board);
    result->trials = st.trials;
    result->pushes = st.pushes;
    result->pops = st.pops;
    result->passes = st.passes;
    result->levels = st.levels;
    result->kernel_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return st.status == 1 ? EMP_INCOMPLETE : EMP_OK;
}

extern "C" emp_status emp_glutton_wide_situation(emp_puzzle puzzle, uint32_t* infos, uint64_t capacity_words)
{
    emp::clear_error();
    if (!puzzle || !infos) return fail(EMP_ERR_INVALID, "emp_glutton_wide_situation: null argument");
    const std::vector<uint32_t> cap = initial_capability(puzzle->model);
    if (capacity_words < cap.size())
        return fail(EMP_ERR_INVALID, "emp_glutton_wide_situation: capacity below 32 words per position");
    std::memcpy(infos, cap.data(), cap.size() * sizeof(uint32_t));
    return EMP_OK;
}
