// C ABI of edge_matching_puzzle_b200 (include/emp_b200.h): puzzle handles and
// the exhaustive backtracker.
#include "emp_b200.h"
#include "emp_bt.h"
#include "emp_common.h"
#include "emp_model.h"
#include "emp_plan.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <chrono>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

using emp::DeviceBuffer;
using emp::fail;

extern "C" uint32_t emp_abi_version(void) { return EMP_ABI_VERSION; }

extern "C" const char* emp_last_error(void) { return emp::last_error().c_str(); }

extern "C" emp_status emp_generate_puzzle(uint32_t width, uint32_t height, uint32_t border_colors,
                                          uint32_t interior_colors, uint64_t seed, uint8_t* colours_out)
{
    emp::clear_error();
    if (!colours_out || width < 2 || height < 2 || width * height > emp::kMaxPieces)
        return fail(EMP_ERR_INVALID, "emp_generate_puzzle: need 2<=w,h, w*h<=256 and an output buffer");
    if (border_colors < 1 || interior_colors < 1 || border_colors + interior_colors + 1 > emp::kMaxColourId)
        return fail(EMP_ERR_INVALID, "emp_generate_puzzle: colour counts out of range");
    emp::generate_puzzle(width, height, border_colors, interior_colors, seed, colours_out);
    return EMP_OK;
}

extern "C" emp_status emp_puzzle_create(const emp_puzzle_desc* desc, emp_puzzle* out)
{
    emp::clear_error();
    if (!desc || !out || !desc->colours) return fail(EMP_ERR_INVALID, "emp_puzzle_create: null argument");
    *out = nullptr;
    std::unique_ptr<emp_puzzle_t> p(new (std::nothrow) emp_puzzle_t());
    if (!p) return fail(EMP_ERR_NOMEM, "emp_puzzle_create: out of host memory");
    std::string err;
    if (desc->width * desc->height > emp::kMaxPieces)
        return fail(EMP_ERR_UNSUPPORTED, "emp_puzzle_create: more than 256 pieces");
    if (!emp::build_model(desc->width, desc->height, desc->colours, p->model, err))
        return fail(err.find("colour ids above") != std::string::npos ? EMP_ERR_UNSUPPORTED : EMP_ERR_INVALID,
                    "emp_puzzle_create: " + err);
    const uint32_t n = p->model.n;
    if (desc->order) p->order.assign(desc->order, desc->order + n);
    else p->order = emp::order_basic(desc->width, desc->height);
    if (!emp::build_plan(p->model, p->order, p->plan, err)) return fail(EMP_ERR_INVALID, "emp_puzzle_create: " + err);
    emp::build_device_tables(p->model, p->plan, p->tables);
    for (uint32_t k = 0; k < 3; ++k)
        for (uint32_t e = 0; e < 4 * p->model.nb_kind(k); ++e)
            p->extra_count += (p->tables.blob[p->tables.tinfo_off[k] + e] >> 20) & 1u;
    *out = p.release();
    return EMP_OK;
}

extern "C" void emp_puzzle_destroy(emp_puzzle puzzle) { delete puzzle; }

extern "C" emp_status emp_puzzle_get_info(emp_puzzle p, emp_puzzle_info* info)
{
    emp::clear_error();
    if (!p || !info) return fail(EMP_ERR_INVALID, "emp_puzzle_get_info: null argument");
    info->width = p->model.width;
    info->height = p->model.height;
    info->nb_pieces = p->model.n;
    info->nb_center = p->model.nb_kind(0);
    info->nb_border = p->model.nb_kind(1);
    info->nb_corner = p->model.nb_kind(2);
    info->border_color_id = p->model.border_id;
    info->has_identical = p->model.has_identical ? 1u : 0u;
    info->identical_masks_with_extra = p->extra_count;
    return EMP_OK;
}

extern "C" emp_status emp_puzzle_export_tables(emp_puzzle p, uint32_t* out, uint64_t capacity, uint64_t* words)
{
    emp::clear_error();
    if (!p || !words) return fail(EMP_ERR_INVALID, "emp_puzzle_export_tables: null argument");
    *words = p->tables.blob.size();
    if (out && capacity >= p->tables.blob.size())
        std::memcpy(out, p->tables.blob.data(), sizeof(uint32_t) * p->tables.blob.size());
    return EMP_OK;
}

// ---------------------------------------------------------------------------
// exhaustive backtracker plans


namespace {

uint32_t auto_depth(uint32_t min_n)
{
    // Deep enough to give every resident thread several subtrees on the
    // project's 8x8 workloads, never the last level.
    const uint32_t d = min_n >= 36 ? 12 : min_n / 2;
    return std::max<uint32_t>(1, std::min<uint32_t>(d, min_n - 1));
}

emp_status expand(emp_bt_plan_t& pl)
{
    const uint32_t P = static_cast<uint32_t>(pl.puzzles.size());
    cudaStream_t st = nullptr;
    emp::BtLaunch L = pl.launch();
    DeviceBuffer parents, parent_puzzle, children, child_puzzle, counts, offsets, bsums, grand, lv;
    CUDA_TRY(lv.alloc(sizeof(unsigned long long) * 2 * P));
    CUDA_TRY(cudaMemsetAsync(lv.p, 0, lv.bytes, st));
    CUDA_TRY(parent_puzzle.alloc(sizeof(uint32_t) * P));
    {
        // subtrees are queued puzzle by puzzle, smaller puzzles first: under a
        // deadline the cheap instances of a mixed batch finish before the threads
        // are taken by large ones (within a puzzle, subtrees stay in search order)
        std::vector<uint32_t> ids(P);
        for (uint32_t i = 0; i < P; ++i) ids[i] = i;
        std::stable_sort(ids.begin(), ids.end(), [&](uint32_t a, uint32_t b) {
            return pl.puzzles[a]->model.n < pl.puzzles[b]->model.n;
        });
        CUDA_TRY(cudaMemcpyAsync(parent_puzzle.p, ids.data(), sizeof(uint32_t) * P, cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    CUDA_TRY(parents.alloc(2));
    CUDA_TRY(grand.alloc(sizeof(uint64_t)));
    uint64_t np = P;
    unsigned long long* lnodes = lv.as<unsigned long long>();
    // per puzzle split depths: a puzzle stops expanding (is frozen) once it has
    // split_subtrees prefixes, reaches its depth limit or runs out of prefixes
    DeviceBuffer frozen_dev;
    std::vector<uint8_t> frozen(P, 0);
    std::vector<uint32_t> cap(P);
    std::vector<unsigned long long> seen(P, 0), now(P, 0);
    uint32_t levels = pl.depth;
    pl.puzzle_depth.assign(P, pl.depth);
    if (pl.adaptive) {
        CUDA_TRY(frozen_dev.alloc(P));
        CUDA_TRY(cudaMemsetAsync(frozen_dev.p, 0, P, st));
        levels = 0;
        for (uint32_t i = 0; i < P; ++i) {
            const uint32_t lim = pl.cfg.split_depth ? std::min<uint32_t>(pl.cfg.split_depth, 64u) : 64u;
            cap[i] = std::max<uint32_t>(1u, std::min<uint32_t>(lim, pl.puzzles[i]->model.n - 1));
            levels = std::max(levels, cap[i]);
        }
    }
    uint32_t level = 0;
    for (; level < levels; ++level) {
        CUDA_TRY(counts.alloc(sizeof(uint32_t) * std::max<uint64_t>(np, 1)));
        CUDA_TRY(offsets.alloc(sizeof(uint64_t) * std::max<uint64_t>(np, 1)));
        CUDA_TRY(bsums.alloc(sizeof(uint64_t) * emp::scan_block_sum_words(np)));
        const uint8_t* fz = pl.adaptive ? frozen_dev.as<uint8_t>() : nullptr;
        CUDA_TRY(emp::launch_expand_frozen(L, parents.as<uint16_t>(), parent_puzzle.as<uint32_t>(), np, level,
                                           counts.as<uint32_t>(), nullptr, nullptr, nullptr, lnodes, lnodes + P, 0,
                                           fz, st));
        CUDA_TRY(emp::launch_scan(counts.as<uint32_t>(), np, offsets.as<uint64_t>(), bsums.as<uint64_t>(),
                                  grand.as<uint64_t>(), st));
        uint64_t total = 0;
        CUDA_TRY(cudaMemcpyAsync(&total, grand.p, sizeof(uint64_t), cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        CUDA_TRY(children.alloc(sizeof(uint16_t) * std::max<uint64_t>(total, 1) * (level + 1)));
        CUDA_TRY(child_puzzle.alloc(sizeof(uint32_t) * std::max<uint64_t>(total, 1)));
        CUDA_TRY(emp::launch_expand_frozen(L, parents.as<uint16_t>(), parent_puzzle.as<uint32_t>(), np, level,
                                           counts.as<uint32_t>(), offsets.as<uint64_t>(), children.as<uint16_t>(),
                                           child_puzzle.as<uint32_t>(), lnodes, lnodes + P, 1, fz, st));
        std::swap(parents, children);
        std::swap(parent_puzzle, child_puzzle);
        if (pl.dump) {
            // keep this level's prefixes (length level + 1) for the solution indices
            if (pl.level_prefixes.size() < level + 2) {
                pl.level_prefixes.resize(level + 2);
                pl.level_counts.resize(level + 2, 0);
            }
            DeviceBuffer keep;
            CUDA_TRY(keep.alloc(sizeof(uint16_t) * std::max<uint64_t>(total, 1) * (level + 1)));
            if (total)
                CUDA_TRY(cudaMemcpyAsync(keep.p, parents.p, sizeof(uint16_t) * total * (level + 1),
                                         cudaMemcpyDeviceToDevice, st));
            pl.level_prefixes[level + 1] = std::move(keep);
            pl.level_counts[level + 1] = total;
        }
        np = total;
        if (pl.adaptive) {
            // placements of this level per puzzle = its prefixes after this level
            CUDA_TRY(cudaMemcpyAsync(now.data(), lnodes, sizeof(unsigned long long) * P, cudaMemcpyDeviceToHost, st));
            CUDA_TRY(cudaStreamSynchronize(st));
            bool all = true;
            for (uint32_t i = 0; i < P; ++i) {
                if (frozen[i]) continue;
                const unsigned long long prefixes = now[i] - seen[i];
                seen[i] = now[i];
                pl.puzzle_depth[i] = level + 1;
                if (prefixes >= pl.cfg.split_subtrees || level + 1 >= cap[i] || !prefixes) frozen[i] = 1;
                all = all && frozen[i];
            }
            CUDA_TRY(cudaMemcpyAsync(frozen_dev.p, frozen.data(), P, cudaMemcpyHostToDevice, st));
            CUDA_TRY(cudaStreamSynchronize(st));
            if (all) {
                ++level;
                break;
            }
        }
        if (!np) {
            ++level;
            break;
        }
    }
    if (pl.adaptive) pl.depth = level;
    pl.exp_nodes.assign(P, 0);
    pl.exp_sols.assign(P, 0);
    CUDA_TRY(cudaMemcpyAsync(pl.exp_nodes.data(), lnodes, sizeof(unsigned long long) * P, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaMemcpyAsync(pl.exp_sols.data(), lnodes + P, sizeof(unsigned long long) * P, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    pl.n_all = np;
    if (pl.adaptive) {
        CUDA_TRY(pl.puzzle_depth_dev.alloc(sizeof(uint32_t) * P));
        CUDA_TRY(cudaMemcpyAsync(pl.puzzle_depth_dev.p, pl.puzzle_depth.data(), sizeof(uint32_t) * P,
                                 cudaMemcpyHostToDevice, st));
        CUDA_TRY(cudaStreamSynchronize(st));
    }
    pl.prefixes = std::move(parents);
    pl.prefix_puzzle = std::move(parent_puzzle);
    return EMP_OK;
}

}  // namespace

// The records are built on the plan's own stream and a run waits for them on its
// stream (ev_select), so a selection does not stall work queued on other streams.
// Buffers only grow: the graph of a graph run stays valid while the initial-record
// buffer stays where it is (its first round reads the record count on the device).
emp_status plan_build_initial(emp_bt_plan_t& pl, uint64_t first, uint64_t stride, uint64_t count)
{
    if (!pl.select_stream) {
        CUDA_TRY(cudaStreamCreateWithFlags(&pl.select_stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&pl.ev_select, cudaEventDisableTiming));
    }
    // the previous run may still read the buffers: order the rebuild after it
    if (pl.ran) CUDA_TRY(cudaStreamWaitEvent(pl.select_stream, pl.ev1, 0));
    CUDA_TRY(pl.rec_init.reserve(sizeof(uint32_t) * pl.rec_words * std::max<uint64_t>(count, 1)));
    if (pl.cfg.keep_subtree_counts) {
        CUDA_TRY(pl.item_nodes.reserve(sizeof(unsigned long long) * std::max<uint64_t>(count, 1)));
        CUDA_TRY(pl.item_sols.reserve(sizeof(unsigned long long) * std::max<uint64_t>(count, 1)));
    }
    CUDA_TRY(emp::launch_make_records(pl.prefixes.as<uint16_t>(), pl.prefix_puzzle.as<uint32_t>(), pl.depth, first,
                                      stride, count, pl.rec_words, pl.rec_init.as<uint32_t>(), pl.select_stream,
                                      pl.adaptive ? pl.puzzle_depth_dev.as<uint32_t>() : nullptr,
                                      pl.ctl.as<emp::BtRunCtl>()));
    CUDA_TRY(cudaEventRecord(pl.ev_select, pl.select_stream));
    if (pl.graph_exec && pl.graph_rec_init != pl.rec_init.p) pl.drop_graph();
    pl.n_init = count;
    return EMP_OK;
}

namespace {
struct ResumeSpec {
    const uint16_t* situation;
    uint32_t placed;
};
emp_status create_plan(const emp_puzzle* puzzles, uint32_t count, const emp_bt_config* config, bool dump,
                       emp_bt_plan* out, const ResumeSpec* resume = nullptr);
}  // namespace

extern "C" emp_status emp_bt_plan_create(const emp_puzzle* puzzles, uint32_t count, const emp_bt_config* config,
                                         emp_bt_plan* out)
{
    return create_plan(puzzles, count, config, false, out);
}

namespace {

// Work records of a search resumed from a partial situation: what
// emp_strategy::set_initial_state leaves for specific_run
// (include/emp_strategy.h:418-467).  Each placed level takes its candidates in
// order up to the situation's transition, applying select_piece (and so the
// identical-piece masks) to every one tried; the search then starts at the LAST
// placed level (the loop steps back from the first empty position), whose
// candidate set specific_run recomputes in full, and it ends when level 1 is
// exhausted (:398, level 0 keeps its transition).  So the records, in visiting
// order, are: the last placed level with all its candidates, then every shallower
// level down to level 1 with the candidates it has left.  The candidate words come
// from the same tables the kernels read.
emp_status resume_records(const emp_puzzle_t& pz, const uint16_t* situation, uint32_t placed, uint32_t rec_words,
                          uint32_t max_kw, std::vector<uint32_t>& recs, uint64_t& count)
{
    const std::vector<uint32_t>& b = pz.tables.blob;
    const uint32_t n = b[1], ncol = b[2], desc_off = b[14], init = b[21], aw = b[9];
    if (placed < 2 || placed >= n)
        return fail(EMP_ERR_INVALID, "emp_bt_resume: the situation must place between 2 and n-1 pieces");
    auto u64at = [&](size_t off) { return static_cast<uint64_t>(b[off]) | (static_cast<uint64_t>(b[off + 1]) << 32); };
    std::vector<uint64_t> av(aw);
    for (uint32_t w = 0; w < aw; ++w) av[w] = u64at(init + 2 * w);
    std::vector<uint32_t> stk(n, 0);
    std::vector<std::vector<uint64_t>> rem(placed);
    std::vector<uint8_t> spilled(placed, 0);
    auto facing = [&](uint32_t e, uint32_t side) { return (e >> (5 * ((side + 2) & 3u))) & 31u; };
    for (uint32_t l = 0; l < placed; ++l) {
        const uint32_t* d = &b[desc_off + emp::kDescWords * l];
        const uint32_t kw = d[0] & 0xFFu, nextra = (d[0] >> 13) & 7u, aoff = d[0] >> 16;
        const uint32_t ea = stk[d[1] & 0xFFu], eb = stk[(d[1] >> 8) & 0xFFu];
        const uint32_t row = d[2] + ((ea >> ((d[1] >> 16) & 0xFFu)) & 31u) * (d[3] & 0xFFFFu) +
                             ((eb >> (d[1] >> 24)) & 31u) * (d[3] >> 16);
        std::vector<uint64_t> c(kw);
        for (uint32_t w = 0; w < kw; ++w) c[w] = u64at(row + 2 * w) & av[aoff + w];
        for (uint32_t j = 0; j < nextra; ++j) {
            const uint32_t sd = (d[7] >> (2 * j)) & 3u, lev = (d[7] >> (8 + 8 * j)) & 0xFFu;
            const size_t sm = d[4] + static_cast<size_t>((sd * ncol + facing(stk[lev], sd)) * kw) * 2;
            for (uint32_t w = 0; w < kw; ++w) c[w] &= u64at(sm + 2 * w);
        }
        const uint32_t want = situation[l];
        uint32_t t = ~0u;
        while (t != want) {
            t = ~0u;
            for (uint32_t w = 0; w < kw && t == ~0u; ++w)
                if (c[w]) t = 64 * w + static_cast<uint32_t>(__builtin_ctzll(c[w]));
            if (t == ~0u)
                return fail(EMP_ERR_INVALID, "emp_bt_resume: the situation's piece at level " + std::to_string(l) +
                                                 " is not reachable in the search order");
            const uint32_t ti = b[d[5] + t];
            if ((ti >> 20) & 1u) {  // select_piece with an identical mask (emp_position_strategy.h:197-200)
                for (uint32_t w = 0; w < kw; ++w) c[w] &= u64at(d[6] + static_cast<size_t>(t) * kw * 2 + 2 * w);
                spilled[l] = 1;
            } else {
                c[t >> 6] &= ~(uint64_t(1) << (t & 63u));
            }
        }
        rem[l] = c;
        av[aoff + (t >> 6)] &= ~(uint64_t(0xF) << (t & 60u));
        stk[l] = b[d[5] + t] & 0xFFFFFu;
    }
    recs.clear();
    count = 0;
    auto emit = [&](uint32_t len, uint32_t start, const std::vector<uint64_t>* rest) {
        std::vector<uint32_t> r(rec_words, 0);
        r[0] = static_cast<uint32_t>(count);
        r[2] = len | (start << 16);
        r[3] = rest ? (1u << 16) : 0u;
        for (uint32_t j = 0; j < len; ++j) r[4 + (j >> 1)] |= static_cast<uint32_t>(situation[j]) << (16 * (j & 1));
        if (rest)
            for (uint32_t w = 0; w < rest->size() && w < max_kw; ++w) {
                r[rec_words - 2 * max_kw + 2 * w] = static_cast<uint32_t>((*rest)[w]);
                r[rec_words - 2 * max_kw + 2 * w + 1] = static_cast<uint32_t>((*rest)[w] >> 32);
            }
        recs.insert(recs.end(), r.begin(), r.end());
        ++count;
    };
    emit(placed - 1, 0, nullptr);
    for (uint32_t l = placed - 1; l-- > 1;) {
        bool any = false;
        for (uint64_t v : rem[l]) any = any || v;
        if (any) emit(l, situation[l] + 1u, spilled[l] ? &rem[l] : nullptr);
    }
    return EMP_OK;
}

emp_status create_plan(const emp_puzzle* puzzles, uint32_t count, const emp_bt_config* config, bool dump,
                       emp_bt_plan* out, const ResumeSpec* resume)
{
    emp::clear_error();
    if (!puzzles || !count || !out) return fail(EMP_ERR_INVALID, "emp_bt_plan_create: no puzzle");
    if (count > 65535) return fail(EMP_ERR_UNSUPPORTED, "emp_bt_plan_create: at most 65535 puzzles per plan");
    *out = nullptr;
    std::unique_ptr<emp_bt_plan_t> pl(new (std::nothrow) emp_bt_plan_t());
    if (!pl) return fail(EMP_ERR_NOMEM, "emp_bt_plan_create: out of host memory");
    if (config) pl->cfg = *config;
    else pl->cfg.device = -1;
    uint32_t min_n = ~0u;
    for (uint32_t i = 0; i < count; ++i) {
        if (!puzzles[i]) return fail(EMP_ERR_INVALID, "emp_bt_plan_create: null puzzle");
        pl->puzzles.push_back(puzzles[i]);
        const emp::DeviceTables& t = puzzles[i]->tables;
        min_n = std::min(min_n, t.n);
        pl->max_levels = std::max(pl->max_levels, t.n);
        pl->max_avail = std::max(pl->max_avail, t.avail_words);
        pl->max_kw = std::max(pl->max_kw, t.max_kw);
    }
    pl->adaptive = pl->cfg.split_subtrees != 0 && !resume;
    pl->depth = resume ? 0u : (pl->cfg.split_depth ? pl->cfg.split_depth : auto_depth(min_n));
    if (resume) {
        if (count != 1) return fail(EMP_ERR_INVALID, "emp_bt_resume: one puzzle");
    } else if (pl->adaptive) {
        if (pl->cfg.split_depth > 64)
            return fail(EMP_ERR_INVALID, "emp_bt_plan_create: split depth limit must be at most 64");
    } else if (pl->depth >= min_n || pl->depth > 64) {
        return fail(EMP_ERR_INVALID, "emp_bt_plan_create: split depth must be below the piece count and at most 64");
    }
    pl->rec_words = emp::record_words(pl->max_levels, pl->max_kw);
    EMP_TRY(emp::select_device(pl->cfg.device, &pl->device));
    // tables
    std::vector<uint32_t> blob;
    std::vector<uint64_t> offs;
    for (emp_puzzle p : pl->puzzles) {
        offs.push_back(blob.size());  // blobs are multiples of 4 words: 16-byte aligned tables
        blob.insert(blob.end(), p->tables.blob.begin(), p->tables.blob.end());
    }
    CUDA_TRY(pl->tables.alloc(sizeof(uint32_t) * blob.size()));
    CUDA_TRY(pl->poff.alloc(sizeof(uint64_t) * offs.size()));
    CUDA_TRY(cudaMemcpy(pl->tables.p, blob.data(), sizeof(uint32_t) * blob.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(pl->poff.p, offs.data(), sizeof(uint64_t) * offs.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(pl->counters.alloc(2 * sizeof(unsigned long long)));
    CUDA_TRY(pl->totals.alloc(2 * sizeof(unsigned long long) * count));
    CUDA_TRY(pl->first_item.alloc(sizeof(unsigned long long) * count));
    CUDA_TRY(pl->records.alloc(sizeof(emp::FirstRecord) * count));
    CUDA_TRY(pl->flags.alloc(2 * sizeof(int)));
    CUDA_TRY(pl->ctl.alloc(sizeof(emp::BtRunCtl)));
    CUDA_TRY(pl->incomplete.alloc(sizeof(uint32_t) * count));
    CUDA_TRY(pl->prefix_out.alloc(sizeof(uint16_t) * 256));
    CUDA_TRY(cudaEventCreate(&pl->ev0));
    CUDA_TRY(cudaEventCreate(&pl->ev1));
    CUDA_TRY(cudaEventCreate(&pl->evr0));
    CUDA_TRY(cudaEventCreate(&pl->evr1));
    if (pl->cfg.use_graph) CUDA_TRY(cudaStreamCreateWithFlags(&pl->capture_stream, cudaStreamNonBlocking));
    pl->dump = dump;
    std::vector<uint32_t> resume_recs;
    if (resume) {
        EMP_TRY(resume_records(*pl->puzzles[0], resume->situation, resume->placed, pl->rec_words, pl->max_kw,
                               resume_recs, pl->n_all));
        pl->exp_nodes.assign(1, 0);
        pl->exp_sols.assign(1, 0);
        pl->puzzle_depth.assign(1, 0);
    } else {
        EMP_TRY(expand(*pl));
    }
    // hot tables in shared memory when the plan holds one puzzle
    const uint32_t hot = (pl->puzzles[0]->tables.blob[26] + 3u) & ~3u;
    const bool want_smem = pl->cfg.table_placement == 2 || (pl->cfg.table_placement == 0 && count == 1);
    pl->smem_tab_words = (want_smem && count == 1 && hot * 4 <= 64 * 1024) ? hot : 0;
    if (pl->cfg.table_placement == 2 && !pl->smem_tab_words)
        return fail(EMP_ERR_UNSUPPORTED, "tables can only be staged in shared memory for a single puzzle up to 64 KB");
    // launch geometry: the block size with the most resident warps per SM
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, pl->device));
    if (pl->cfg.stack_placement > 4)
        return fail(EMP_ERR_INVALID, "stack_placement must be 0 (default), 1, 2, 3 or 4");
    // default: the shared 32-bit stack next to staged tables (a single puzzle) while it
    // leaves at least 16 warps per SM, else the global stack.  Measured on a B200: 8x8
    // 2.7e10 placements/s shared against 2.0e10 global; 12x12 (8 warps per SM shared)
    // 1.8e10 against 2.3e10; the 4096-instance batch (tables in global memory) 2.2e10
    // against 2.7e10.
    const bool default_stack = pl->cfg.stack_placement == 0;
    pl->stack_mode = default_stack ? (pl->smem_tab_words ? emp::kStackShared32 : emp::kStackGlobal32)
                                   : static_cast<int>(pl->cfg.stack_placement);
    std::vector<uint32_t> candidates;
    if (pl->cfg.threads_per_block) candidates.push_back(pl->cfg.threads_per_block);
    else candidates = {128, 256, 512};
    // the block size with the most resident warps per SM for the current stack mode
    int best_warps = 0;
    auto pick_geometry = [&]() -> emp_status {
        best_warps = 0;
        for (uint32_t threads : candidates) {
            const void* fn = emp::dfs_kernel_symbol(pl->max_kw, pl->smem_tab_words != 0, threads, pl->stack_mode);
            if (!fn) return fail(EMP_ERR_INVALID, "threads_per_block must be 128, 256 or 512");
            const size_t smem =
                emp::dfs_smem_bytes(pl->max_levels, pl->max_avail, threads, pl->smem_tab_words, pl->stack_mode);
            if (smem > static_cast<size_t>(prop.sharedMemPerBlockOptin)) continue;
            CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
            int per_sm = 0;
            CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, static_cast<int>(threads), smem));
            if (pl->cfg.blocks_per_sm) per_sm = std::min<int>(per_sm, static_cast<int>(pl->cfg.blocks_per_sm));
            const int warps = per_sm * static_cast<int>(threads / 32);
            if (per_sm >= 1 && warps > best_warps) {
                best_warps = warps;
                pl->threads = threads;
                pl->blocks = static_cast<uint32_t>(per_sm) * static_cast<uint32_t>(prop.multiProcessorCount);
            }
        }
        return EMP_OK;
    };
    EMP_TRY(pick_geometry());
    if (default_stack && pl->stack_mode == emp::kStackShared32 && best_warps < 16) {
        pl->stack_mode = emp::kStackGlobal32;
        EMP_TRY(pick_geometry());
    }
    if (!best_warps)
        return fail(EMP_ERR_UNSUPPORTED, "per-thread DFS state does not fit shared memory; use fewer threads per block");
    CUDA_TRY(pl->spill.alloc(sizeof(uint64_t) * static_cast<size_t>(pl->blocks) * pl->threads * pl->max_levels *
                             pl->max_kw));
    if (pl->stack_mode == emp::kStackGlobal32)
        CUDA_TRY(pl->stack.alloc(sizeof(uint32_t) * static_cast<size_t>(pl->blocks) * pl->threads * pl->max_levels));
    // round queues: room for every resident thread to hand back a full path twice
    const uint64_t resident = static_cast<uint64_t>(pl->blocks) * pl->threads;
    pl->capacity = std::max<uint64_t>(resident * 2 * (pl->max_levels - pl->depth + 1) / 4, 1u << 16);
    pl->capacity = std::min<uint64_t>(pl->capacity, (uint64_t)1 << 23);
    CUDA_TRY(pl->rec_a.alloc(sizeof(uint32_t) * pl->rec_words * pl->capacity));
    CUDA_TRY(pl->rec_b.alloc(sizeof(uint32_t) * pl->rec_words * pl->capacity));
    // default split budget.  Without a deadline the whole tree gets searched and a small
    // budget shares each round's tail out sooner: measured on a B200 over slices of four
    // 8x8 workload puzzles, 2.68e10 placements/s at 2048 steps, 3.65e10 at 256, 3.79e10
    // at 64.  Under a deadline, instances that cannot finish would hand 64-step pieces
    // back every round and bury the last records of the small ones (a batch of small
    // puzzles and two 9x9 ones left small ones unfinished at 400 ms); 2048 keeps records
    // whole longer, so the small instances finish first.
    pl->budget = pl->cfg.split_budget ? pl->cfg.split_budget : (pl->cfg.timeout_ms ? 2048u : 64u);
    if (resume) {
        CUDA_TRY(pl->rec_init.reserve(sizeof(uint32_t) * resume_recs.size()));
        CUDA_TRY(cudaMemcpy(pl->rec_init.p, resume_recs.data(), sizeof(uint32_t) * resume_recs.size(),
                            cudaMemcpyHostToDevice));
        const unsigned long long n_init = pl->n_all;
        CUDA_TRY(cudaMemcpy(reinterpret_cast<char*>(pl->ctl.p) + offsetof(emp::BtRunCtl, n_init), &n_init,
                            sizeof(n_init), cudaMemcpyHostToDevice));
        if (pl->cfg.keep_subtree_counts) {
            CUDA_TRY(pl->item_nodes.reserve(sizeof(unsigned long long) * pl->n_all));
            CUDA_TRY(pl->item_sols.reserve(sizeof(unsigned long long) * pl->n_all));
        }
        pl->n_init = pl->n_all;
        pl->resumed = true;
    } else {
        EMP_TRY(plan_build_initial(*pl, 0, 1, pl->n_all));
    }
    *out = pl.release();
    return EMP_OK;
}

}  // namespace

extern "C" emp_status emp_bt_plan_subtrees(emp_bt_plan plan, uint64_t* subtrees)
{
    emp::clear_error();
    if (!plan || !subtrees) return fail(EMP_ERR_INVALID, "emp_bt_plan_subtrees: null argument");
    *subtrees = plan->n_all;
    return EMP_OK;
}

extern "C" emp_status emp_bt_plan_select(emp_bt_plan plan, uint64_t first, uint64_t stride, uint64_t count)
{
    emp::clear_error();
    if (!plan || !stride) return fail(EMP_ERR_INVALID, "emp_bt_plan_select: null plan or zero stride");
    if (plan->resumed) return fail(EMP_ERR_INVALID, "emp_bt_plan_select: not for a resumed search");
    if (count && first + (count - 1) * stride >= plan->n_all)
        return fail(EMP_ERR_INVALID, "emp_bt_plan_select: selection past the last subtree");
    CUDA_TRY(cudaSetDevice(plan->device));
    EMP_TRY(plan_build_initial(*plan, first, stride, count));
    plan->sampled = true;
    return EMP_OK;
}

namespace {

constexpr uint32_t kMaxRounds = 100000;

// The whole run as one graph:
//   reset -> zero the queue counters -> DFS round 1 (initial records) -> advance
//   -> while (records were handed back) { copy them to the input queue -> DFS -> advance }
// The advance kernel sets the loop's condition on the device, so the host
// launches the graph once and never waits between rounds.
emp_status build_graph(emp_bt_plan_t& pl)
{
    cudaStream_t cs = pl.capture_stream;
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaGraphCreate(&g, 0));
    pl.graph = g;
    cudaGraphConditionalHandle loop;
    CUDA_TRY(cudaGraphConditionalHandleCreate(&loop, g, 0, 0));
    emp::BtLaunch P = pl.launch();
    P.in_rec = pl.rec_init.as<uint32_t>();
    P.n_in = 0;
    P.n_in_from_ctl = 1;  // the selection's count, left in the run control block by make_records
    P.out_rec = pl.rec_b.as<uint32_t>();
    pl.graph_rec_init = pl.rec_init.p;
    CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, g, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = emp::launch_bt_reset(P, static_cast<uint32_t>(pl.puzzles.size()), cs);
    if (e == cudaSuccess) e = cudaMemsetAsync(pl.counters.p, 0, pl.counters.bytes, cs);
    if (e == cudaSuccess && pl.item_nodes.p) e = cudaMemsetAsync(pl.item_nodes.p, 0, pl.item_nodes.bytes, cs);
    if (e == cudaSuccess && pl.item_sols.p) e = cudaMemsetAsync(pl.item_sols.p, 0, pl.item_sols.bytes, cs);
    if (e == cudaSuccess) e = emp::launch_dfs(P, pl.blocks, pl.threads, cs);
    if (e == cudaSuccess) e = emp::launch_round_advance(P, loop, kMaxRounds, cs);
    cudaError_t e2 = cudaStreamEndCapture(cs, &g);
    CUDA_TRY(e);
    CUDA_TRY(e2);
    // the loop hangs below the captured chain's last node
    size_t n = 0;
    CUDA_TRY(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    CUDA_TRY(cudaGraphGetNodes(g, nodes.data(), &n));
    cudaGraphNode_t sink = nullptr;
    for (cudaGraphNode_t nd : nodes) {
        size_t deps = 0;
        CUDA_TRY(cudaGraphNodeGetDependentNodes(nd, nullptr, &deps));
        if (!deps) sink = nd;
    }
    if (!sink) return fail(EMP_ERR_CUDA, "graph build: no last node");
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = loop;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t cnode;
    CUDA_TRY(cudaGraphAddNode(&cnode, g, &sink, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    emp::BtLaunch Q = P;
    Q.in_rec = pl.rec_a.as<uint32_t>();
    CUDA_TRY(cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    e = emp::launch_round_copy(Q, pl.rec_a.as<uint32_t>(), pl.rec_b.as<uint32_t>(), cs);
    if (e == cudaSuccess) e = emp::launch_dfs(Q, pl.blocks, pl.threads, cs);
    if (e == cudaSuccess) e = emp::launch_round_advance(Q, loop, kMaxRounds, cs);
    e2 = cudaStreamEndCapture(cs, &body);
    CUDA_TRY(e);
    CUDA_TRY(e2);
    CUDA_TRY(cudaGraphInstantiate(&pl.graph_exec, g, 0));
    return EMP_OK;
}

}  // namespace

extern "C" emp_status emp_bt_plan_run(emp_bt_plan plan, void* stream)
{
    emp::clear_error();
    if (!plan) return fail(EMP_ERR_INVALID, "emp_bt_plan_run: null plan");
    CUDA_TRY(cudaSetDevice(plan->device));
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (plan->ev_select) CUDA_TRY(cudaStreamWaitEvent(st, plan->ev_select, 0));
    if (plan->cfg.use_graph) {
        if (!plan->graph_exec) {
            const emp_status s = build_graph(*plan);
            if (s != EMP_OK) {
                plan->drop_graph();
                return s;
            }
        }
        CUDA_TRY(cudaEventRecord(plan->ev0, st));
        CUDA_TRY(cudaGraphLaunch(plan->graph_exec, st));
        CUDA_TRY(cudaEventRecord(plan->ev1, st));
        plan->graph_ran = true;
        plan->ran = true;
        return EMP_OK;
    }
    plan->graph_ran = false;
    emp::BtLaunch P = plan->launch();
    CUDA_TRY(emp::launch_bt_reset(P, static_cast<uint32_t>(plan->puzzles.size()), st));
    if (plan->item_nodes.p) {
        CUDA_TRY(cudaMemsetAsync(plan->item_nodes.p, 0, plan->item_nodes.bytes, st));
        CUDA_TRY(cudaMemsetAsync(plan->item_sols.p, 0, plan->item_sols.bytes, st));
    }
    CUDA_TRY(cudaEventRecord(plan->ev0, st));
    // rounds: the initial records, then the work handed back by each round
    const uint32_t* in = plan->rec_init.as<uint32_t>();
    uint64_t n_in = plan->n_init;
    DeviceBuffer* out = &plan->rec_a;
    DeviceBuffer* spare = &plan->rec_b;
    plan->rounds = 0;
    plan->busy_ms = 0;
    plan->records_in = 0;
    plan->records_out = 0;
    while (n_in) {
        plan->records_in += n_in;
        CUDA_TRY(cudaMemsetAsync(plan->counters.p, 0, plan->counters.bytes, st));
        P.in_rec = in;
        P.n_in = n_in;
        P.out_rec = out->as<uint32_t>();
        CUDA_TRY(cudaEventRecord(plan->evr0, st));
        CUDA_TRY(emp::launch_dfs(P, plan->blocks, plan->threads, st));
        CUDA_TRY(cudaEventRecord(plan->evr1, st));
        ++plan->rounds;
        unsigned long long tail = 0;
        CUDA_TRY(cudaMemcpyAsync(&tail, plan->counters.as<unsigned long long>() + 1, sizeof(tail),
                                 cudaMemcpyDeviceToHost, st));
        CUDA_TRY(cudaStreamSynchronize(st));
        float rms = 0;
        CUDA_TRY(cudaEventElapsedTime(&rms, plan->evr0, plan->evr1));
        plan->busy_ms += rms;
        n_in = std::min<uint64_t>(tail, plan->capacity);
        plan->records_out += n_in;
        in = out->as<uint32_t>();
        std::swap(out, spare);
        if (plan->rounds > kMaxRounds) return fail(EMP_ERR_CUDA, "emp_bt_plan_run: too many rounds");
    }
    CUDA_TRY(cudaEventRecord(plan->ev1, st));
    plan->ran = true;
    return EMP_OK;
}

extern "C" emp_status emp_bt_plan_results(emp_bt_plan plan, emp_bt_result* results)
{
    emp::clear_error();
    if (!plan || !results) return fail(EMP_ERR_INVALID, "emp_bt_plan_results: null argument");
    if (!plan->ran) return fail(EMP_ERR_INVALID, "emp_bt_plan_results: plan has not run");
    CUDA_TRY(cudaSetDevice(plan->device));
    CUDA_TRY(cudaEventSynchronize(plan->ev1));
    float ms = 0;
    CUDA_TRY(cudaEventElapsedTime(&ms, plan->ev0, plan->ev1));
    const uint32_t P = static_cast<uint32_t>(plan->puzzles.size());
    std::vector<unsigned long long> tot(2 * P);
    std::vector<emp::FirstRecord> rec(P);
    int flags[2];
    CUDA_TRY(cudaMemcpy(tot.data(), plan->totals.p, sizeof(unsigned long long) * 2 * P, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(rec.data(), plan->records.p, sizeof(emp::FirstRecord) * P, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(flags, plan->flags.p, sizeof(flags), cudaMemcpyDeviceToHost));
    std::vector<uint32_t> incomplete(P);
    CUDA_TRY(cudaMemcpy(incomplete.data(), plan->incomplete.p, sizeof(uint32_t) * P, cudaMemcpyDeviceToHost));
    (void)flags;
    emp::BtRunCtl c{};
    CUDA_TRY(cudaMemcpy(&c, plan->ctl.p, sizeof(c), cudaMemcpyDeviceToHost));
    const uint32_t first_found_us =
        c.first_found_ns ? static_cast<uint32_t>(std::min<unsigned long long>((c.first_found_ns - c.start_ns) / 1000,
                                                                              0xFFFFFFFFull))
                         : 0u;
    if (plan->graph_ran) {
        if (c.n_in) return fail(EMP_ERR_CUDA, "emp_bt_plan_results: the graph run stopped after too many rounds");
        plan->rounds = static_cast<uint32_t>(c.rounds);
        plan->records_in = c.records_in;
        plan->records_out = c.records_out;
        plan->busy_ms = ms;
    }
    for (uint32_t i = 0; i < P; ++i) {
        emp_bt_result& r = results[i];
        std::memset(&r, 0, sizeof(r));
        const emp_puzzle pz = plan->puzzles[i];
        r.subtrees = plan->n_init;
        r.split_depth = plan->puzzle_depth.empty() ? plan->depth : plan->puzzle_depth[i];
        r.expansion_nodes = plan->exp_nodes[i];
        r.nodes = tot[2 * i] + (plan->sampled ? 0 : plan->exp_nodes[i]);
        r.solutions = tot[2 * i + 1] + (plan->sampled ? 0 : plan->exp_sols[i]);
        r.status = incomplete[i] ? EMP_INCOMPLETE : (rec[i].missed ? EMP_FIRST_LOST : EMP_OK);
        r.kernel_ms = ms;
        r.rounds = plan->rounds;
        r.first_found_us = first_found_us;
        r.dfs_busy_ms = plan->busy_ms;
        r.work_records = plan->records_in;
        r.handed_back = plan->records_out;
        for (uint32_t pos = 0; pos < 256; ++pos) r.first_solution[pos] = 0xFFFFFFFFu;
        if (rec[i].has && !rec[i].missed) {
            for (uint32_t l = 0; l < pz->model.n; ++l) {
                const emp::LevelPlan& lp = pz->plan[l];
                const uint32_t t = rec[i].t[l];
                const uint32_t piece = pz->model.members[lp.kind][t >> 2];
                r.first_solution[lp.position] = (piece << 2) | (t & 3u);
            }
            r.has_first_solution = 1;
        }
    }
    return EMP_OK;
}

extern "C" emp_status emp_bt_plan_subtree_counts(emp_bt_plan plan, uint64_t* nodes, uint64_t* solutions,
                                                 uint64_t capacity)
{
    emp::clear_error();
    if (!plan || !nodes || !solutions) return fail(EMP_ERR_INVALID, "emp_bt_plan_subtree_counts: null argument");
    if (!plan->item_nodes.p) return fail(EMP_ERR_INVALID, "emp_bt_plan_subtree_counts: keep_subtree_counts was 0");
    const uint64_t n = std::min<uint64_t>(capacity, plan->n_init);
    CUDA_TRY(cudaSetDevice(plan->device));
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(nodes, plan->item_nodes.p, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(solutions, plan->item_sols.p, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" emp_status emp_bt_plan_subtree_prefix(emp_bt_plan plan, uint64_t index, uint16_t* prefix, uint32_t capacity)
{
    emp::clear_error();
    if (!plan || !prefix) return fail(EMP_ERR_INVALID, "emp_bt_plan_subtree_prefix: null argument");
    if (index >= plan->n_init || capacity < plan->depth) return fail(EMP_ERR_INVALID, "emp_bt_plan_subtree_prefix: bad index");
    CUDA_TRY(cudaSetDevice(plan->device));
    if (plan->ev_select) CUDA_TRY(cudaEventSynchronize(plan->ev_select));
    CUDA_TRY(emp::launch_record_prefix(plan->rec_init.as<uint32_t>(), plan->rec_words, index,
                                       plan->prefix_out.as<uint16_t>(), nullptr));
    CUDA_TRY(cudaMemcpy(prefix, plan->prefix_out.p, sizeof(uint16_t) * plan->depth, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" void emp_bt_plan_destroy(emp_bt_plan plan)
{
    if (plan) {
        cudaSetDevice(plan->device);
        delete plan;
    }
}

namespace {

emp_status count_one_plan(const emp_puzzle* puzzles, uint32_t count, const emp_bt_config* config,
                          emp_bt_result* results)
{
    emp_bt_plan plan = nullptr;
    emp_status s = emp_bt_plan_create(puzzles, count, config, &plan);
    if (s != EMP_OK) return s;
    std::unique_ptr<emp_bt_plan_t> guard(plan);
    if (config && config->sample_stride) {
        const uint64_t first = config->sample_first, stride = config->sample_stride;
        const uint64_t n = first < plan->n_all ? (plan->n_all - first + stride - 1) / stride : 0;
        s = emp_bt_plan_select(plan, first, stride, n);
        if (s != EMP_OK) return s;
    }
    s = emp_bt_plan_run(plan, nullptr);
    if (s != EMP_OK) return s;
    return emp_bt_plan_results(plan, results);
}

}  // namespace

extern "C" emp_status emp_bt_count_batch(const emp_puzzle* puzzles, uint32_t count, const emp_bt_config* config,
                                         emp_bt_result* results)
{
    emp::clear_error();
    if (!puzzles || !count || !results) return fail(EMP_ERR_INVALID, "emp_bt_count_batch: no puzzle");
    const auto t0 = std::chrono::steady_clock::now();
    // Puzzles with big trees run one plan each (tables staged in shared memory);
    // many small puzzles share one launch (tables read from global memory).
    bool separate = count <= 64 && (!config || config->table_placement != 1);
    for (uint32_t i = 0; i < count && separate; ++i) separate = puzzles[i] && puzzles[i]->model.n >= 36;
    emp_status s = EMP_OK;
    if (separate && count > 1) {
        for (uint32_t i = 0; i < count && s == EMP_OK; ++i) s = count_one_plan(&puzzles[i], 1, config, &results[i]);
    } else {
        s = count_one_plan(puzzles, count, config, results);
    }
    if (s != EMP_OK) return s;
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    bool incomplete = false, lost = false;
    for (uint32_t i = 0; i < count; ++i) {
        results[i].total_ms = ms;
        incomplete |= results[i].status == EMP_INCOMPLETE;
        lost |= results[i].status == EMP_FIRST_LOST;
    }
    if (incomplete) return EMP_INCOMPLETE;
    if (lost) return fail(EMP_FIRST_LOST, "a first-solution record was not written: its lock wait ran out");
    return EMP_OK;
}

extern "C" emp_status emp_bt_count(emp_puzzle puzzle, const emp_bt_config* config, emp_bt_result* result)
{
    return emp_bt_count_batch(&puzzle, 1, config, result);
}

extern "C" emp_status emp_bt_resume(emp_puzzle puzzle, const uint16_t* situation, uint32_t placed,
                                    const emp_bt_config* config, emp_bt_result* result)
{
    emp::clear_error();
    if (!puzzle || !result || (placed && !situation)) return fail(EMP_ERR_INVALID, "emp_bt_resume: null argument");
    if (placed <= 1) return emp_bt_count(puzzle, config, result);  // the search starts at level 0 as usual
    emp_bt_config cfg{};
    cfg.device = -1;
    if (config) cfg = *config;
    cfg.sample_stride = 0;
    cfg.split_subtrees = 0;
    const ResumeSpec spec{situation, placed};
    emp_bt_plan plan = nullptr;
    emp_status s = create_plan(&puzzle, 1, &cfg, false, &plan, &spec);
    if (s != EMP_OK) return s;
    std::unique_ptr<emp_bt_plan_t> guard(plan);
    s = emp_bt_plan_run(plan, nullptr);
    if (s != EMP_OK) return s;
    s = emp_bt_plan_results(plan, result);
    if (s != EMP_OK) return s;
    if (result->status == EMP_INCOMPLETE) return EMP_INCOMPLETE;
    if (result->status == EMP_FIRST_LOST)
        return fail(EMP_FIRST_LOST, "a first-solution record was not written: its lock wait ran out");
    return EMP_OK;
}

namespace {

emp_status solutions_impl(emp_puzzle puzzle, const emp_bt_config* config, const ResumeSpec* resume,
                          emp_bt_solution* out, uint64_t capacity, uint64_t* found, emp_bt_result* result)
{
    emp::clear_error();
    if (!puzzle || !found || (capacity && !out)) return fail(EMP_ERR_INVALID, "emp_bt_solutions: null argument");
    emp_bt_config cfg{};
    cfg.device = -1;
    if (config) cfg = *config;
    cfg.keep_subtree_counts = 1;
    cfg.stop_at_first = 0;
    cfg.stop_at_any = 0;
    cfg.sample_stride = 0;
    cfg.use_graph = 0;
    cfg.split_subtrees = 0;
    emp_bt_plan plan = nullptr;
    emp_status s = create_plan(&puzzle, 1, &cfg, true, &plan, resume);
    if (s != EMP_OK) return s;
    std::unique_ptr<emp_bt_plan_t> guard(plan);
    plan->budget = 0;  // never hand work back: each subtree is searched in order by one thread
    CUDA_TRY(plan->sol_count.alloc(sizeof(unsigned long long)));
    // Threads record solutions in arrival order; ranking them needs all of them.  When
    // more solutions exist than the caller holds, the (deterministic) search runs
    // again with room for every one, and the first `capacity` by node index are kept.
    constexpr uint64_t kMaxRanked = 1ull << 20;
    uint64_t room = std::max<uint64_t>(capacity, 1);
    emp_bt_result res{};
    unsigned long long total = 0;
    for (int pass = 0; pass < 2; ++pass) {
        CUDA_TRY(plan->sol_buf.alloc(sizeof(emp::SolutionRecord) * room));
        CUDA_TRY(cudaMemset(plan->sol_count.p, 0, sizeof(unsigned long long)));
        plan->sol_capacity = room;
        s = emp_bt_plan_run(plan, nullptr);
        if (s != EMP_OK) return s;
        s = emp_bt_plan_results(plan, &res);
        if (s != EMP_OK) return s;
        if (result) *result = res;
        if (res.status == EMP_INCOMPLETE)
            return fail(EMP_INCOMPLETE, "emp_bt_solutions: the search stopped before the end");
        CUDA_TRY(cudaMemcpy(&total, plan->sol_count.p, sizeof(total), cudaMemcpyDeviceToHost));
        if (total <= room) break;
        if (total > kMaxRanked)
            return fail(EMP_ERR_UNSUPPORTED, "emp_bt_solutions: more than 2^20 solutions to rank; count them with "
                                             "emp_bt_count and dump them with a capacity of at least the count");
        room = total;
    }
    *found = total;
    const uint64_t nall = std::min<uint64_t>(total, room);  // every solution when a second pass ran
    const uint64_t nsol = std::min<uint64_t>(total, capacity);
    if (!nsol) return EMP_OK;
    // level arrays: device pointer table (index L = prefixes of length L)
    const uint32_t depth = plan->depth;
    std::vector<const uint16_t*> ptrs(depth + 1, nullptr);
    std::vector<uint64_t> counts(depth + 1, 0);
    for (uint32_t L = 1; L <= depth && L < plan->level_prefixes.size(); ++L) {
        ptrs[L] = plan->level_prefixes[L].as<uint16_t>();
        counts[L] = plan->level_counts[L];
    }
    DeviceBuffer d_ptrs, d_counts, d_idx;
    CUDA_TRY(d_ptrs.alloc(sizeof(void*) * ptrs.size()));
    CUDA_TRY(d_counts.alloc(sizeof(uint64_t) * counts.size()));
    CUDA_TRY(d_idx.alloc(sizeof(unsigned long long) * nall));
    CUDA_TRY(cudaMemcpy(d_ptrs.p, ptrs.data(), sizeof(void*) * ptrs.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_counts.p, counts.data(), sizeof(uint64_t) * counts.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(emp::launch_solution_index(plan->sol_buf.as<emp::SolutionRecord>(), nall,
                                        reinterpret_cast<const uint16_t* const*>(d_ptrs.p), d_counts.as<uint64_t>(),
                                        depth, plan->item_nodes.as<unsigned long long>(),
                                        d_idx.as<unsigned long long>(), nullptr));
    std::vector<emp::SolutionRecord> recs(nall);
    std::vector<unsigned long long> idx(nall);
    CUDA_TRY(cudaMemcpy(recs.data(), plan->sol_buf.p, sizeof(emp::SolutionRecord) * nall, cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(idx.data(), d_idx.p, sizeof(unsigned long long) * nall, cudaMemcpyDeviceToHost));
    std::vector<uint64_t> order(nall);
    for (uint64_t i = 0; i < nall; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return idx[a] < idx[b]; });
    const emp::PuzzleModel& m = puzzle->model;
    for (uint64_t k = 0; k < nsol; ++k) {
        const emp::SolutionRecord& r = recs[order[k]];
        emp_bt_solution& o = out[k];
        o.node_index = idx[order[k]];
        for (uint32_t pos = 0; pos < 256; ++pos) o.board[pos] = 0xFFFFFFFFu;
        for (uint32_t l = 0; l < m.n; ++l) {
            const emp::LevelPlan& lp = puzzle->plan[l];
            const uint32_t t = r.t[l];
            o.board[lp.position] = (m.members[lp.kind][t >> 2] << 2) | (t & 3u);
        }
    }
    return EMP_OK;
}

}  // namespace

extern "C" emp_status emp_bt_solutions(emp_puzzle puzzle, const emp_bt_config* config, emp_bt_solution* out,
                                       uint64_t capacity, uint64_t* found, emp_bt_result* result)
{
    return solutions_impl(puzzle, config, nullptr, out, capacity, found, result);
}

extern "C" emp_status emp_bt_resume_solutions(emp_puzzle puzzle, const uint16_t* situation, uint32_t placed,
                                              const emp_bt_config* config, emp_bt_solution* out, uint64_t capacity,
                                              uint64_t* found, emp_bt_result* result)
{
    if (placed <= 1) return solutions_impl(puzzle, config, nullptr, out, capacity, found, result);
    if (!situation) return fail(EMP_ERR_INVALID, "emp_bt_resume_solutions: null situation");
    const ResumeSpec spec{situation, placed};
    return solutions_impl(puzzle, config, &spec, out, capacity, found, result);
}
