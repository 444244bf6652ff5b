// C ABI of the learned value ordering: the scoring network, its features, its
// training on the solver's traces (emp_mlp_*).
#include "emp_b200.h"
#include "emp_bt.h"
#include "emp_common.h"
#include "emp_mlp.h"
#include "emp_model.h"
#include "emp_plan.h"

#include <cub/device/device_radix_sort.cuh>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <numeric>
#include <vector>

using emp::fail;

struct emp_mlp_t {
    int device = 0;
    DeviceBuffer params, w1b, w2b, m1, m2;
    uint32_t adam_steps = 0;
    emp::MlpDevice dev() const
    {
        emp::MlpDevice d;
        d.params = params.as<float>();
        d.w1_bf16 = w1b.as<uint16_t>();
        d.w2_bf16 = w2b.as<uint16_t>();
        return d;
    }
};

namespace {

// training workspace for up to `rows` rows
struct Work {
    DeviceBuffer h1, h2, s, ds, dh2, dh1, grad, loss;
    emp::MlpWork w;
    cudaError_t alloc(uint64_t rows)
    {
        const uint64_t H = emp::kMlpHidden;
        cudaError_t e;
        if ((e = h1.alloc(4 * rows * H)) || (e = h2.alloc(4 * rows * H)) || (e = s.alloc(4 * rows)) ||
            (e = ds.alloc(4 * rows)) || (e = dh2.alloc(4 * rows * H)) || (e = dh1.alloc(4 * rows * H)) ||
            (e = grad.alloc(4ull * emp::kMlpParams)) || (e = loss.alloc(2 * sizeof(double))))
            return e;
        w.rows = rows;
        w.h1 = h1.as<float>();
        w.h2 = h2.as<float>();
        w.s = s.as<float>();
        w.ds = ds.as<float>();
        w.dh2 = dh2.as<float>();
        w.dh1 = dh1.as<float>();
        w.grad = grad.as<float>();
        w.loss = loss.as<double>();
        return cudaSuccess;
    }
};

uint64_t splitmix(uint64_t& s)
{
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// feature tables of several puzzles, concatenated on the device
struct FeatTables {
    DeviceBuffer tab, off;
    emp_status upload(const std::vector<emp_puzzle>& puzzles)
    {
        std::vector<uint32_t> all;
        std::vector<unsigned long long> offs;
        for (emp_puzzle p : puzzles) {
            offs.push_back(all.size());
            const std::vector<uint32_t> t = emp::build_feature_table(p->model, p->plan);
            all.insert(all.end(), t.begin(), t.end());
        }
        CUDA_TRY(tab.alloc(4 * all.size()));
        CUDA_TRY(off.alloc(8 * offs.size()));
        CUDA_TRY(cudaMemcpy(tab.p, all.data(), 4 * all.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(off.p, offs.data(), 8 * offs.size(), cudaMemcpyHostToDevice));
        return EMP_OK;
    }
};

emp_status use_device(int device)
{
    CUDA_TRY(cudaSetDevice(device));
    return EMP_OK;
}

// sort key of prefix i: its puzzle's place in the queue, then the score, highest first
__global__ void order_keys_kernel(const float* __restrict__ score, const uint32_t* __restrict__ prefix_puzzle,
                                  const uint32_t* __restrict__ rank, uint64_t n, unsigned long long* __restrict__ keys,
                                  uint32_t* __restrict__ vals)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t u = __float_as_uint(score[i]);
        u ^= (u >> 31) ? 0xFFFFFFFFu : 0x80000000u;  // increasing with the score
        keys[i] = (static_cast<unsigned long long>(rank[prefix_puzzle[i]]) << 32) | (~u);
        vals[i] = static_cast<uint32_t>(i);
    }
}

__global__ void gather_prefixes_kernel(const uint16_t* __restrict__ src, const uint32_t* __restrict__ src_puzzle,
                                       const uint32_t* __restrict__ perm, uint64_t n, uint32_t depth,
                                       uint16_t* __restrict__ dst, uint32_t* __restrict__ dst_puzzle)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n * depth;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t r = i / depth, l = i % depth;
        const uint64_t from = perm[r];
        dst[i] = src[from * depth + l];
        if (l == 0) dst_puzzle[r] = src_puzzle[from];
    }
}

uint32_t blocks_for(uint64_t n) { return static_cast<uint32_t>(std::min<uint64_t>((n + 255) / 256, 148ull * 16)); }

}  // namespace

extern "C" emp_status emp_mlp_create(uint64_t seed, int32_t device, emp_mlp* out)
{
    emp::clear_error();
    if (!out) return fail(EMP_ERR_INVALID, "emp_mlp_create: null output");
    *out = nullptr;
    std::unique_ptr<emp_mlp_t> m(new (std::nothrow) emp_mlp_t());
    if (!m) return fail(EMP_ERR_NOMEM, "emp_mlp_create: out of host memory");
    EMP_TRY(emp::select_device(device, &m->device));
    std::vector<float> p(emp::kMlpParams, 0.f);
    uint64_t s = seed;
    auto fill = [&](uint32_t off, uint32_t count, uint32_t fan_in) {
        const float scale = 1.0f / std::sqrt(static_cast<float>(fan_in));
        for (uint32_t i = 0; i < count; ++i) {
            const double u = (splitmix(s) >> 11) * (1.0 / 9007199254740992.0);  // [0, 1)
            p[off + i] = static_cast<float>((2.0 * u - 1.0) * scale);
        }
    };
    fill(emp::kOffW1, emp::kMlpHidden * emp::kMlpIn, emp::kMlpIn);
    fill(emp::kOffW2, emp::kMlpHidden * emp::kMlpHidden, emp::kMlpHidden);
    fill(emp::kOffW3, emp::kMlpHidden, emp::kMlpHidden);
    CUDA_TRY(m->params.alloc(4ull * emp::kMlpParams));
    CUDA_TRY(m->w1b.alloc(2ull * emp::kMlpHidden * emp::kMlpIn));
    CUDA_TRY(m->w2b.alloc(2ull * emp::kMlpHidden * emp::kMlpHidden));
    CUDA_TRY(m->m1.alloc(4ull * emp::kMlpParams));
    CUDA_TRY(m->m2.alloc(4ull * emp::kMlpParams));
    CUDA_TRY(cudaMemcpy(m->params.p, p.data(), 4ull * emp::kMlpParams, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemset(m->m1.p, 0, m->m1.bytes));
    CUDA_TRY(cudaMemset(m->m2.p, 0, m->m2.bytes));
    CUDA_TRY(emp::launch_mlp_pack_bf16(m->dev(), nullptr));
    CUDA_TRY(cudaDeviceSynchronize());
    *out = m.release();
    return EMP_OK;
}

extern "C" void emp_mlp_destroy(emp_mlp model)
{
    if (model) {
        cudaSetDevice(model->device);
        delete model;
    }
}

extern "C" emp_status emp_mlp_get_params(emp_mlp model, float* params)
{
    emp::clear_error();
    if (!model || !params) return fail(EMP_ERR_INVALID, "emp_mlp_get_params: null argument");
    EMP_TRY(use_device(model->device));
    CUDA_TRY(cudaMemcpy(params, model->params.p, 4ull * emp::kMlpParams, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" emp_status emp_mlp_set_params(emp_mlp model, const float* params)
{
    emp::clear_error();
    if (!model || !params) return fail(EMP_ERR_INVALID, "emp_mlp_set_params: null argument");
    EMP_TRY(use_device(model->device));
    CUDA_TRY(cudaMemcpy(model->params.p, params, 4ull * emp::kMlpParams, cudaMemcpyHostToDevice));
    CUDA_TRY(emp::launch_mlp_pack_bf16(model->dev(), nullptr));
    CUDA_TRY(cudaDeviceSynchronize());
    return EMP_OK;
}

extern "C" emp_status emp_mlp_features(emp_puzzle puzzle, const uint16_t* prefixes, uint32_t stride,
                                       const uint16_t* lens, const uint16_t* cands, uint64_t n, float* out)
{
    emp::clear_error();
    if (!puzzle || !lens || !cands || !out || (!prefixes && stride)) return fail(EMP_ERR_INVALID, "emp_mlp_features: null argument");
    int dev = 0;
    EMP_TRY(emp::select_device(-1, &dev));
    const emp::PuzzleModel& m = puzzle->model;
    std::vector<emp::FeatItem> items(n);
    std::vector<uint16_t> pre(std::max<uint64_t>(n * stride, 1), 0);
    if (n * stride) std::memcpy(pre.data(), prefixes, 2 * n * stride);
    for (uint64_t i = 0; i < n; ++i) {
        if (lens[i] >= m.n || lens[i] > stride) return fail(EMP_ERR_INVALID, "emp_mlp_features: prefix length out of range");
        if (cands[i] >= 4 * m.nb_kind(puzzle->plan[lens[i]].kind))
            return fail(EMP_ERR_INVALID, "emp_mlp_features: candidate out of range");
        for (uint32_t l = 0; l < lens[i]; ++l)
            if (pre[i * stride + l] >= 4 * m.nb_kind(puzzle->plan[l].kind))
                return fail(EMP_ERR_INVALID, "emp_mlp_features: prefix transition out of range");
        items[i] = emp::FeatItem{i * stride, 0u, lens[i], cands[i]};
    }
    FeatTables ft;
    EMP_TRY(ft.upload({puzzle}));
    DeviceBuffer d_items, d_pre, d_out;
    CUDA_TRY(d_items.alloc(sizeof(emp::FeatItem) * std::max<uint64_t>(n, 1)));
    CUDA_TRY(d_pre.alloc(2 * pre.size()));
    CUDA_TRY(d_out.alloc(4ull * emp::kMlpIn * std::max<uint64_t>(n, 1)));
    CUDA_TRY(cudaMemcpy(d_items.p, items.data(), sizeof(emp::FeatItem) * n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_pre.p, pre.data(), 2 * pre.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(emp::launch_features(ft.tab.as<uint32_t>(), ft.off.as<unsigned long long>(), d_items.as<emp::FeatItem>(),
                                  n, d_pre.as<uint16_t>(), nullptr, d_out.as<float>(), nullptr));
    CUDA_TRY(cudaMemcpy(out, d_out.p, 4ull * emp::kMlpIn * n, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" emp_status emp_mlp_score(emp_mlp model, const float* features, uint64_t n, float* scores)
{
    emp::clear_error();
    if (!model || (n && (!features || !scores))) return fail(EMP_ERR_INVALID, "emp_mlp_score: null argument");
    if (!n) return EMP_OK;
    EMP_TRY(use_device(model->device));
    DeviceBuffer x32, x16, s, err;
    CUDA_TRY(x32.alloc(4ull * emp::kMlpIn * n));
    CUDA_TRY(x16.alloc(2ull * emp::kMlpIn * n));
    CUDA_TRY(s.alloc(4ull * n));
    CUDA_TRY(err.alloc(sizeof(int)));
    CUDA_TRY(cudaMemset(err.p, 0, sizeof(int)));
    CUDA_TRY(cudaMemcpy(x32.p, features, 4ull * emp::kMlpIn * n, cudaMemcpyHostToDevice));
    CUDA_TRY(emp::launch_f32_to_bf16(x32.as<float>(), x16.as<uint16_t>(), emp::kMlpIn * n, nullptr));
    CUDA_TRY(emp::launch_mlp_infer_tc(model->dev(), x16.p, n, s.as<float>(), err.as<int>(), nullptr));
    int e = 0;
    CUDA_TRY(cudaMemcpy(&e, err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (e) return fail(EMP_ERR_CUDA, "emp_mlp_score: a tensor-core wait ran out of time");
    CUDA_TRY(cudaMemcpy(scores, s.p, 4ull * n, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" emp_status emp_mlp_score_f32(emp_mlp model, const float* features, uint64_t n, float* scores)
{
    emp::clear_error();
    if (!model || (n && (!features || !scores))) return fail(EMP_ERR_INVALID, "emp_mlp_score_f32: null argument");
    if (!n) return EMP_OK;
    EMP_TRY(use_device(model->device));
    DeviceBuffer x;
    Work w;
    CUDA_TRY(x.alloc(4ull * emp::kMlpIn * n));
    CUDA_TRY(w.alloc(n));
    CUDA_TRY(cudaMemcpy(x.p, features, 4ull * emp::kMlpIn * n, cudaMemcpyHostToDevice));
    CUDA_TRY(emp::mlp_forward_f32(model->dev(), w.w, x.as<float>(), n, nullptr));
    CUDA_TRY(cudaMemcpy(scores, w.s.p, 4ull * n, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" emp_status emp_mlp_loss_grad(emp_mlp model, const float* features, const float* labels,
                                        const float* weights, uint64_t n, double* loss, float* grads)
{
    emp::clear_error();
    if (!model || !features || !labels || !weights || !loss || !grads || !n)
        return fail(EMP_ERR_INVALID, "emp_mlp_loss_grad: null argument");
    EMP_TRY(use_device(model->device));
    DeviceBuffer x, y, w8;
    Work w;
    CUDA_TRY(x.alloc(4ull * emp::kMlpIn * n));
    CUDA_TRY(y.alloc(4ull * n));
    CUDA_TRY(w8.alloc(4ull * n));
    CUDA_TRY(w.alloc(n));
    CUDA_TRY(cudaMemcpy(x.p, features, 4ull * emp::kMlpIn * n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(y.p, labels, 4ull * n, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(w8.p, weights, 4ull * n, cudaMemcpyHostToDevice));
    CUDA_TRY(emp::mlp_forward_f32(model->dev(), w.w, x.as<float>(), n, nullptr));
    CUDA_TRY(emp::mlp_loss_backward_f32(model->dev(), w.w, x.as<float>(), y.as<float>(), w8.as<float>(), n, nullptr));
    double l[2];
    CUDA_TRY(cudaMemcpy(l, w.loss.p, sizeof(l), cudaMemcpyDeviceToHost));
    *loss = l[1] > 0 ? l[0] / l[1] : 0.0;
    CUDA_TRY(cudaMemcpy(grads, w.grad.p, 4ull * emp::kMlpParams, cudaMemcpyDeviceToHost));
    return EMP_OK;
}

extern "C" emp_status emp_mlp_train(emp_mlp model, const emp_puzzle* puzzles, uint32_t count, const uint32_t* solutions,
                                    const emp_mlp_train_config* config, emp_mlp_train_report* report)
{
    emp::clear_error();
    if (!model || !puzzles || !count || !solutions) return fail(EMP_ERR_INVALID, "emp_mlp_train: null argument");
    const auto t0 = std::chrono::steady_clock::now();
    emp_mlp_train_config cfg{};
    if (config) cfg = *config;
    const uint32_t epochs = cfg.epochs ? cfg.epochs : 30;
    const uint32_t batch = cfg.batch ? cfg.batch : 2048;
    const float lr = cfg.learning_rate > 0 ? cfg.learning_rate : 1e-3f;
    EMP_TRY(use_device(model->device));
    // solution paths: transition per level, from the solution boards
    std::vector<emp_puzzle> used;
    std::vector<std::vector<uint16_t>> paths;
    for (uint32_t i = 0; i < count; ++i) {
        const emp_puzzle pz = puzzles[i];
        if (!pz) return fail(EMP_ERR_INVALID, "emp_mlp_train: null puzzle");
        const uint32_t* board = solutions + 256ull * i;
        std::vector<uint16_t> path(pz->model.n);
        bool ok = true;
        for (uint32_t l = 0; l < pz->model.n && ok; ++l) {
            const uint32_t v = board[pz->plan[l].position];
            if (v == 0xFFFFFFFFu || (v >> 2) >= pz->model.n) {
                ok = false;
                break;
            }
            const uint32_t piece = v >> 2;
            if (pz->model.kind[piece] != pz->plan[l].kind) return fail(EMP_ERR_INVALID, "emp_mlp_train: board does not fit the puzzle");
            path[l] = static_cast<uint16_t>((pz->model.kind_index[piece] << 2) | (v & 3u));
        }
        if (!ok) continue;
        used.push_back(pz);
        paths.push_back(std::move(path));
    }
    if (used.empty()) return fail(EMP_ERR_INVALID, "emp_mlp_train: no puzzle with a solution");
    const uint32_t P = static_cast<uint32_t>(used.size());
    // tables for the sibling enumeration (the search's own candidate step)
    std::vector<uint32_t> blob;
    std::vector<uint64_t> offs;
    uint32_t max_n = 0;
    for (emp_puzzle p : used) {
        offs.push_back(blob.size());
        blob.insert(blob.end(), p->tables.blob.begin(), p->tables.blob.end());
        max_n = std::max(max_n, p->model.n);
    }
    DeviceBuffer d_tab, d_off, d_parents, d_ppz, d_counts, d_offsets, d_bsums, d_grand, d_children, d_cpz, d_lv;
    CUDA_TRY(d_tab.alloc(4 * blob.size()));
    CUDA_TRY(d_off.alloc(8 * offs.size()));
    CUDA_TRY(cudaMemcpy(d_tab.p, blob.data(), 4 * blob.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_off.p, offs.data(), 8 * offs.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(d_lv.alloc(16ull * P));
    CUDA_TRY(d_grand.alloc(8));
    emp::BtLaunch L;
    L.tables = d_tab.as<uint32_t>();
    L.puzzle_offset = d_off.as<uint64_t>();
    // samples: prefix store + items + labels
    std::vector<uint16_t> store;
    std::vector<emp::FeatItem> items;
    std::vector<float> labels;
    // levels past 63 are left out: the candidate step replays prefixes of at most 64 levels
    const uint32_t level_limit = cfg.max_level ? std::min<uint32_t>(cfg.max_level, 64u) : 64u;
    for (uint32_t l = 1; l + 1 < max_n && l < level_limit; ++l) {
        std::vector<uint16_t> parents;
        std::vector<uint32_t> ppz;
        for (uint32_t i = 0; i < P; ++i)
            if (used[i]->model.n > l + 1) {
                parents.insert(parents.end(), paths[i].begin(), paths[i].begin() + l);
                ppz.push_back(i);
            }
        const uint64_t np = ppz.size();
        if (!np) continue;
        CUDA_TRY(d_parents.alloc(2 * parents.size()));
        CUDA_TRY(d_ppz.alloc(4 * np));
        CUDA_TRY(d_counts.alloc(4 * np));
        CUDA_TRY(d_offsets.alloc(8 * np));
        CUDA_TRY(d_bsums.alloc(8 * emp::scan_block_sum_words(np)));
        CUDA_TRY(cudaMemcpy(d_parents.p, parents.data(), 2 * parents.size(), cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(d_ppz.p, ppz.data(), 4 * np, cudaMemcpyHostToDevice));
        unsigned long long* lv = d_lv.as<unsigned long long>();
        CUDA_TRY(emp::launch_expand(L, d_parents.as<uint16_t>(), d_ppz.as<uint32_t>(), np, l, d_counts.as<uint32_t>(),
                                    nullptr, nullptr, nullptr, lv, lv + P, 0, nullptr));
        CUDA_TRY(emp::launch_scan(d_counts.as<uint32_t>(), np, d_offsets.as<uint64_t>(), d_bsums.as<uint64_t>(),
                                  d_grand.as<uint64_t>(), nullptr));
        uint64_t total = 0;
        CUDA_TRY(cudaMemcpy(&total, d_grand.p, 8, cudaMemcpyDeviceToHost));
        if (!total) continue;
        CUDA_TRY(d_children.alloc(2 * total * (l + 1)));
        CUDA_TRY(d_cpz.alloc(4 * total));
        CUDA_TRY(emp::launch_expand(L, d_parents.as<uint16_t>(), d_ppz.as<uint32_t>(), np, l, d_counts.as<uint32_t>(),
                                    d_offsets.as<uint64_t>(), d_children.as<uint16_t>(), d_cpz.as<uint32_t>(), lv,
                                    lv + P, 1, nullptr));
        std::vector<uint16_t> ch(total * (l + 1));
        std::vector<uint32_t> cpz(total);
        CUDA_TRY(cudaMemcpy(ch.data(), d_children.p, 2 * ch.size(), cudaMemcpyDeviceToHost));
        CUDA_TRY(cudaMemcpy(cpz.data(), d_cpz.p, 4 * total, cudaMemcpyDeviceToHost));
        for (uint64_t c = 0; c < total; ++c) {
            const uint32_t pz = cpz[c];
            const uint16_t t = ch[c * (l + 1) + l];
            items.push_back(emp::FeatItem{store.size(), pz, static_cast<uint16_t>(l), t});
            store.insert(store.end(), ch.begin() + c * (l + 1), ch.begin() + c * (l + 1) + l);
            labels.push_back(t == paths[pz][l] ? 1.f : 0.f);
        }
    }
    const uint64_t N = items.size();
    if (!N) return fail(EMP_ERR_INVALID, "emp_mlp_train: no training sample");
    const uint64_t pos = static_cast<uint64_t>(std::count(labels.begin(), labels.end(), 1.f));
    const float wpos = pos ? static_cast<float>(N - pos) / static_cast<float>(pos) : 1.f;
    std::vector<float> weights(N);
    for (uint64_t i = 0; i < N; ++i) weights[i] = labels[i] > 0.5f ? wpos : 1.f;
    // features of every sample (f32, on the device)
    FeatTables ft;
    EMP_TRY(ft.upload(used));
    DeviceBuffer d_store, d_items, d_x, d_y, d_w;
    CUDA_TRY(d_store.alloc(2 * std::max<size_t>(store.size(), 1)));
    CUDA_TRY(d_items.alloc(sizeof(emp::FeatItem) * N));
    CUDA_TRY(d_x.alloc(4ull * emp::kMlpIn * N));
    CUDA_TRY(d_y.alloc(4 * N));
    CUDA_TRY(d_w.alloc(4 * N));
    if (!store.empty()) CUDA_TRY(cudaMemcpy(d_store.p, store.data(), 2 * store.size(), cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_items.p, items.data(), sizeof(emp::FeatItem) * N, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_y.p, labels.data(), 4 * N, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(d_w.p, weights.data(), 4 * N, cudaMemcpyHostToDevice));
    CUDA_TRY(emp::launch_features(ft.tab.as<uint32_t>(), ft.off.as<unsigned long long>(), d_items.as<emp::FeatItem>(),
                                  N, d_store.as<uint16_t>(), nullptr, d_x.as<float>(), nullptr));
    // minibatch Adam
    Work w;
    const uint64_t B = std::min<uint64_t>(batch, N);
    CUDA_TRY(w.alloc(B));
    DeviceBuffer d_idx, d_xb, d_yb, d_wb;
    CUDA_TRY(d_idx.alloc(4 * B));
    CUDA_TRY(d_xb.alloc(4ull * emp::kMlpIn * B));
    CUDA_TRY(d_yb.alloc(4 * B));
    CUDA_TRY(d_wb.alloc(4 * B));
    std::vector<uint32_t> order(N);
    std::iota(order.begin(), order.end(), 0u);
    uint64_t rng = cfg.seed ? cfg.seed : 1;
    double first_loss = 0, last_loss = 0;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        for (uint64_t i = N - 1; i > 0; --i) std::swap(order[i], order[splitmix(rng) % (i + 1)]);
        double ep_loss = 0, ep_w = 0;
        for (uint64_t b0 = 0; b0 < N; b0 += B) {
            const uint64_t nb = std::min<uint64_t>(B, N - b0);
            CUDA_TRY(cudaMemcpy(d_idx.p, order.data() + b0, 4 * nb, cudaMemcpyHostToDevice));
            CUDA_TRY(emp::launch_gather_rows(d_x.as<float>(), d_idx.as<uint32_t>(), nb, emp::kMlpIn, d_xb.as<float>(),
                                             d_y.as<float>(), d_w.as<float>(), d_yb.as<float>(), d_wb.as<float>(),
                                             nullptr));
            CUDA_TRY(emp::mlp_forward_f32(model->dev(), w.w, d_xb.as<float>(), nb, nullptr));
            CUDA_TRY(emp::mlp_loss_backward_f32(model->dev(), w.w, d_xb.as<float>(), d_yb.as<float>(),
                                                d_wb.as<float>(), nb, nullptr));
            CUDA_TRY(emp::mlp_adam_step(model->dev(), w.w.grad, model->m1.as<float>(), model->m2.as<float>(), lr,
                                        ++model->adam_steps, nullptr));
            double l[2];
            CUDA_TRY(cudaMemcpy(l, w.loss.p, sizeof(l), cudaMemcpyDeviceToHost));
            ep_loss += l[0];
            ep_w += l[1];
        }
        const double mean = ep_w > 0 ? ep_loss / ep_w : 0.0;
        if (ep == 0) first_loss = mean;
        last_loss = mean;
    }
    CUDA_TRY(emp::launch_mlp_pack_bf16(model->dev(), nullptr));
    CUDA_TRY(cudaDeviceSynchronize());
    if (report) {
        std::memset(report, 0, sizeof(*report));
        report->samples = N;
        report->positives = pos;
        report->puzzles = P;
        report->epochs = epochs;
        report->first_loss = first_loss;
        report->last_loss = last_loss;
        report->train_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    }
    return EMP_OK;
}

extern "C" emp_status emp_bt_plan_order(emp_bt_plan plan, emp_mlp model)
{
    emp::clear_error();
    if (!plan || !model) return fail(EMP_ERR_INVALID, "emp_bt_plan_order: null argument");
    if (plan->cfg.stop_at_first)
        return fail(EMP_ERR_INVALID, "emp_bt_plan_order: stop_at_first needs the subtrees in search order");
    if (plan->device != model->device) return fail(EMP_ERR_INVALID, "emp_bt_plan_order: plan and model on different devices");
    EMP_TRY(use_device(plan->device));
    const uint64_t N = plan->n_all;
    const uint32_t depth = plan->depth;
    if (N < 2 || depth < 2) return EMP_OK;  // nothing to reorder
    if (N > 0xFFFFFFFFull) return fail(EMP_ERR_UNSUPPORTED, "emp_bt_plan_order: more than 2^32 subtrees");
    const uint32_t P = static_cast<uint32_t>(plan->puzzles.size());
    // the expansion queues puzzles by piece count (stable); ordering keeps that
    std::vector<uint32_t> ids(P), rank(P);
    std::iota(ids.begin(), ids.end(), 0u);
    std::stable_sort(ids.begin(), ids.end(),
                     [&](uint32_t a, uint32_t b) { return plan->puzzles[a]->model.n < plan->puzzles[b]->model.n; });
    for (uint32_t i = 0; i < P; ++i) rank[ids[i]] = i;
    FeatTables ft;
    EMP_TRY(ft.upload(plan->puzzles));
    const uint32_t per = depth - 1;
    const uint64_t chunk = std::max<uint64_t>(1, (1ull << 21) / per);  // 2M feature rows (2 GB of bf16) at most
    DeviceBuffer d_rank, d_score, d_items, d_x, d_s, d_err;
    CUDA_TRY(d_rank.alloc(4ull * P));
    CUDA_TRY(cudaMemcpy(d_rank.p, rank.data(), 4ull * P, cudaMemcpyHostToDevice));
    CUDA_TRY(d_score.alloc(4 * N));
    const uint64_t rows = std::min<uint64_t>(chunk, N) * per;
    CUDA_TRY(d_items.alloc(sizeof(emp::FeatItem) * rows));
    CUDA_TRY(d_x.alloc(2ull * emp::kMlpIn * rows));
    CUDA_TRY(d_s.alloc(4 * rows));
    CUDA_TRY(d_err.alloc(sizeof(int)));
    CUDA_TRY(cudaMemset(d_err.p, 0, sizeof(int)));
    const uint32_t* pdepth = plan->adaptive ? plan->puzzle_depth_dev.as<uint32_t>() : nullptr;
    for (uint64_t c0 = 0; c0 < N; c0 += chunk) {
        const uint64_t cnt = std::min<uint64_t>(chunk, N - c0);
        CUDA_TRY(emp::launch_order_items(plan->prefixes.as<uint16_t>(), plan->prefix_puzzle.as<uint32_t>(), pdepth,
                                         depth, c0, cnt, d_items.as<emp::FeatItem>(), nullptr));
        CUDA_TRY(emp::launch_features(ft.tab.as<uint32_t>(), ft.off.as<unsigned long long>(),
                                      d_items.as<emp::FeatItem>(), cnt * per, plan->prefixes.as<uint16_t>(), d_x.p,
                                      nullptr, nullptr));
        CUDA_TRY(emp::launch_mlp_infer_tc(model->dev(), d_x.p, cnt * per, d_s.as<float>(), d_err.as<int>(), nullptr));
        CUDA_TRY(emp::launch_order_accumulate(d_s.as<float>(), d_items.as<emp::FeatItem>(), cnt, depth,
                                              d_score.as<float>() + c0, nullptr));
    }
    int err = 0;
    CUDA_TRY(cudaMemcpy(&err, d_err.p, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) return fail(EMP_ERR_CUDA, "emp_bt_plan_order: a tensor-core wait ran out of time");
    // stable radix sort of (puzzle rank, score) keys carrying the prefix index
    DeviceBuffer k_in, k_out, v_in, v_out, temp;
    CUDA_TRY(k_in.alloc(8 * N));
    CUDA_TRY(k_out.alloc(8 * N));
    CUDA_TRY(v_in.alloc(4 * N));
    CUDA_TRY(v_out.alloc(4 * N));
    order_keys_kernel<<<blocks_for(N), 256>>>(d_score.as<float>(), plan->prefix_puzzle.as<uint32_t>(),
                                              d_rank.as<uint32_t>(), N, k_in.as<unsigned long long>(), v_in.as<uint32_t>());
    CUDA_TRY(cudaGetLastError());
    size_t temp_bytes = 0;
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, k_in.as<unsigned long long>(),
                                             k_out.as<unsigned long long>(), v_in.as<uint32_t>(), v_out.as<uint32_t>(),
                                             static_cast<int>(N)));
    CUDA_TRY(temp.alloc(std::max<size_t>(temp_bytes, 1)));
    CUDA_TRY(cub::DeviceRadixSort::SortPairs(temp.p, temp_bytes, k_in.as<unsigned long long>(),
                                             k_out.as<unsigned long long>(), v_in.as<uint32_t>(), v_out.as<uint32_t>(),
                                             static_cast<int>(N)));
    DeviceBuffer new_prefixes, new_puzzle;
    CUDA_TRY(new_prefixes.alloc(2 * N * depth));
    CUDA_TRY(new_puzzle.alloc(4 * N));
    gather_prefixes_kernel<<<blocks_for(N * depth), 256>>>(plan->prefixes.as<uint16_t>(),
                                                           plan->prefix_puzzle.as<uint32_t>(), v_out.as<uint32_t>(), N,
                                                           depth, new_prefixes.as<uint16_t>(), new_puzzle.as<uint32_t>());
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaDeviceSynchronize());
    plan->prefixes = std::move(new_prefixes);
    plan->prefix_puzzle = std::move(new_puzzle);
    plan->drop_graph();
    EMP_TRY(plan_build_initial(*plan, 0, 1, N));
    plan->sampled = false;
    return EMP_OK;
}
