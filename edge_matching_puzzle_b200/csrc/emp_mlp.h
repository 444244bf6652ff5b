// Learned value ordering (emp_mlp.cu): candidate features, the scoring network's
// inference on the tensor cores and its training kernels.
//
// The network scores one candidate placement (position, piece, rotation) given
// the placements before it:  s = w3 . relu(W2 relu(W1 x + b1) + b2) + b3  with x
// the 512 features below, hidden widths 256, and sigma(s) read as the chance
// that the placement lies on a solution path.
#pragma once

#include "emp_model.h"

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace emp {

constexpr uint32_t kMlpIn = 512;
constexpr uint32_t kMlpHidden = 256;
// parameter order: W1 [256][512] (row = hidden unit), b1[256], W2 [256][256], b2[256], w3[256], b3
constexpr uint32_t kMlpParams = kMlpHidden * kMlpIn + kMlpHidden + kMlpHidden * kMlpHidden + kMlpHidden + kMlpHidden + 1;
constexpr uint32_t kOffW1 = 0;
constexpr uint32_t kOffB1 = kOffW1 + kMlpHidden * kMlpIn;
constexpr uint32_t kOffW2 = kOffB1 + kMlpHidden;
constexpr uint32_t kOffB2 = kOffW2 + kMlpHidden * kMlpHidden;
constexpr uint32_t kOffW3 = kOffB2 + kMlpHidden;
constexpr uint32_t kOffB3 = kOffW3 + kMlpHidden;

// Feature table of one puzzle (32-bit words), built on the host:
//   [0] n, [1] width, [2] height, [3] border colour id
//   [4, 36)    edge colour totals over all pieces, colour 0..31 (0 = frame)
//   [36, 39)   word offset of each kind's candidate entries
//   [40, 296)  per level: position | kind << 8 | x << 16 | y << 24
//   [296, 808) per level, two words: levels of the neighbours on sides N | E << 16 and
//              S | W << 16 (0xFFFF = outside the board)
//   [808, ...) per (kind, transition t): piece index << 20 | oriented colours N | E << 5 | S << 10 | W << 15
constexpr uint32_t kFtColours = 4, kFtKindOff = 36, kFtLevelA = 40, kFtLevelB = 296, kFtCand = 808;
std::vector<uint32_t> build_feature_table(const PuzzleModel& m, const std::vector<LevelPlan>& plan);

// One feature row: the candidate `t` placed at level `len` after the transitions
// prefixes[prefix_off .. prefix_off + len).
struct FeatItem {
    unsigned long long prefix_off;  // in uint16 units
    uint32_t puzzle;
    uint16_t len;
    uint16_t t;
};

// Feature rows (kMlpIn values each) as bf16 (inference) or f32 (training): one
// of out_bf16 / out_f32 is null.
cudaError_t launch_features(const uint32_t* ftab, const unsigned long long* ftab_off, const FeatItem* items,
                            uint64_t n, const uint16_t* prefixes, void* out_bf16, float* out_f32,
                            cudaStream_t stream);

// Device copy of the network: f32 master parameters and the bf16 operands of the
// tensor-core inference (W1 and W2 as stored, K-major).
struct MlpDevice {
    float* params = nullptr;        // kMlpParams
    uint16_t* w1_bf16 = nullptr;    // [256][512]
    uint16_t* w2_bf16 = nullptr;    // [256][256]
};
cudaError_t launch_mlp_pack_bf16(const MlpDevice& m, cudaStream_t stream);
cudaError_t launch_f32_to_bf16(const float* src, uint16_t* dst, uint64_t n, cudaStream_t stream);
// rows[i] = src[idx[i]] for rows of `cols` floats, and the per-row values y, w
cudaError_t launch_gather_rows(const float* src, const uint32_t* idx, uint64_t n, uint32_t cols, float* dst,
                               const float* y, const float* w, float* y_out, float* w_out, cudaStream_t stream);
// Ordering of prefixes: items (prefix i, level 1 + k) for k < depth - 1, and the sum
// of log sigmoid(score) over each prefix's levels below its own length.
cudaError_t launch_order_items(const uint16_t* prefixes, const uint32_t* prefix_puzzle, const uint32_t* puzzle_depth,
                               uint32_t depth, uint64_t first, uint64_t count, FeatItem* items, cudaStream_t stream);
cudaError_t launch_order_accumulate(const float* scores, const FeatItem* items, uint64_t count, uint32_t depth,
                                    float* prefix_score, cudaStream_t stream);

// Scores of n feature rows (bf16, row-major [n][512]) with the tensor cores
// (tcgen05, BF16 operands, FP32 accumulation in tensor memory).  err receives a
// nonzero code when a wait inside the kernel ran out of time.
cudaError_t launch_mlp_infer_tc(const MlpDevice& m, const void* x_bf16, uint64_t n, float* scores, int* err,
                                cudaStream_t stream);
size_t mlp_infer_smem_bytes();

// Training (f32, CUDA cores).  Workspace holds the activations of `rows` rows.
struct MlpWork {
    uint64_t rows = 0;
    float* h1 = nullptr;    // [rows][256] post-relu
    float* h2 = nullptr;    // [rows][256]
    float* s = nullptr;     // [rows]
    float* ds = nullptr;    // [rows]
    float* dh2 = nullptr;   // [rows][256]
    float* dh1 = nullptr;   // [rows][256]
    float* grad = nullptr;  // kMlpParams
    double* loss = nullptr; // [2]: weighted loss sum, weight sum
};
// Forward of rows x[n][512] (f32) into h1, h2, s.
cudaError_t mlp_forward_f32(const MlpDevice& m, const MlpWork& w, const float* x, uint64_t n, cudaStream_t stream);
// Weighted logistic loss and its gradient with respect to every parameter (grad,
// loss[0] = sum of w * loss, loss[1] = sum of w; grad is already divided by sum w).
cudaError_t mlp_loss_backward_f32(const MlpDevice& m, const MlpWork& w, const float* x, const float* y,
                                  const float* weight, uint64_t n, cudaStream_t stream);
// One Adam step on the master parameters.
cudaError_t mlp_adam_step(const MlpDevice& m, const float* grad, float* m1, float* m2, float lr, uint32_t step,
                          cudaStream_t stream);

}  // namespace emp
