// Learned value ordering: candidate features, tensor-core inference (tcgen05) and
// f32 training kernels of the scoring network (interface in emp_mlp.h).
#include "emp_mlp.h"

#include <cuda_bf16.h>

#include <algorithm>

namespace emp {

// ---------------------------------------------------------------------------
// feature table (host)

std::vector<uint32_t> build_feature_table(const PuzzleModel& m, const std::vector<LevelPlan>& plan)
{
    const uint32_t n = m.n;
    std::vector<uint32_t> t(kFtCand, 0);
    t[0] = n;
    t[1] = m.width;
    t[2] = m.height;
    t[3] = m.border_id;
    for (uint32_t p = 0; p < n; ++p)
        for (uint32_t s = 0; s < 4; ++s)
            if (m.colours[p][s] < 32) ++t[kFtColours + m.colours[p][s]];
    std::vector<uint32_t> level_of(n, 0);
    for (uint32_t l = 0; l < n; ++l) level_of[plan[l].position] = l;
    for (uint32_t l = 0; l < n; ++l) {
        const uint32_t pos = plan[l].position, x = pos % m.width, y = pos / m.width;
        t[kFtLevelA + l] = pos | (plan[l].kind << 8) | (std::min<uint32_t>(x, 255) << 16) |
                           (std::min<uint32_t>(y, 255) << 24);
        const uint32_t nn = y ? level_of[pos - m.width] : 0xFFFFu;
        const uint32_t ne = x + 1 < m.width ? level_of[pos + 1] : 0xFFFFu;
        const uint32_t ns = y + 1 < m.height ? level_of[pos + m.width] : 0xFFFFu;
        const uint32_t nw = x ? level_of[pos - 1] : 0xFFFFu;
        t[kFtLevelB + 2 * l] = nn | (ne << 16);
        t[kFtLevelB + 2 * l + 1] = ns | (nw << 16);
    }
    uint32_t off = kFtCand;
    for (uint32_t k = 0; k < 3; ++k) {
        t[kFtKindOff + k] = off;
        off += 4 * m.nb_kind(k);
    }
    t.resize(off, 0);
    for (uint32_t k = 0; k < 3; ++k)
        for (uint32_t e = 0; e < 4 * m.nb_kind(k); ++e) {
            const uint32_t p = m.members[k][e >> 2], o = e & 3u;
            uint32_t col = 0;
            for (uint32_t s = 0; s < 4; ++s) col |= (m.colour(p, s, o) & 31u) << (5 * s);
            t[t[kFtKindOff + k] + e] = (p << 20) | col;
        }
    while (t.size() % 4) t.push_back(0);  // tables concatenate 16-byte aligned
    return t;
}

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t side_colour(uint32_t cand, uint32_t s) { return (cand >> (5 * s)) & 31u; }

__device__ __forceinline__ uint32_t colour_edges(uint32_t cand, uint32_t c)
{
    return (side_colour(cand, 0) == c) + (side_colour(cand, 1) == c) + (side_colour(cand, 2) == c) +
           (side_colour(cand, 3) == c);
}

// ---------------------------------------------------------------------------
// features: one warp per row; the lanes clear the row and count the colours of
// the placed pieces, lane 0 sets the active entries
//
//   [0, 128)    colour of each side of the oriented candidate (4 x 32 one-hot)
//   [128, 140)  state of each side's neighbour: outside / placed / free (4 x 3)
//   [140, 204)  free sides: edges of that colour still on unplaced pieces, 0..15+ (4 x 16)
//   [204, 236)  x and y of the position (2 x 16)
//   [236, 252)  depth: level * 16 / n
//   [252, 255)  kind: centre / border / corner
//   255         constant 1
//   [256, 512)  colours of the first two free sides, hashed (c1 * 32 + c2) mod 256
__global__ void features_kernel(const uint32_t* __restrict__ ftab, const unsigned long long* __restrict__ ftab_off,
                                const FeatItem* __restrict__ items, uint64_t n, const uint16_t* __restrict__ prefixes,
                                uint16_t* __restrict__ out_bf16, float* __restrict__ out_f32)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nwarps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5; i < n; i += nwarps) {
        if (out_bf16) {
            uint4* row = reinterpret_cast<uint4*>(out_bf16 + i * kMlpIn);
            row[lane] = make_uint4(0, 0, 0, 0);
            row[lane + 32] = make_uint4(0, 0, 0, 0);
        } else {
            uint4* row = reinterpret_cast<uint4*>(out_f32 + i * kMlpIn);
            for (uint32_t j = 0; j < 4; ++j) row[lane + 32 * j] = make_uint4(0, 0, 0, 0);
        }
        const FeatItem it = items[i];
        const uint32_t* T = ftab + ftab_off[it.puzzle];
        const uint32_t l = it.len, nlev = T[0];
        const uint32_t A = T[kFtLevelA + l];
        const uint32_t kind = (A >> 8) & 0xFFu;
        const uint32_t x = min((A >> 16) & 0xFFu, 15u), y = min(A >> 24, 15u);
        const uint32_t cand = T[T[kFtKindOff + kind] + it.t];
        const uint32_t b0 = T[kFtLevelB + 2 * l], b1 = T[kFtLevelB + 2 * l + 1];
        const uint32_t nb[4] = {b0 & 0xFFFFu, b0 >> 16, b1 & 0xFFFFu, b1 >> 16};
        // edges of each free side's colour on the pieces placed before this level
        const uint16_t* pre = prefixes + it.prefix_off;
        uint32_t placed[4] = {0, 0, 0, 0};
        for (uint32_t j = lane; j < l; j += 32) {
            const uint32_t kj = (T[kFtLevelA + j] >> 8) & 0xFFu;
            const uint32_t cj = T[T[kFtKindOff + kj] + pre[j]];
            for (uint32_t s = 0; s < 4; ++s) placed[s] += colour_edges(cj, side_colour(cand, s));
        }
        for (uint32_t s = 0; s < 4; ++s) placed[s] = __reduce_add_sync(kFull, placed[s]);
        __syncwarp();
        if (lane == 0) {
            uint32_t idx[24];
            uint32_t k = 0;
            uint32_t free_col[2];
            uint32_t nfree = 0;
            for (uint32_t s = 0; s < 4; ++s) {
                const uint32_t c = side_colour(cand, s);
                idx[k++] = 32 * s + c;
                const uint32_t state = nb[s] == 0xFFFFu ? 0u : (nb[s] < l ? 1u : 2u);
                idx[k++] = 128 + 3 * s + state;
                if (state == 2) {
                    const uint32_t left = T[kFtColours + c] - placed[s] - colour_edges(cand, c);
                    idx[k++] = 140 + 16 * s + min(left, 15u);
                    if (nfree < 2) free_col[nfree++] = c;
                }
            }
            idx[k++] = 204 + x;
            idx[k++] = 220 + y;
            idx[k++] = 236 + min(l * 16 / max(nlev, 1u), 15u);
            idx[k++] = 252 + min(kind, 2u);
            idx[k++] = 255;
            if (nfree == 2) idx[k++] = 256 + ((free_col[0] * 32 + free_col[1]) & 255u);
            else if (nfree == 1) idx[k++] = 256 + free_col[0];
            for (uint32_t j = 0; j < k; ++j) {
                if (out_bf16) out_bf16[i * kMlpIn + idx[j]] = 0x3F80u;  // bf16 1.0
                else out_f32[i * kMlpIn + idx[j]] = 1.0f;
            }
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// tensor-core inference
//
// One CTA (128 threads) scores 128 rows at a time:
//   layer 1  D1[128 x 256] = X[128 x 512] . W1^T      4 chunks of K = 128
//   layer 2  D2[128 x 256] = relu(D1 + b1) . W2^T     2 chunks of K = 128
//   score    relu(D2 + b2) . w3 + b3                  in the epilogue
// Operands sit in shared memory in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, K-adjacent core matrices 128 bytes
// apart (LBO), 8-row groups K*2*8 bytes apart (SBO).  Accumulators live in
// tensor memory (512 columns: D1 in [0, 256), D2 in [256, 512)); thread 0
// issues the MMAs, an mbarrier signalled by tcgen05.commit reports completion.
constexpr uint32_t kTileRows = 128;
constexpr uint32_t kChunk = 128;
constexpr uint32_t kSmX = 0;                              // 128 x 128 bf16: 32 KB
constexpr uint32_t kSmB = kSmX + kTileRows * kChunk * 2;  // 256 x 128 bf16: 64 KB
constexpr uint32_t kSmH = kSmB + kMlpHidden * kChunk * 2; // 128 x 256 bf16: 64 KB
constexpr uint32_t kSmVec = kSmH + kTileRows * kMlpHidden * 2;  // b1, b2, w3 (f32)
constexpr uint32_t kSmBar = kSmVec + 3 * kMlpHidden * 4;
constexpr uint32_t kSmTotal = kSmBar + 16;
constexpr unsigned long long kWaitNs = 2000000000ull;     // 2 s per wait

// byte offset of element (r, k) in a K-major canonical tile whose rows hold kk elements
__device__ __forceinline__ uint32_t canon(uint32_t r, uint32_t k, uint32_t kk)
{
    return (r >> 3) * (kk * 16) + (k >> 3) * 128 + (r & 7u) * 16 + (k & 7u) * 2;
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= 1ull << 46;  // descriptor version of sm_100
    return d;         // base offset 0, layout type 0 (no swizzle)
}

// kind::f16 instruction descriptor: F32 accumulate, BF16 A and B, both K-major,
// N = 256, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((kMlpHidden >> 3) << 17) | ((kTileRows >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity)
{
    const unsigned long long deadline = global_ns() + kWaitNs;
    for (;;) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (global_ns() > deadline) return false;
    }
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 32 consecutive f32 accumulator columns of this thread's row
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v)
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// copies rows [0, rows) x k-range [k0, k0 + kChunk) of a row-major bf16 matrix
// (ld elements per row) into a canonical tile; rows >= valid are zero
__device__ __forceinline__ void stage_chunk(uint8_t* dst, const uint16_t* src, uint32_t rows, uint64_t valid,
                                            uint32_t ld, uint32_t k0)
{
    for (uint32_t p = threadIdx.x; p < rows * (kChunk / 8); p += blockDim.x) {
        const uint32_t r = p / (kChunk / 8), kb = p % (kChunk / 8);
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r < valid) v = *reinterpret_cast<const uint4*>(src + static_cast<uint64_t>(r) * ld + k0 + kb * 8);
        *reinterpret_cast<uint4*>(dst + canon(r, kb * 8, kChunk)) = v;
    }
}

__global__ void __launch_bounds__(128, 1)
    mlp_infer_kernel(const uint16_t* __restrict__ x, uint64_t n, const uint16_t* __restrict__ w1,
                     const uint16_t* __restrict__ w2, const float* __restrict__ params, float* __restrict__ out,
                     int* err)
{
    extern __shared__ __align__(1024) uint8_t sm[];
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    const uint32_t base = static_cast<uint32_t>(__cvta_generic_to_shared(sm));
    const uint32_t bar = base + kSmBar;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + kSmBar + 8);
    float* vb1 = reinterpret_cast<float*>(sm + kSmVec);
    float* vb2 = vb1 + kMlpHidden;
    float* vw3 = vb2 + kMlpHidden;
    for (uint32_t j = tid; j < kMlpHidden; j += blockDim.x) {
        vb1[j] = params[kOffB1 + j];
        vb2[j] = params[kOffB2 + j];
        vw3[j] = params[kOffW3 + j];
    }
    const float b3 = params[kOffB3];
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        const uint32_t slot = static_cast<uint32_t>(__cvta_generic_to_shared(tmem_slot));
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(slot) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t d1 = tmem, d2 = tmem + kMlpHidden;
    const uint32_t lane_base = (32u * (warp & 3u)) << 16;  // this warp's 32 tensor-memory lanes
    uint32_t phase = 0;
    bool failed = false;
    const uint64_t tiles = (n + kTileRows - 1) / kTileRows;

    for (uint64_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const uint64_t row0 = tile * kTileRows;
        const uint64_t valid = n - row0 < kTileRows ? n - row0 : kTileRows;
        // ---- layer 1 ----
        for (uint32_t c = 0; c < kMlpIn / kChunk && !failed; ++c) {
            stage_chunk(sm + kSmX, x + row0 * kMlpIn, kTileRows, valid, kMlpIn, c * kChunk);
            stage_chunk(sm + kSmB, w1, kMlpHidden, kMlpHidden, kMlpIn, c * kChunk);
            fence_proxy_async();
            fence_before();
            __syncthreads();
            if (tid == 0) {
                fence_after();
                for (uint32_t kk = 0; kk < kChunk / 16; ++kk) {
                    const uint64_t a = smem_desc(base + kSmX + kk * 256, 128, kChunk * 16);
                    const uint64_t b = smem_desc(base + kSmB + kk * 256, 128, kChunk * 16);
                    mma_bf16(d1, a, b, (c | kk) != 0);
                }
                mma_commit(bar);
            }
            failed = __syncthreads_or(!bar_wait(bar, phase));
            phase ^= 1u;
            fence_after();
        }
        if (failed) break;
        // ---- epilogue 1: bias, relu, bf16 into the layer-2 operand ----
        const uint32_t r = tid;  // this thread's row = its tensor-memory lane
        for (uint32_t c0 = 0; c0 < kMlpHidden; c0 += 32) {
            float v[32];
            tmem_ld32(d1 + lane_base + c0, v);
            for (uint32_t g = 0; g < 4; ++g) {
                uint32_t w[4];
                for (uint32_t h = 0; h < 4; ++h) {
                    const uint32_t j = c0 + g * 8 + 2 * h;
                    const __nv_bfloat162 pr =
                        __floats2bfloat162_rn(fmaxf(v[g * 8 + 2 * h] + vb1[j], 0.f), fmaxf(v[g * 8 + 2 * h + 1] + vb1[j + 1], 0.f));
                    w[h] = *reinterpret_cast<const uint32_t*>(&pr);
                }
                *reinterpret_cast<uint4*>(sm + kSmH + canon(r, c0 + g * 8, kMlpHidden)) = make_uint4(w[0], w[1], w[2], w[3]);
            }
        }
        fence_proxy_async();
        // ---- layer 2 ----
        for (uint32_t c = 0; c < kMlpHidden / kChunk && !failed; ++c) {
            stage_chunk(sm + kSmB, w2, kMlpHidden, kMlpHidden, kMlpHidden, c * kChunk);
            fence_proxy_async();
            fence_before();
            __syncthreads();
            if (tid == 0) {
                fence_after();
                for (uint32_t kk = 0; kk < kChunk / 16; ++kk) {
                    const uint64_t a = smem_desc(base + kSmH + (c * kChunk / 8 + kk * 2) * 128, 128, kMlpHidden * 16);
                    const uint64_t b = smem_desc(base + kSmB + kk * 256, 128, kChunk * 16);
                    mma_bf16(d2, a, b, (c | kk) != 0);
                }
                mma_commit(bar);
            }
            failed = __syncthreads_or(!bar_wait(bar, phase));
            phase ^= 1u;
            fence_after();
        }
        if (failed) break;
        // ---- epilogue 2: bias, relu, dot with w3 ----
        float score = b3;
        for (uint32_t c0 = 0; c0 < kMlpHidden; c0 += 32) {
            float v[32];
            tmem_ld32(d2 + lane_base + c0, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) score += fmaxf(v[j] + vb2[c0 + j], 0.f) * vw3[c0 + j];
        }
        if (r < valid) out[row0 + r] = score;
        fence_before();
        __syncthreads();
    }
    if (failed) {
        if (tid == 0) atomicExch(err, 1);
        bar_wait(bar, phase ^ 1u);  // the phase that timed out: let its MMAs finish (bounded) before freeing
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
    }
}

// ---------------------------------------------------------------------------
// f32 training kernels

// C[m][n] = alpha * sum_k A(m, k) B(k, n) + beta * C[m][n]; A(m, k) = A[m*sam + k*sak],
// B(k, n) = B[k*sbk + n*sbn], C row-major with ldc.  32x32 tiles, 256 threads.
__global__ void gemm_f32_kernel(const float* __restrict__ A, const float* __restrict__ B, float* __restrict__ C,
                                uint32_t M, uint32_t N, uint32_t K, uint64_t sam, uint64_t sak, uint64_t sbk,
                                uint64_t sbn, uint32_t ldc, float alpha, float beta)
{
    __shared__ float As[32][33];
    __shared__ float Bs[32][33];
    const uint32_t tx = threadIdx.x & 31u, ty = threadIdx.x >> 5;  // ty in 0..7
    const uint32_t m0 = blockIdx.y * 32, n0 = blockIdx.x * 32;
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (uint32_t k0 = 0; k0 < K; k0 += 32) {
        for (uint32_t i = ty; i < 32; i += 8) {
            const uint32_t m = m0 + i, k = k0 + tx;
            As[i][tx] = (m < M && k < K) ? A[m * sam + k * sak] : 0.f;
            const uint32_t kb = k0 + i, nb = n0 + tx;
            Bs[i][tx] = (kb < K && nb < N) ? B[kb * sbk + nb * sbn] : 0.f;
        }
        __syncthreads();
        for (uint32_t kk = 0; kk < 32; ++kk) {
            const float b = Bs[kk][tx];
            for (uint32_t j = 0; j < 4; ++j) acc[j] += As[ty + 8 * j][kk] * b;
        }
        __syncthreads();
    }
    for (uint32_t j = 0; j < 4; ++j) {
        const uint32_t m = m0 + ty + 8 * j, nn = n0 + tx;
        if (m < M && nn < N) {
            float* c = C + static_cast<uint64_t>(m) * ldc + nn;
            *c = alpha * acc[j] + (beta != 0.f ? beta * *c : 0.f);
        }
    }
}

cudaError_t gemm_f32(const float* A, const float* B, float* C, uint32_t M, uint32_t N, uint32_t K, uint64_t sam,
                     uint64_t sak, uint64_t sbk, uint64_t sbn, uint32_t ldc, float alpha, float beta,
                     cudaStream_t st)
{
    if (!M || !N) return cudaSuccess;
    dim3 grid((N + 31) / 32, (M + 31) / 32);
    gemm_f32_kernel<<<grid, 256, 0, st>>>(A, B, C, M, N, K, sam, sak, sbk, sbn, ldc, alpha, beta);
    return cudaGetLastError();
}

__global__ void bias_relu_kernel(float* h, const float* __restrict__ b, uint64_t rows, uint32_t cols)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < rows * cols;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        h[i] = fmaxf(h[i] + b[i % cols], 0.f);
}

// s[r] = h2[r] . w3 + b3 (one warp per row)
__global__ void score_f32_kernel(const float* __restrict__ h2, const float* __restrict__ params, uint64_t rows,
                                 float* __restrict__ s)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t nw = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t r = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5; r < rows; r += nw) {
        float acc = 0.f;
        for (uint32_t j = lane; j < kMlpHidden; j += 32) acc += h2[r * kMlpHidden + j] * params[kOffW3 + j];
        for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
        if (lane == 0) s[r] = acc + params[kOffB3];
    }
}

// weighted logistic loss: loss[0] += w * (softplus(s) - y s), loss[1] += w; ds = w (sigmoid(s) - y)
__global__ void loss_kernel(const float* __restrict__ s, const float* __restrict__ y, const float* __restrict__ wt,
                            uint64_t rows, float* __restrict__ ds, double* loss)
{
    double l = 0, wsum = 0;
    for (uint64_t r = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; r < rows;
         r += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const float v = s[r], w = wt[r];
        const float sp = v > 0.f ? v + log1pf(expf(-v)) : log1pf(expf(v));
        const float sig = 1.f / (1.f + expf(-v));
        l += static_cast<double>(w) * (sp - y[r] * v);
        wsum += w;
        ds[r] = w * (sig - y[r]);
    }
    for (int o = 16; o; o >>= 1) {
        l += __shfl_xor_sync(kFull, l, o);
        wsum += __shfl_xor_sync(kFull, wsum, o);
    }
    if ((threadIdx.x & 31u) == 0) {
        atomicAdd(&loss[0], l);
        atomicAdd(&loss[1], wsum);
    }
}

__global__ void scale_by_weight_sum_kernel(float* v, uint64_t n, const double* loss)
{
    const float inv = loss[1] > 0 ? static_cast<float>(1.0 / loss[1]) : 0.f;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        v[i] *= inv;
}

// dh2 = ds (x) w3, masked where h2 == 0 (relu)
__global__ void dh2_kernel(const float* __restrict__ ds, const float* __restrict__ h2, const float* __restrict__ params,
                           uint64_t rows, float* __restrict__ dh2)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < rows * kMlpHidden;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t r = i / kMlpHidden;
        const uint32_t j = static_cast<uint32_t>(i % kMlpHidden);
        dh2[i] = h2[i] > 0.f ? ds[r] * params[kOffW3 + j] : 0.f;
    }
}

__global__ void relu_mask_kernel(float* d, const float* __restrict__ h, uint64_t n)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        if (!(h[i] > 0.f)) d[i] = 0.f;
}

// out[j] = sum_r d[r][j] (one thread per column; column sums of small matrices)
__global__ void colsum_kernel(const float* __restrict__ d, uint64_t rows, uint32_t cols, float* __restrict__ out)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols) return;
    float acc = 0.f;
    for (uint64_t r = 0; r < rows; ++r) acc += d[r * cols + j];
    out[j] = acc;
}

__global__ void adam_kernel(float* p, const float* __restrict__ g, float* m1, float* m2, uint32_t n, float lr,
                            float c1, float c2)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float a = 0.9f * m1[i] + 0.1f * gi;
        const float b = 0.999f * m2[i] + 0.001f * gi * gi;
        m1[i] = a;
        m2[i] = b;
        p[i] -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
    }
}

__global__ void pack_bf16_kernel(const float* __restrict__ src, uint16_t* __restrict__ dst, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const __nv_bfloat16 v = __float2bfloat16_rn(src[i]);
        dst[i] = *reinterpret_cast<const uint16_t*>(&v);
    }
}

uint32_t grid_for(uint64_t n, uint32_t threads)
{
    return static_cast<uint32_t>(std::min<uint64_t>((n + threads - 1) / threads, 148ull * 16));
}

__global__ void f32_to_bf16_kernel(const float* __restrict__ src, uint16_t* __restrict__ dst, uint64_t n)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const __nv_bfloat16 v = __float2bfloat16_rn(src[i]);
        dst[i] = *reinterpret_cast<const uint16_t*>(&v);
    }
}

__global__ void gather_rows_kernel(const float* __restrict__ src, const uint32_t* __restrict__ idx, uint64_t n,
                                   uint32_t cols, float* __restrict__ dst, const float* __restrict__ y,
                                   const float* __restrict__ w, float* __restrict__ y_out, float* __restrict__ w_out)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n * cols;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t r = i / cols;
        const uint32_t c = static_cast<uint32_t>(i % cols);
        const uint64_t from = idx[r];
        dst[i] = src[from * cols + c];
        if (c == 0) {
            y_out[r] = y[from];
            w_out[r] = w[from];
        }
    }
}

// item (prefix first + j, level 1 + k); levels at or past the puzzle's own prefix
// length get len = 0 (skipped when summing)
__global__ void order_items_kernel(const uint16_t* __restrict__ prefixes, const uint32_t* __restrict__ prefix_puzzle,
                                   const uint32_t* __restrict__ puzzle_depth, uint32_t depth, uint64_t first,
                                   uint64_t count, FeatItem* __restrict__ items)
{
    const uint32_t per = depth - 1;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < count * per;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t p = first + i / per;
        const uint32_t l = 1 + static_cast<uint32_t>(i % per);
        const uint32_t pz = prefix_puzzle[p];
        const uint32_t len = puzzle_depth ? puzzle_depth[pz] : depth;
        FeatItem it;
        it.prefix_off = p * depth;
        it.puzzle = pz;
        if (l < len) {
            it.len = static_cast<uint16_t>(l);
            it.t = prefixes[p * depth + l];
        } else {
            it.len = 0;
            it.t = prefixes[p * depth];
        }
        items[i] = it;
    }
}

__global__ void order_accumulate_kernel(const float* __restrict__ scores, const FeatItem* __restrict__ items,
                                        uint64_t count, uint32_t depth, float* __restrict__ prefix_score)
{
    const uint32_t per = depth - 1;
    for (uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; j < count;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        float acc = 0.f;
        for (uint32_t k = 0; k < per; ++k) {
            const uint64_t i = j * per + k;
            if (!items[i].len) continue;
            const float v = scores[i];
            acc -= fmaxf(-v, 0.f) + log1pf(expf(-fabsf(v)));  // log sigmoid(v)
        }
        prefix_score[j] = acc;
    }
}

}  // namespace

cudaError_t launch_f32_to_bf16(const float* src, uint16_t* dst, uint64_t n, cudaStream_t stream)
{
    if (!n) return cudaSuccess;
    f32_to_bf16_kernel<<<grid_for(n, 256), 256, 0, stream>>>(src, dst, n);
    return cudaGetLastError();
}

cudaError_t launch_gather_rows(const float* src, const uint32_t* idx, uint64_t n, uint32_t cols, float* dst,
                               const float* y, const float* w, float* y_out, float* w_out, cudaStream_t stream)
{
    if (!n) return cudaSuccess;
    gather_rows_kernel<<<grid_for(n * cols, 256), 256, 0, stream>>>(src, idx, n, cols, dst, y, w, y_out, w_out);
    return cudaGetLastError();
}

cudaError_t launch_order_items(const uint16_t* prefixes, const uint32_t* prefix_puzzle, const uint32_t* puzzle_depth,
                               uint32_t depth, uint64_t first, uint64_t count, FeatItem* items, cudaStream_t stream)
{
    if (!count || depth < 2) return cudaSuccess;
    order_items_kernel<<<grid_for(count * (depth - 1), 256), 256, 0, stream>>>(prefixes, prefix_puzzle, puzzle_depth,
                                                                               depth, first, count, items);
    return cudaGetLastError();
}

cudaError_t launch_order_accumulate(const float* scores, const FeatItem* items, uint64_t count, uint32_t depth,
                                    float* prefix_score, cudaStream_t stream)
{
    if (!count || depth < 2) return cudaSuccess;
    order_accumulate_kernel<<<grid_for(count, 256), 256, 0, stream>>>(scores, items, count, depth, prefix_score);
    return cudaGetLastError();
}

cudaError_t launch_features(const uint32_t* ftab, const unsigned long long* ftab_off, const FeatItem* items,
                            uint64_t n, const uint16_t* prefixes, void* out_bf16, float* out_f32, cudaStream_t stream)
{
    if (!n) return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 7) / 8, 148ull * 32);  // 8 warps (rows) per block
    features_kernel<<<static_cast<uint32_t>(blocks), 256, 0, stream>>>(
        ftab, ftab_off, items, n, prefixes, static_cast<uint16_t*>(out_bf16), out_f32);
    return cudaGetLastError();
}

cudaError_t launch_mlp_pack_bf16(const MlpDevice& m, cudaStream_t stream)
{
    pack_bf16_kernel<<<256, 256, 0, stream>>>(m.params + kOffW1, m.w1_bf16, kMlpHidden * kMlpIn);
    pack_bf16_kernel<<<256, 256, 0, stream>>>(m.params + kOffW2, m.w2_bf16, kMlpHidden * kMlpHidden);
    return cudaGetLastError();
}

size_t mlp_infer_smem_bytes() { return kSmTotal; }

cudaError_t launch_mlp_infer_tc(const MlpDevice& m, const void* x_bf16, uint64_t n, float* scores, int* err,
                                cudaStream_t stream)
{
    if (!n) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(mlp_infer_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kSmTotal));
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t tiles = (n + kTileRows - 1) / kTileRows;
    const uint32_t grid = static_cast<uint32_t>(std::min<uint64_t>(tiles, static_cast<uint64_t>(sms)));
    mlp_infer_kernel<<<grid, 128, kSmTotal, stream>>>(static_cast<const uint16_t*>(x_bf16), n, m.w1_bf16, m.w2_bf16,
                                                      m.params, scores, err);
    return cudaGetLastError();
}

cudaError_t mlp_forward_f32(const MlpDevice& m, const MlpWork& w, const float* x, uint64_t n, cudaStream_t st)
{
    const uint32_t H = kMlpHidden;
    // h1 = x . W1^T + b1, relu
    cudaError_t e = gemm_f32(x, m.params + kOffW1, w.h1, static_cast<uint32_t>(n), H, kMlpIn, kMlpIn, 1, 1, kMlpIn, H,
                             1.f, 0.f, st);
    if (e != cudaSuccess) return e;
    bias_relu_kernel<<<grid_for(n * H, 256), 256, 0, st>>>(w.h1, m.params + kOffB1, n, H);
    // h2 = h1 . W2^T + b2, relu
    e = gemm_f32(w.h1, m.params + kOffW2, w.h2, static_cast<uint32_t>(n), H, H, H, 1, 1, H, H, 1.f, 0.f, st);
    if (e != cudaSuccess) return e;
    bias_relu_kernel<<<grid_for(n * H, 256), 256, 0, st>>>(w.h2, m.params + kOffB2, n, H);
    score_f32_kernel<<<grid_for(n * 32, 256), 256, 0, st>>>(w.h2, m.params, n, w.s);
    return cudaGetLastError();
}

cudaError_t mlp_loss_backward_f32(const MlpDevice& m, const MlpWork& w, const float* x, const float* y,
                                  const float* weight, uint64_t n, cudaStream_t st)
{
    const uint32_t H = kMlpHidden;
    const uint32_t R = static_cast<uint32_t>(n);
    cudaError_t e = cudaMemsetAsync(w.loss, 0, 2 * sizeof(double), st);
    if (e != cudaSuccess) return e;
    loss_kernel<<<grid_for(n, 256), 256, 0, st>>>(w.s, y, weight, n, w.ds, w.loss);
    scale_by_weight_sum_kernel<<<grid_for(n, 256), 256, 0, st>>>(w.ds, n, w.loss);
    float* g = w.grad;
    // dw3 = h2^T ds, db3 = sum ds
    if ((e = gemm_f32(w.ds, w.h2, g + kOffW3, 1, H, R, 0, 1, H, 1, H, 1.f, 0.f, st)) != cudaSuccess) return e;
    colsum_kernel<<<1, 32, 0, st>>>(w.ds, n, 1, g + kOffB3);
    // dh2 = ds w3 masked; dW2 = dh2^T h1; db2 = colsum dh2
    dh2_kernel<<<grid_for(n * H, 256), 256, 0, st>>>(w.ds, w.h2, m.params, n, w.dh2);
    if ((e = gemm_f32(w.dh2, w.h1, g + kOffW2, H, H, R, 1, H, H, 1, H, 1.f, 0.f, st)) != cudaSuccess) return e;
    colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(w.dh2, n, H, g + kOffB2);
    // dh1 = dh2 W2 masked; dW1 = dh1^T x; db1 = colsum dh1
    if ((e = gemm_f32(w.dh2, m.params + kOffW2, w.dh1, R, H, H, H, 1, H, 1, H, 1.f, 0.f, st)) != cudaSuccess) return e;
    relu_mask_kernel<<<grid_for(n * H, 256), 256, 0, st>>>(w.dh1, w.h1, n * H);
    if ((e = gemm_f32(w.dh1, x, g + kOffW1, H, kMlpIn, R, 1, H, kMlpIn, 1, kMlpIn, 1.f, 0.f, st)) != cudaSuccess)
        return e;
    colsum_kernel<<<(H + 127) / 128, 128, 0, st>>>(w.dh1, n, H, g + kOffB1);
    return cudaGetLastError();
}

cudaError_t mlp_adam_step(const MlpDevice& m, const float* grad, float* m1, float* m2, float lr, uint32_t step,
                          cudaStream_t st)
{
    const float c1 = 1.f - powf(0.9f, static_cast<float>(step));
    const float c2 = 1.f - powf(0.999f, static_cast<float>(step));
    adam_kernel<<<256, 256, 0, st>>>(m.params, grad, m1, m2, kMlpParams, lr, c1, c2);
    return cudaGetLastError();
}

}  // namespace emp
