// Fitness evaluation, plain FP32 form: every individual's Wordle episodes played in lockstep.
//
// Replaces the reference's evaluation kernels (genetic_algorithm/device/slab_runtime.cu:311-549) and
// their per-warp forward (inference/dynamic_policy.hpp:67-151, model/*). One CTA owns a chunk of up
// to 128 games of one individual, all at the same turn count, and plays them turn by turn. Every
// layer runs as a CTA-wide FFMA register-tiled GEMM with the games as rows:
//
//   encoder (new turn only)  gather of the 10 one-hot weight columns, then 128 -> 64
//   trunk layer 1            cached accumulator per game, extended by the new turn's 64 inputs
//   trunk layers 2, 3        256 -> 128 ReLU -> 64
//   scoring + argmax         policy (128 x 64) x catalog embeddings (64 x A), fused masked argmax
//                            (at <= 128 selectable actions: the reference's FP16 tensor-tile scoring instead)
//
// Bit-exactness with the reference's device arithmetic: each output is the same chain of fused
// multiply-adds in the same input order as the reference's `sum += w * x` loops (bias first, inputs
// ascending). Terms whose input is exactly zero (empty turn slots, one-hot zeros) change a chain only
// in the sign of a zero result, which no comparison can see, so the encoder's one-hot layer is a gather
// and the trunk's first layer keeps its running accumulator from turn to turn (a new turn appends
// its 64 inputs to the end of the chain). Ties in the argmax go to the lowest action index, and
// guessed words are masked by word equality, as in the reference.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <mma.h>

#include <cstdint>

#include "eval_common.cuh"
#include "trunk_fp32.cuh"

namespace nwg {
namespace {

using namespace evalx;

// Per-cell word counts and chunk offsets (one CTA, block-wide scan).
__global__ void EvalPrepareKernel(WordSource src, std::uint32_t population, std::uint32_t catalog_count,
                                  std::uint32_t *local_words, std::uint32_t *chunk_start, std::uint32_t *score_sum,
                                  int *status) {
    __shared__ std::uint32_t partial[1024];
    const std::uint32_t t = threadIdx.x;
    const std::uint32_t per = (population + blockDim.x - 1) / blockDim.x;
    const std::uint32_t begin = t * per;
    const std::uint32_t end = min(population, begin + per);
    std::uint32_t sum = 0;
    for (std::uint32_t i = begin; i < end; ++i) {
        std::uint32_t w = 0;
        // explicit lists: a decreasing pair of offsets would read as a huge count; such a cell, an empty one and
        // one longer than kMaxCellWords are refused and get no chunks, so no kernel reads past its list
        const bool ordered = src.mode != 0 || src.cell_offsets[i + 1] >= src.cell_offsets[i];
        if (ordered) {
            w = CountWords(src, i);
        }
        if (!ordered || w == 0 || w > kMaxCellWords) {
            SetStatus(status, kInvalidTrainingShard);
            w = 0;
        }
        local_words[i] = w;
        score_sum[i] = 0;
        sum += ChunksForWords(w);
    }
    partial[t] = sum;
    __syncthreads();
    for (std::uint32_t off = 1; off < blockDim.x; off <<= 1) {
        const std::uint32_t v = t >= off ? partial[t - off] : 0;
        __syncthreads();
        partial[t] += v;
        __syncthreads();
    }
    std::uint32_t run = partial[t] - sum;
    for (std::uint32_t i = begin; i < end; ++i) {
        chunk_start[i] = run;
        run += ChunksForWords(local_words[i]);
    }
    if (t == blockDim.x - 1) {
        chunk_start[population] = partial[t];
    }
    (void)catalog_count;
}

// Scores every action for every game (policy vectors in arena[0 .. kTile)), with the FP32 register-tiled
// micro-kernel and a fused masked argmax; the choice lands in st.best[g].
__device__ __forceinline__ void ScoreFp32(const EvalParams &p, ChunkState &st, const __half *gh, float *arena, int t) {
    const int tid = threadIdx.x;
    const int ty = tid >> 4;
    const int tx = tid & 15;
    const float *pv = arena;
    float best_s[8];
    int best_i[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        best_s[i] = 0.0f;
        best_i[i] = -1;
    }
    const int n_tiles = static_cast<int>((p.action_count + 127) / 128);
    const __half2 *tail2 = reinterpret_cast<const __half2 *>(reinterpret_cast<const std::uint8_t *>(gh) +
                                                             kTailOffsetBytes);
    for (int tile = 0; tile < n_tiles; ++tile) {
        float *eb = arena + kTile + (tile & 1) * kTile;  // [64][kLd] embeddings of 128 actions
        const int a0 = tile * 128;
        for (int idx = tid; idx < kFixedDim * 128; idx += kEvalThreads) {
            const int k = idx >> 7;
            const int a = idx & 127;
            eb[k * kLd + a] = p.fixed_t[static_cast<std::size_t>(k) * p.action_pad + a0 + a];
        }
        for (int idx = tid; idx < 128 * (kTailDim / 2); idx += kEvalThreads) {
            const int a = idx / (kTailDim / 2);
            const int j = idx - a * (kTailDim / 2);
            float2 v = make_float2(0.0f, 0.0f);
            if (a0 + a < static_cast<int>(p.action_count)) {
                v = __half22float2(tail2[static_cast<std::size_t>(a0) * (kTailDim / 2) + idx]);
            }
            eb[(kFixedDim + 2 * j) * kLd + a] = v.x;
            eb[(kFixedDim + 2 * j + 1) * kLd + a] = v.y;
        }
        if (tid < 128) {
            st.tile_codes[tile & 1][tid] =
                (a0 + tid < static_cast<int>(p.action_count)) ? p.codes[a0 + tid] : 0u;
        }
        __syncthreads();
        float sacc[8][8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                sacc[i][j] = 0.0f;
            }
        }
        MmaChain<8>(sacc, pv, eb, kLd, 64, ty, tx);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int g = RowOf(ty, i);
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int al = ColOf8(tx, j);
                const int a = a0 + al;
                const float s = sacc[i][j];
                if (a < static_cast<int>(p.action_count) && (best_i[i] < 0 || s > best_s[i])) {
                    const std::uint32_t code = st.tile_codes[tile & 1][al];
                    bool masked = false;
                    for (int u = 0; u < t; ++u) {
                        masked |= st.guess[u][g] == code;
                    }
                    if (!masked) {
                        best_s[i] = s;
                        best_i[i] = a;
                    }
                }
            }
        }
    }
    // reduce over the 16 threads that share these games (score desc, index asc)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int off = 8; off > 0; off >>= 1) {
            const float os = __shfl_xor_sync(0xffffffffu, best_s[i], off);
            const int oi = __shfl_xor_sync(0xffffffffu, best_i[i], off);
            if (oi >= 0 && (best_i[i] < 0 || os > best_s[i] || (os == best_s[i] && oi < best_i[i]))) {
                best_s[i] = os;
                best_i[i] = oi;
            }
        }
        if (tx == 0) {
            st.best[RowOf(ty, i)] = best_i[i];
        }
    }
    __syncthreads();

}

// Action spaces of at most kSmallActionSpace selectable actions, where the reference scores with its tensor-tile
// path (slab_runtime.cu:70 and :1126-1140; evaluation_ops.cuh:286-388): the policy vector rounded to FP16, the
// fixed features rounded to FP16 (small integers, exact) and the FP16 tail form a 64-deep product, accumulated in
// FP32 by a 16x16x16 FP16 tensor-core MMA over the depth chunks [0,16), [16,32), [32,48), [48,64) in that order,
// from a zero accumulator. Each score depends only on its own policy row and action column, so the same MMA over
// this chunk's 128 games x 128 actions gives the reference's scores bit for bit; the argmax walks the actions in
// ascending order with ties to the lowest index, as the reference's lane-0 scan does.
constexpr int kSmallActionSpace = 128;
constexpr int kSmallALd = 72;   // halfs per policy row (64 + 8)
constexpr int kSmallBLd = 136;  // halfs per feature row of the action tile (128 + 8)
constexpr int kSmallCLd = 20;   // floats per row of a warp's 16 x 16 score tile

__device__ __forceinline__ void ScoreSmallActionSpace(const EvalParams &p, ChunkState &st, const __half *gh,
                                                      float *arena, int t) {
    namespace wmma = nvcuda::wmma;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int actions = static_cast<int>(p.action_count);
    const float *pv = arena;  // [64][kLd] policy vectors, feature-major
    // MMA operands must start on 32-byte boundaries: align the base up to 128 bytes (the buffers below end
    // 21,504 bytes before the arena does)
    const std::uintptr_t free_base = reinterpret_cast<std::uintptr_t>(arena + kTile);
    __half *ah = reinterpret_cast<__half *>((free_base + 127u) & ~static_cast<std::uintptr_t>(127u));  // [128][72]
    __half *bh = ah + kChunkGames * kSmallALd;               // [64 features][kSmallBLd]
    float *cw = reinterpret_cast<float *>(bh + 64 * kSmallBLd) + warp * 16 * kSmallCLd;
    const __half *tail = reinterpret_cast<const __half *>(reinterpret_cast<const std::uint8_t *>(gh) +
                                                          kTailOffsetBytes);
    for (int idx = tid; idx < kChunkGames * 64; idx += kEvalThreads) {
        const int g = idx >> 6;
        const int k = idx & 63;
        ah[g * kSmallALd + k] = __float2half_rn(pv[k * kLd + g]);
    }
    for (int idx = tid; idx < 64 * kSmallActionSpace; idx += kEvalThreads) {
        const int k = idx >> 7;
        const int a = idx & 127;
        __half v = __float2half_rn(0.0f);
        if (a < actions) {
            v = k < kFixedDim ? __float2half_rn(p.fixed_t[static_cast<std::size_t>(k) * p.action_pad + a])
                              : tail[static_cast<std::size_t>(a) * kTailDim + (k - kFixedDim)];
        }
        bh[k * kSmallBLd + a] = v;
    }
    if (tid < kSmallActionSpace) {
        st.tile_codes[0][tid] = tid < actions ? p.codes[tid] : 0u;
    }
    __syncthreads();
    // warp w: games 16w .. 16w+15; lanes 0..15 keep one game's running best
    const int g = warp * 16 + (lane & 15);
    float best_s = 0.0f;
    int best_i = -1;
    wmma::fragment<wmma::matrix_a, 16, 16, 16, __half, wmma::row_major> fa;
    wmma::fragment<wmma::matrix_b, 16, 16, 16, __half, wmma::row_major> fb;
    wmma::fragment<wmma::accumulator, 16, 16, 16, float> fc;
    for (int a0 = 0; a0 < actions; a0 += 16) {
        wmma::fill_fragment(fc, 0.0f);
#pragma unroll
        for (int k0 = 0; k0 < 64; k0 += 16) {
            wmma::load_matrix_sync(fa, ah + warp * 16 * kSmallALd + k0, kSmallALd);
            wmma::load_matrix_sync(fb, bh + k0 * kSmallBLd + a0, kSmallBLd);
            wmma::mma_sync(fc, fa, fb, fc);
        }
        wmma::store_matrix_sync(cw, fc, kSmallCLd, wmma::mem_row_major);
        __syncwarp();
        if (lane < 16) {
            for (int c = 0; c < 16 && a0 + c < actions; ++c) {
                const std::uint32_t code = st.tile_codes[0][a0 + c];
                bool masked = false;
                for (int u = 0; u < t; ++u) {
                    masked |= st.guess[u][g] == code;
                }
                const float s = cw[(lane & 15) * kSmallCLd + c];
                if (!masked && (best_i < 0 || s > best_s)) {
                    best_s = s;
                    best_i = a0 + c;
                }
            }
        }
        __syncwarp();
    }
    if (lane < 16) {
        st.best[g] = best_i;
    }
    __syncthreads();
}

// kStreamed: the encoder and trunk stream their weights from the exact trunk tables (p.xt), else from the genome.
template <bool kStreamed>
__global__ void __launch_bounds__(kEvalThreads, 2) EvalFp32Kernel(const EvalParams p) {
    extern __shared__ __align__(16) float arena[];
    __shared__ ChunkState st;
    const int tid = threadIdx.x;
    float *scratch = p.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats;
    unsigned long long decisions = 0;
    unsigned long long encoded = 0;
    unsigned long long episodes = 0;
    const std::uint32_t total_chunks = p.chunk_start[p.population];

    for (std::uint32_t chunk = blockIdx.x; chunk < total_chunks; chunk += gridDim.x) {
        if (!BeginChunk(p, st, chunk)) {
            break;
        }
        const std::uint32_t ind = static_cast<std::uint32_t>(st.individual);
        const __half *gh = reinterpret_cast<const __half *>(p.slab + static_cast<std::size_t>(st.slot) * p.pitch);
        const std::uint8_t *xt = kStreamed ? p.xt + static_cast<std::size_t>(ind) * p.xt_pitch : nullptr;
        auto encode = [&](int u) {
            if constexpr (kStreamed) {
                EncodeRoundX(st, gh, xt, arena, scratch, u);
            } else {
                EncodeRound(st, gh, arena, scratch, u);
            }
        };
        SetupGames(p, st, gh, scratch);
        if (st.cls == 1 && CountActive(st) > 0) {
            encode(0);
            encode(1);
            encoded += tid == 0 ? 2ull * st.active : 0ull;
        }
        for (int step = 0; step < kMaxTurns; ++step) {
            if (CountActive(st) == 0) {
                break;
            }
            const int t = st.cls == 0 ? step : step + 2;  // turns already on every active grid
            if (step > 0) {
                encode(t - 1);  // the turn appended by the previous decision
                encoded += tid == 0 ? static_cast<unsigned long long>(st.active) : 0ull;
            }
            if constexpr (kStreamed) {
                TrunkForwardX(p, st, gh, xt, arena, scratch, t, step, ind);
            } else {
                TrunkForward(p, st, gh, arena, scratch, t, step, ind);
            }
            if (p.action_count <= static_cast<std::uint32_t>(kSmallActionSpace)) {
                ScoreSmallActionSpace(p, st, gh, arena, t);
            } else {
                ScoreFp32(p, st, gh, arena, t);
            }
            AppendGuesses(p, st, step, decisions);
        }
        FinishChunk(p, st, ind, episodes);
    }
    FlushCounters(p, decisions, encoded, episodes);
}

// slab_runtime.cu:551-586 with evaluation_ops.cuh:97-111
__global__ void FinalizeFitnessKernel(const std::uint32_t *score_sum, const std::uint32_t *local_words,
                                      std::uint32_t population, float *fitness, std::uint32_t *evaluation_counts,
                                      std::uint8_t *has_fitness, int *status) {
    const std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= population) {
        return;
    }
    const std::uint32_t w = local_words[i];
    if (w == 0) {
        SetStatus(status, kInvalidTrainingShard);
        return;
    }
    const float raw = static_cast<float>(score_sum[i]);
    const float maximum = 3.0f * 15.0f * static_cast<float>(w);
    const float floor_value = 1.40129846e-45f;
    float normalized = raw / maximum;
    normalized = normalized >= 1.0f ? 1.0f : (normalized > floor_value ? normalized : floor_value);
    fitness[i] = normalized;
    evaluation_counts[i] += 1;
    has_fitness[i] = 1;
}

// slab_runtime.cu:588-631: best (ties to the lower index) and the sequential fp32 mean; FP64 mean and
// variance are added for the adaptive shard-release statistics.
__global__ void SummarizeKernel(const float *fitness, const std::uint8_t *has_fitness, const std::uint32_t *slots,
                                std::uint32_t population, SummaryDevice *out, int *status) {
    const int lane = threadIdx.x;
    float best = 0.0f;
    std::uint32_t best_i = 0xFFFFFFFFu;
    double sum = 0.0;
    bool missing = false;
    for (std::uint32_t i = lane; i < population; i += 32) {
        const float f = fitness[i];
        missing |= has_fitness[i] == 0;
        if (best_i == 0xFFFFFFFFu || f > best) {
            best = f;
            best_i = i;
        }
        sum += static_cast<double>(f);
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float ob = __shfl_xor_sync(0xffffffffu, best, off);
        const std::uint32_t oi = __shfl_xor_sync(0xffffffffu, best_i, off);
        if (oi != 0xFFFFFFFFu && (best_i == 0xFFFFFFFFu || ob > best || (ob == best && oi < best_i))) {
            best = ob;
            best_i = oi;
        }
        sum += __shfl_xor_sync(0xffffffffu, sum, off);
    }
    missing = __any_sync(0xffffffffu, missing);
    const double mean = sum / static_cast<double>(population);
    double sq = 0.0;
    for (std::uint32_t i = lane; i < population; i += 32) {
        const double d = static_cast<double>(fitness[i]) - mean;
        sq += d * d;
    }
    for (int off = 16; off > 0; off >>= 1) {
        sq += __shfl_xor_sync(0xffffffffu, sq, off);
    }
    if (lane == 0) {
        if (missing) {
            SetStatus(status, kPopulationNotEvaluated);
            return;
        }
        float fsum = 0.0f;
        for (std::uint32_t i = 0; i < population; ++i) {
            fsum += fitness[i];
        }
        out->best_fitness = best;
        out->average_fitness = fsum / static_cast<float>(population);
        out->best_index = best_i;
        out->best_slot_index = slots[best_i];
        out->mean_fp64 = mean;
        out->variance_fp64 = sq / static_cast<double>(population);
    }
}

// Single-model inference (inference/single_model_device_runtime.cu:53-87, dynamic_policy.hpp:67-151): the next
// guess of one genome for caller-given grids. The reference runs one grid per warp through its FP32 warp scorer,
// whatever the action count; here a CTA takes a chunk of up to 128 grids that share a turn count and runs the plain
// form's encoder, trunk and FP32 scoring (ScoreFp32, never the small-action tensor-tile path), so index and score
// are the reference's chains bit for bit. The winner's score is its 64-term chain recomputed in the scorer's
// order (zero start, inputs ascending).
__global__ void __launch_bounds__(kEvalThreads, 2) SingleModelSelectKernel(const SingleModelParams q) {
    extern __shared__ __align__(16) float arena[];
    __shared__ ChunkState st;
    const int tid = threadIdx.x;
    EvalParams p{};  // no trace
    p.action_count = q.action_count;
    p.codes = q.codes;
    p.fixed_t = q.fixed_t;
    p.action_pad = q.action_pad;
    float *scratch = q.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats;
    const __half *gh = reinterpret_cast<const __half *>(q.genome);
    const __half *tail = reinterpret_cast<const __half *>(q.genome + kTailOffsetBytes);
    for (int ck = blockIdx.x; ck < q.chunk_count; ck += gridDim.x) {
        const int4 c = q.chunks[ck];
        const int turns = c.x;
        const int begin = c.y;
        const int grids = c.z;
        if (tid < kChunkGames) {
            const int g = tid;
            const std::uint32_t grid = g < grids ? q.order[begin + g] : 0u;
            for (int u = 0; u < kMaxTurns; ++u) {
                const bool live = g < grids && u < turns;
                st.guess[u][g] = live ? q.guess_codes[grid * 5 + u] : 0u;
                st.tiles[u][g] = live ? q.tiles[grid * 5 + u] : std::uint16_t{0};
            }
        }
        for (int idx = tid; idx < kScratchFloats / 4; idx += kEvalThreads) {
            const float b = H2F(gh, kTrB1 + (idx * 4) / kChunkGames);
            reinterpret_cast<float4 *>(scratch)[idx] = make_float4(b, b, b, b);
        }
        __syncthreads();
        for (int u = 0; u < turns; ++u) {
            EncodeRound(st, gh, arena, scratch, u);
        }
        TrunkForward(p, st, gh, arena, scratch, turns, 0, 0);
        ScoreFp32(p, st, gh, arena, turns);
        if (tid < grids) {
            const int g = tid;
            const int a = st.best[g];
            float s = 0.0f;
            if (a >= 0) {
                for (int k = 0; k < 64; ++k) {
                    const float e = k < kFixedDim ? p.fixed_t[static_cast<std::size_t>(k) * p.action_pad + a]
                                                  : __half2float(tail[static_cast<std::size_t>(a) * kTailDim +
                                                                      (k - kFixedDim)]);
                    s = __fmaf_rn(arena[k * kLd + g], e, s);
                }
            }
            const std::uint32_t grid = q.order[begin + g];
            q.best_index[grid] = a;
            q.best_score[grid] = s;
        }
        __syncthreads();
    }
}

// Behavioural descriptors of a brood: each genome's policy on the 128 probe states, all in one chunk although the
// probes have 0..4 turns (EncodeRound<true> appends zeros for absent turns; a virgin probe's layer-1 chains start
// from the bias plus its virgin-flag weight, which is what the t = 0 path of TrunkForward computes). The probes'
// guesses and tiles are loaded once per CTA; each genome then costs four encode rounds and one trunk pass.
__global__ void __launch_bounds__(kEvalThreads, 2) DescriptorKernel(const DescriptorParams q) {
    extern __shared__ __align__(16) float arena[];
    __shared__ ChunkState st;
    const int tid = threadIdx.x;
    EvalParams p{};  // no trace
    float *scratch = q.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats;
    if (tid < kProbeStates) {
        st.turns[tid] = q.probe_turns[tid];
        for (int u = 0; u < kMaxTurns; ++u) {
            const bool live = u < kProbeMaxTurns && u < q.probe_turns[tid];
            st.guess[u][tid] = live ? q.probe_codes[tid * kProbeMaxTurns + u] : 0u;
            st.tiles[u][tid] = live ? q.probe_tiles[tid * kProbeMaxTurns + u] : std::uint16_t{0};
        }
    }
    __syncthreads();
    for (std::uint32_t g = blockIdx.x; g < q.count; g += gridDim.x) {
        const __half *gh = reinterpret_cast<const __half *>(q.slab + static_cast<std::size_t>(q.slots[g]) * q.pitch);
        for (int idx = tid; idx < kScratchFloats; idx += kEvalThreads) {
            const int o = idx / kChunkGames;
            const int probe = idx - o * kChunkGames;
            const float b = H2F(gh, kTrB1 + o);
            scratch[idx] = st.turns[probe] == 0 ? __fmaf_rn(H2F(gh, kTrW1 + o * kModelInput), 1.0f, b) : b;
        }
        __syncthreads();
        for (int u = 0; u < kProbeMaxTurns; ++u) {
            EncodeRound<true>(st, gh, arena, scratch, u);
        }
        TrunkForward(p, st, gh, arena, scratch, 1, 0, 0);
        std::uint16_t *row = q.out + static_cast<std::size_t>(g) * q.out_ld;
        for (int idx = tid; idx < kDescriptorWidth / 2; idx += kEvalThreads) {
            const int probe = (2 * idx) >> 6;
            const int k = (2 * idx) & 63;
            const __nv_bfloat162 v = __floats2bfloat162_rn(arena[k * kLd + probe] * q.scale,
                                                           arena[(k + 1) * kLd + probe] * q.scale);
            reinterpret_cast<__nv_bfloat162 *>(row)[idx] = v;
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t LaunchDescriptors(const DescriptorParams &params, int cta_count, cudaStream_t stream) {
    static std::atomic<unsigned long long> configured{0};
    if (const cudaError_t e =
            RaiseSharedLimit(DescriptorKernel, kArenaFloats * static_cast<int>(sizeof(float)), configured);
        e != cudaSuccess) {
        return e;
    }
    if (cta_count <= 0 || params.count == 0) {
        return cudaSuccess;
    }
    DescriptorKernel<<<cta_count, kEvalThreads, kArenaFloats * sizeof(float), stream>>>(params);
    return cudaGetLastError();
}

cudaError_t LaunchSingleModelSelect(const SingleModelParams &params, int cta_count, cudaStream_t stream) {
    static std::atomic<unsigned long long> configured{0};
    if (const cudaError_t e =
            RaiseSharedLimit(SingleModelSelectKernel, kArenaFloats * static_cast<int>(sizeof(float)), configured);
        e != cudaSuccess) {
        return e;
    }
    if (cta_count <= 0 || params.chunk_count <= 0) {
        return cudaSuccess;
    }
    SingleModelSelectKernel<<<cta_count, kEvalThreads, kArenaFloats * sizeof(float), stream>>>(params);
    return cudaGetLastError();
}

std::size_t EvalScratchFloatsPerCta() { return kScratchFloats; }

int EvalCtaCount(std::uint32_t total_chunks) {
    static int sm_count = 0;
    if (sm_count == 0) {
        int device = 0;
        cudaGetDevice(&device);
        cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, device);
        if (sm_count <= 0) {
            sm_count = 148;
        }
    }
    const int resident = 2 * sm_count;
    return static_cast<int>(total_chunks < static_cast<std::uint32_t>(resident) ? total_chunks : resident);
}

cudaError_t LaunchEvalPrepare(const WordSource &source, std::uint32_t population, std::uint32_t catalog_count,
                              std::uint32_t *local_words, std::uint32_t *chunk_start, std::uint32_t *score_sum,
                              int *status, cudaStream_t stream) {
    EvalPrepareKernel<<<1, 1024, 0, stream>>>(source, population, catalog_count, local_words, chunk_start, score_sum,
                                              status);
    return cudaGetLastError();
}

cudaError_t LaunchEvalFp32(const EvalParams &params, int cta_count, cudaStream_t stream) {
    static std::atomic<unsigned long long> configured[2]{{0}, {0}};
    const int bytes = kArenaFloats * static_cast<int>(sizeof(float));
    if (const cudaError_t e = params.xt != nullptr ? RaiseSharedLimit(EvalFp32Kernel<true>, bytes, configured[1])
                                                   : RaiseSharedLimit(EvalFp32Kernel<false>, bytes, configured[0]);
        e != cudaSuccess) {
        return e;
    }
    if (cta_count <= 0) {
        return cudaSuccess;
    }
    if (params.xt != nullptr) {
        EvalFp32Kernel<true><<<cta_count, kEvalThreads, bytes, stream>>>(params);
    } else {
        EvalFp32Kernel<false><<<cta_count, kEvalThreads, bytes, stream>>>(params);
    }
    return cudaGetLastError();
}

cudaError_t LaunchFinalizeFitness(const std::uint32_t *score_sum, const std::uint32_t *local_words,
                                  std::uint32_t population, float *fitness, std::uint32_t *evaluation_counts,
                                  std::uint8_t *has_fitness, int *status, cudaStream_t stream) {
    FinalizeFitnessKernel<<<(population + 255) / 256, 256, 0, stream>>>(score_sum, local_words, population, fitness,
                                                                         evaluation_counts, has_fitness, status);
    return cudaGetLastError();
}

cudaError_t LaunchSummarize(const float *fitness, const std::uint8_t *has_fitness, const std::uint32_t *slots,
                            std::uint32_t population, SummaryDevice *out, int *status, cudaStream_t stream) {
    SummarizeKernel<<<1, 32, 0, stream>>>(fitness, has_fitness, slots, population, out, status);
    return cudaGetLastError();
}

}  // namespace nwg
