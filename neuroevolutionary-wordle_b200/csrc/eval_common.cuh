// Device functions shared by the evaluation kernels (plain FP32 form and tensor-core scoring form).
//
// A CTA of kEvalThreads threads owns a chunk of up to 128 games of one individual that share a turn count
// and plays them in lockstep (see eval_fp32.cu for the arithmetic contract). These functions are the
// phases of one chunk: mapping a chunk id to its individual, episode set-up, the encoder round for a new
// turn with the layer-1 chain extension, trunk layers 2 and 3, appending the chosen guesses and summing
// the episode scores. The scoring phase is the kernels' own.
#pragma once

#include <cuda_fp16.h>

#include "nwg_internal.cuh"

namespace nwg {
namespace evalx {

constexpr int kLd = 132;                 // leading dimension of 128-wide operand tiles (floats)
constexpr int kLd64 = 68;                // leading dimension of 64-wide operand tiles
constexpr int kTile = 64 * kLd;          // one 64 x 128 operand tile: 8,448 floats
constexpr int kArenaFloats = 3 * kTile;  // 101,376 bytes of dynamic shared memory
constexpr int kWsLd = 130;               // halfs per row of the staged encoder input weights
constexpr int kWsFloats = 9428;          // 145 x 130 halfs, rounded up to 16 bytes (in floats)
constexpr int kScratchFloats = kHidden0 * kChunkGames;  // layer-1 accumulators, [256 outputs][128 games]

struct ChunkState {
    std::uint32_t secret[kChunkGames];
    std::uint32_t guess[kMaxTurns][kChunkGames];
    std::uint16_t tiles[kMaxTurns][kChunkGames];
    std::int16_t choice[kMaxTurns][kChunkGames];
    std::int16_t word_index[kMaxTurns][kChunkGames];  // catalog index of each turn's word
    std::int32_t episode[kChunkGames];
    std::int32_t best[kChunkGames];
    std::uint8_t turns[kChunkGames];
    std::uint8_t done[kChunkGames];
    std::uint8_t won[kChunkGames];
    std::uint32_t tile_codes[2][128];
    int individual;
    int cls;  // 0: fresh games, 1: prefilled games
    int slice;
    int cell_words;
    int active;
    int stop;
    std::uint32_t slot;
};

__device__ __forceinline__ float H2F(const __half *p, int i) { return __half2float(p[i]); }

__device__ __forceinline__ int RowOf(int ty, int i) { return i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4); }
__device__ __forceinline__ int ColOf8(int tx, int j) { return j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4); }

// A thread's eight rows RowOf(ty, 0..7) of one column (col = the column's start, 16-byte aligned) as two 16-byte
// stores: rows 4 ty .. 4 ty + 3 and 64 + 4 ty .. 64 + 4 ty + 3.
__device__ __forceinline__ void StoreRows8(float *col, int ty, const float (&v)[8]) {
    *reinterpret_cast<float4 *>(col + ty * 4) = make_float4(v[0], v[1], v[2], v[3]);
    *reinterpret_cast<float4 *>(col + 64 + ty * 4) = make_float4(v[4], v[5], v[6], v[7]);
}

// acc[i][j] = fma(A[k][row i], B[k][col j], acc[i][j]) for k = 0..K-1 in ascending order.
template <int TN>
__device__ __forceinline__ void MmaChain(float (&acc)[8][TN], const float *As, const float *Bs, int ldb, int K,
                                         int ty, int tx) {
#pragma unroll 2
    for (int k = 0; k < K; ++k) {
        const float4 a0 = *reinterpret_cast<const float4 *>(As + k * kLd + ty * 4);
        const float4 a1 = *reinterpret_cast<const float4 *>(As + k * kLd + 64 + ty * 4);
        const float a[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
        float b[TN];
        const float4 b0 = *reinterpret_cast<const float4 *>(Bs + k * ldb + tx * 4);
        b[0] = b0.x;
        b[1] = b0.y;
        b[2] = b0.z;
        b[3] = b0.w;
        if constexpr (TN == 8) {
            const float4 b1 = *reinterpret_cast<const float4 *>(Bs + k * ldb + 64 + tx * 4);
            b[4] = b1.x;
            b[5] = b1.y;
            b[6] = b1.z;
            b[7] = b1.w;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
#pragma unroll
            for (int j = 0; j < TN; ++j) {
                acc[i][j] = __fmaf_rn(a[i], b[j], acc[i][j]);
            }
        }
    }
}

// training_data.hpp:135-143 + :208-223
__device__ inline bool ShardCovers(const ShardRecord &s, std::uint32_t rows, std::uint32_t cols, std::uint32_t cell) {
    if (s.word_count == 0 || s.first_catalog_word_index >= kCatalogCapacity ||
        s.word_count > kCatalogCapacity - s.first_catalog_word_index) {
        return false;
    }
    if (!s.global_from_outset && (s.center_row >= rows || s.center_column >= cols)) {
        return false;
    }
    if (cell >= rows * cols) {
        return false;
    }
    if (s.global_from_outset) {
        return true;
    }
    auto axis = [](std::uint64_t a, std::uint64_t b, std::uint64_t side) {
        const std::uint64_t f = a >= b ? a - b : b - a;
        const std::uint64_t w = side - f;
        return f < w ? f : w;
    };
    const std::uint64_t center = s.center_row * cols + s.center_column;
    const std::uint64_t dr = axis(center / cols, cell / cols, rows);
    const std::uint64_t dc = axis(center % cols, cell % cols, cols);
    return (dr > dc ? dr : dc) <= s.radius;
}

// Catalog index of the cell's local word j (evaluation_ops.cuh:143-169), or UINT32_MAX.
__device__ inline std::uint32_t ResolveWord(const WordSource &src, std::uint32_t cell, std::uint32_t j) {
    if (src.mode == 0) {
        return src.cell_words[src.cell_offsets[cell] + j];
    }
    std::uint64_t remaining = j;
    for (std::uint32_t s = 0; s < src.shard_count; ++s) {
        const ShardRecord &rec = src.shards[s];
        if (!ShardCovers(rec, src.rows, src.cols, cell)) {
            continue;
        }
        if (remaining < rec.word_count) {
            return static_cast<std::uint32_t>(rec.first_catalog_word_index + remaining);
        }
        remaining -= rec.word_count;
    }
    return 0xFFFFFFFFu;
}

__device__ inline std::uint32_t CountWords(const WordSource &src, std::uint32_t cell) {
    if (src.mode == 0) {
        return src.cell_offsets[cell + 1] - src.cell_offsets[cell];
    }
    std::uint64_t n = 0;
    for (std::uint32_t s = 0; s < src.shard_count; ++s) {
        if (ShardCovers(src.shards[s], src.rows, src.cols, cell)) {
            n += src.shards[s].word_count;
        }
    }
    return static_cast<std::uint32_t>(n);
}

__device__ __forceinline__ std::uint32_t ChunksForWords(std::uint32_t w) {
    return (w + kChunkGames - 1) / kChunkGames + (2 * w + kChunkGames - 1) / kChunkGames;
}

// Maps `chunk` to (individual, class, slice) in st; returns false (for every thread) when a failure was
// recorded and the kernel must stop.
__device__ __forceinline__ bool BeginChunk(const EvalParams &p, ChunkState &st, std::uint32_t chunk) {
    const int tid = threadIdx.x;
    if (tid == 0) {
        std::uint32_t lo = 0, hi = p.population;  // last i with chunk_start[i] <= chunk
        while (hi - lo > 1) {
            const std::uint32_t mid = (lo + hi) / 2;
            if (p.chunk_start[mid] <= chunk) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const std::uint32_t w = p.local_words[lo];
        const std::uint32_t local = chunk - p.chunk_start[lo];
        const std::uint32_t fresh_chunks = (w + kChunkGames - 1) / kChunkGames;
        st.individual = static_cast<int>(lo);
        st.cls = local < fresh_chunks ? 0 : 1;
        st.slice = static_cast<int>(local < fresh_chunks ? local : local - fresh_chunks);
        st.cell_words = static_cast<int>(w);
        st.slot = p.slot_of_individual[lo];
        st.stop = *reinterpret_cast<volatile int *>(p.status) != 0;
    }
    __syncthreads();
    return !st.stop;
}

// Episode set-up (evaluation_ops.cuh:203-237) and layer-1 accumulators initialised to the bias.
__device__ __forceinline__ void SetupGames(const EvalParams &p, ChunkState &st, const __half *gh, float *scratch) {
    const int tid = threadIdx.x;
    const int cls = st.cls;
    const std::uint32_t ind = static_cast<std::uint32_t>(st.individual);
    const std::uint32_t w = static_cast<std::uint32_t>(st.cell_words);
    if (tid < kChunkGames) {
        const int g = tid;
        st.episode[g] = -1;
        st.turns[g] = 0;
        st.done[g] = 1;
        st.won[g] = 0;
        for (int t = 0; t < kMaxTurns; ++t) {
            st.choice[t][g] = -1;
            st.word_index[t][g] = -1;
            st.guess[t][g] = 0;
            st.tiles[t][g] = 0;
        }
        const std::uint32_t q = static_cast<std::uint32_t>(st.slice) * kChunkGames + g;
        const bool valid = cls == 0 ? q < w : q < 2 * w;
        if (valid) {
            const std::uint32_t entry = cls == 0 ? q : q / 2;
            const std::uint32_t episode = cls == 0 ? 3 * q : 3 * (q / 2) + 1 + (q % 2);
            const std::uint32_t si = ResolveWord(p.source, ind, entry);
            int error = 0;
            if (si >= p.catalog_count) {
                error = kInvalidTrainingShard;
            } else {
                const std::uint32_t secret = p.codes[si];
                st.secret[g] = secret;
                int turns = 0;
                bool won = false;
                if (cls == 1) {
                    const std::uint32_t first = entry + ((q % 2) == 0 ? 1 : 3);
                    for (int k = 0; k < 2 && error == 0; ++k) {
                        const std::uint32_t wi = ResolveWord(p.source, ind, (first + k) % w);
                        if (wi >= p.catalog_count) {
                            error = kInvalidTrainingShard;
                        } else if (won) {
                            error = kGuessAppendFailed;  // wordle_grid.hpp:69-77 rejects a finished grid
                        } else {
                            const std::uint32_t code = p.codes[wi];
                            st.guess[turns][g] = code;
                            st.tiles[turns][g] = static_cast<std::uint16_t>(FeedbackPacked(code, secret));
                            st.word_index[turns][g] = static_cast<std::int16_t>(wi);
                            ++turns;
                            won = code == secret;
                        }
                    }
                }
                st.turns[g] = static_cast<std::uint8_t>(turns);
                st.won[g] = won ? 1 : 0;
                st.done[g] = won ? 1 : 0;
                st.episode[g] = static_cast<std::int32_t>(episode);
            }
            if (error != 0) {
                SetStatus(p.status, error);
                st.done[g] = 1;
            }
        }
    }
    // layer-1 accumulators start at the bias (the virgin-flag term of a non-virgin state adds a zero);
    // a form that keeps no FP32 layer-1 accumulators passes no scratch
    for (int idx = tid; scratch != nullptr && idx < kScratchFloats / 4; idx += kEvalThreads) {
        const int o = (idx * 4) / kChunkGames;
        const float b = H2F(gh, kTrB1 + o);
        reinterpret_cast<float4 *>(scratch)[idx] = make_float4(b, b, b, b);
    }
    __syncthreads();
}

__device__ __forceinline__ int CountActive(ChunkState &st) {
    if (threadIdx.x == 0) {
        int active = 0;
        for (int g = 0; g < kChunkGames; ++g) {
            active += st.done[g] == 0;
        }
        st.active = active;
    }
    __syncthreads();
    return st.active;
}

// Encodes turn t of every game (10-column gather, ReLU, 128 -> 64) and appends its 64 inputs to the
// layer-1 chains held in scratch ([256 outputs][128 games]). With kMaskByTurns the games of a chunk may have
// different turn counts (st.turns): a game without turn t appends zeros, which leaves its chains unchanged.
template <bool kMaskByTurns = false>
__device__ __forceinline__ void EncodeRound(ChunkState &st, const __half *gh, float *arena, float *scratch, int t) {
    const int tid = threadIdx.x;
    const int ty = tid >> 4;
    const int tx = tid & 15;
    __half *ws = reinterpret_cast<__half *>(arena);  // [145][kWsLd] encoder input weights
    float *ah = arena + kWsFloats;                     // [64][kLd] encoder hidden half
    float *be = arena + kWsFloats + kTile;             // [64][kLd64] encoder output weights half
    for (int idx = tid; idx < kEncoderHidden * kTurnFeatures; idx += kEvalThreads) {
        const int o = idx / kTurnFeatures;
        const int f = idx - o * kTurnFeatures;
        ws[f * kWsLd + o] = gh[kEncW1 + idx];
    }
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float b = H2F(gh, kEncB2 + tx * 4 + j);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            acc[i][j] = b;
        }
    }
    for (int half = 0; half < 2; ++half) {
        __syncthreads();
        // hidden[o] = relu(b1[o] + w[o][letter features] + w[o][tile features]) in ascending feature order
        const int ol = tid & 63;
        const int o = half * 64 + ol;
        const float bias = H2F(gh, kEncB1 + o);
        for (int g = tid >> 6; g < kChunkGames; g += 4) {
            const std::uint32_t code = st.guess[t][g];
            const std::uint32_t tiles = st.tiles[t][g];
            float h = bias;
#pragma unroll
            for (int pos = 0; pos < kWordLength; ++pos) {
                h = __fmaf_rn(__half2float(ws[(pos * kAlphabet + WordLetter(code, pos)) * kWsLd + o]), 1.0f, h);
            }
#pragma unroll
            for (int pos = 0; pos < kWordLength; ++pos) {
                const int f = kWordLength * kAlphabet + pos * 3 + ((tiles >> (2 * pos)) & 3);
                h = __fmaf_rn(__half2float(ws[f * kWsLd + o]), 1.0f, h);
            }
            ah[ol * kLd + g] = h < 0.0f ? 0.0f : h;
        }
        for (int idx = tid; idx < 64 * 64; idx += kEvalThreads) {
            const int oo = idx >> 6;
            const int k = idx & 63;
            be[k * kLd64 + oo] = H2F(gh, kEncW2 + oo * kEncoderHidden + half * 64 + k);
        }
        __syncthreads();
        MmaChain<4>(acc, ah, be, kLd64, 64, ty, tx);
    }
    __syncthreads();
    float *enc = arena;  // [64][kLd] encoded turn, k-major
    {
        bool live[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            live[i] = !kMaskByTurns || t < st.turns[RowOf(ty, i)];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                v[i] = live[i] ? acc[i][j] : 0.0f;
            }
            StoreRows8(enc + (tx * 4 + j) * kLd, ty, v);
        }
    }
    // trunk layer 1: chains continue with inputs 1 + 64t .. 64 + 64t
    float *bw = arena + kTile;  // [64][kLd]
    for (int nh = 0; nh < 2; ++nh) {
        __syncthreads();
        for (int idx = tid; idx < 128 * 64; idx += kEvalThreads) {
            const int n = idx >> 6;
            const int k = idx & 63;
            bw[k * kLd + n] = H2F(gh, kTrW1 + (nh * 128 + n) * kModelInput + 1 + 64 * t + k);
        }
        float a1[8][8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int o = nh * 128 + ColOf8(tx, j);
#pragma unroll
            for (int i2 = 0; i2 < 2; ++i2) {
                const float4 v = *reinterpret_cast<const float4 *>(scratch + o * kChunkGames + i2 * 64 + ty * 4);
                a1[i2 * 4 + 0][j] = v.x;
                a1[i2 * 4 + 1][j] = v.y;
                a1[i2 * 4 + 2][j] = v.z;
                a1[i2 * 4 + 3][j] = v.w;
            }
        }
        __syncthreads();
        MmaChain<8>(a1, enc, bw, kLd, 64, ty, tx);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int o = nh * 128 + ColOf8(tx, j);
#pragma unroll
            for (int i2 = 0; i2 < 2; ++i2) {
                *reinterpret_cast<float4 *>(scratch + o * kChunkGames + i2 * 64 + ty * 4) =
                    make_float4(a1[i2 * 4 + 0][j], a1[i2 * 4 + 1][j], a1[i2 * 4 + 2][j], a1[i2 * 4 + 3][j]);
            }
        }
    }
    __syncthreads();
}

// Trunk layers 2 and 3 for every game at turn count t; leaves the FP32 policy vectors in
// arena[0 .. kTile) as [64 k][kLd games] and records them in the trace when one is requested.
__device__ __forceinline__ void TrunkForward(const EvalParams &p, ChunkState &st, const __half *gh, float *arena,
                                             const float *scratch, int t, int step, std::uint32_t ind) {
    const int tid = threadIdx.x;
    const int ty = tid >> 4;
    const int tx = tid & 15;
    // ---- trunk layer 2: h1 = relu(b2 + W2 . relu(layer-1)) ----
    float acc[8][8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const float b = H2F(gh, kTrB2 + ColOf8(tx, j));
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            acc[i][j] = b;
        }
    }
    float *as = arena;
    float *bs = arena + kTile;
    for (int kc = 0; kc < 4; ++kc) {
        __syncthreads();
        if (t == 0) {
            for (int idx = tid; idx < 64 * kChunkGames; idx += kEvalThreads) {
                const int k = idx >> 7;
                const int g = idx & 127;
                const int o = kc * 64 + k;
                const float v = __fmaf_rn(H2F(gh, kTrW1 + o * kModelInput), 1.0f, H2F(gh, kTrB1 + o));
                as[k * kLd + g] = v < 0.0f ? 0.0f : v;
            }
        } else {
            for (int idx = tid; idx < 64 * kChunkGames / 4; idx += kEvalThreads) {
                const int k = idx >> 5;
                const int g4 = (idx & 31) * 4;
                float4 v = *reinterpret_cast<const float4 *>(scratch + (kc * 64 + k) * kChunkGames + g4);
                v.x = v.x < 0.0f ? 0.0f : v.x;
                v.y = v.y < 0.0f ? 0.0f : v.y;
                v.z = v.z < 0.0f ? 0.0f : v.z;
                v.w = v.w < 0.0f ? 0.0f : v.w;
                *reinterpret_cast<float4 *>(as + k * kLd + g4) = v;
            }
        }
        for (int idx = tid; idx < 128 * 64; idx += kEvalThreads) {
            const int n = idx >> 6;
            const int k = idx & 63;
            bs[k * kLd + n] = H2F(gh, kTrW2 + n * kHidden0 + kc * 64 + k);
        }
        __syncthreads();
        MmaChain<8>(acc, as, bs, kLd, 64, ty, tx);
    }
    __syncthreads();
    float *h1 = arena;  // [128][kLd]
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            v[i] = acc[i][j] < 0.0f ? 0.0f : acc[i][j];
        }
        StoreRows8(h1 + ColOf8(tx, j) * kLd, ty, v);
    }

    // ---- trunk layer 3: policy = b3 + W3 . h1 ----
    float pacc[8][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float b = H2F(gh, kTrB3 + tx * 4 + j);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            pacc[i][j] = b;
        }
    }
    float *b3 = arena + 2 * kTile;  // [64][kLd64]
    for (int kh = 0; kh < 2; ++kh) {
        __syncthreads();
        for (int idx = tid; idx < 64 * 64; idx += kEvalThreads) {
            const int n = idx >> 6;
            const int k = idx & 63;
            b3[k * kLd64 + n] = H2F(gh, kTrW3 + n * kHidden1 + kh * 64 + k);
        }
        __syncthreads();
        MmaChain<4>(pacc, h1 + kh * 64 * kLd, b3, kLd64, 64, ty, tx);
    }
    __syncthreads();
    float *pv = arena;  // [64][kLd] policy vectors, k-major
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        float v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            v[i] = pacc[i][j];
        }
        StoreRows8(pv + (tx * 4 + j) * kLd, ty, v);
    }
    __syncthreads();
    if (p.trace_policy != nullptr) {
        for (int idx = tid; idx < kChunkGames * kPolicy; idx += kEvalThreads) {
            const int g = idx >> 6;
            const int k = idx & 63;
            const std::int32_t e = st.episode[g];
            if (!st.done[g] && e >= 0 && static_cast<std::uint32_t>(e) < p.trace_episodes) {
                const std::size_t slot = static_cast<std::size_t>(ind) * p.trace_episodes + e;
                p.trace_policy[(slot * kMaxTurns + step) * kPolicy + k] = pv[k * kLd + g];
            }
        }
    }

}

// Appends each active game's chosen guess st.best[g] (wordle_grid.hpp:69-77).
__device__ __forceinline__ void AppendGuesses(const EvalParams &p, ChunkState &st, int step,
                                              unsigned long long &decisions) {
    const int tid = threadIdx.x;
    if (tid < kChunkGames && !st.done[tid]) {
        const int g = tid;
        const int choice = st.best[g];
        if (choice < 0) {
            SetStatus(p.status, kActionSelectionFailed);
            st.done[g] = 1;
        } else {
            const std::uint32_t code = p.codes[choice];
            const int turn = st.turns[g];
            st.guess[turn][g] = code;
            st.tiles[turn][g] = static_cast<std::uint16_t>(FeedbackPacked(code, st.secret[g]));
            st.choice[step][g] = static_cast<std::int16_t>(choice);
            st.word_index[turn][g] = static_cast<std::int16_t>(choice);
            st.turns[g] = static_cast<std::uint8_t>(turn + 1);
            const bool won = code == st.secret[g];
            st.won[g] = won ? 1 : 0;
            st.done[g] = (won || turn + 1 >= kMaxTurns) ? 1 : 0;
            ++decisions;
        }
    }
    __syncthreads();
}

// Episode scores (evaluation_ops.cuh:239-242), summed exactly as integers, and the trace.
__device__ __forceinline__ void FinishChunk(const EvalParams &p, ChunkState &st, std::uint32_t ind,
                                            unsigned long long &episodes) {
    const int tid = threadIdx.x;
    if (tid < kChunkGames) {
        const int g = tid;
        episodes += st.episode[g] >= 0 ? 1ull : 0ull;
        std::uint32_t score = 0;
        if (st.episode[g] >= 0 && st.won[g]) {
            score = 10u + static_cast<std::uint32_t>(kMaxTurns - st.turns[g]);
        }
        const std::int32_t e = st.episode[g];
        if (e >= 0 && static_cast<std::uint32_t>(e) < p.trace_episodes) {
            const std::size_t slot = static_cast<std::size_t>(ind) * p.trace_episodes + e;
            if (p.trace_scores != nullptr) {
                p.trace_scores[slot] = static_cast<float>(score);
            }
            if (p.trace_turns != nullptr) {
                p.trace_turns[slot] = st.turns[g];
            }
            if (p.trace_choices != nullptr) {
                for (int s = 0; s < kMaxTurns; ++s) {
                    p.trace_choices[slot * kMaxTurns + s] = st.choice[s][g];
                }
            }
        }
        std::uint32_t won = st.episode[g] >= 0 && st.won[g] ? 1u : 0u;
        for (int off = 16; off > 0; off >>= 1) {
            score += __shfl_xor_sync(0xffffffffu, score, off);
            won += __shfl_xor_sync(0xffffffffu, won, off);
        }
        if ((tid & 31) == 0 && score != 0) {
            atomicAdd(p.score_sum + ind, score);
        }
        if ((tid & 31) == 0 && won != 0 && p.won_sum != nullptr) {
            atomicAdd(p.won_sum + ind, won);
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void FlushCounters(const EvalParams &p, unsigned long long decisions,
                                              unsigned long long encoded, unsigned long long episodes) {
    const int tid = threadIdx.x;
    for (int off = 16; off > 0; off >>= 1) {
        decisions += __shfl_xor_sync(0xffffffffu, decisions, off);
        encoded += __shfl_xor_sync(0xffffffffu, encoded, off);
        episodes += __shfl_xor_sync(0xffffffffu, episodes, off);
    }
    if ((tid & 31) == 0) {
        if (decisions != 0) {
            atomicAdd(p.steps, decisions);
        }
        if (encoded != 0) {
            atomicAdd(p.steps + 1, encoded);
        }
        if (episodes != 0) {
            atomicAdd(p.steps + 2, episodes);
        }
    }
}


}  // namespace evalx
}  // namespace nwg
