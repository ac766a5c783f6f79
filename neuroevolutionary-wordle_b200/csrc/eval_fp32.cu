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
//
// Bit-exactness with the reference's device arithmetic: each output is the same chain of fused
// multiply-adds in the same input order as the reference's `sum += w * x` loops (bias first, inputs
// ascending). Terms whose input is exactly zero (empty turn slots, one-hot zeros) change a chain only
// in the sign of a zero result, which no comparison can see, so the encoder's one-hot layer is a gather
// and the trunk's first layer keeps its running accumulator from turn to turn (a new turn appends
// its 64 inputs to the end of the chain). Ties in the argmax go to the lowest action index, and
// guessed words are masked by word equality, as in the reference.
#include <cuda_fp16.h>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

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

// acc[i][j] = fma(A[k][row i], B[k][col j], acc[i][j]) for k = 0..K-1 in ascending order.
template <int TN>
__device__ __forceinline__ void MmaChain(float (&acc)[8][TN], const float *As, const float *Bs, int ldb, int K,
                                         int ty, int tx) {
#pragma unroll 4
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
__device__ bool ShardCovers(const ShardRecord &s, std::uint32_t rows, std::uint32_t cols, std::uint32_t cell) {
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
__device__ std::uint32_t ResolveWord(const WordSource &src, std::uint32_t cell, std::uint32_t j) {
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

__device__ std::uint32_t CountWords(const WordSource &src, std::uint32_t cell) {
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
        const std::uint32_t w = CountWords(src, i);
        local_words[i] = w;
        score_sum[i] = 0;
        if (w == 0) {
            SetStatus(status, kInvalidTrainingShard);
        }
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

__global__ void __launch_bounds__(kEvalThreads, 2) EvalFp32Kernel(const EvalParams p) {
    extern __shared__ __align__(16) float arena[];
    __shared__ ChunkState st;
    const int tid = threadIdx.x;
    const int ty = tid >> 4;
    const int tx = tid & 15;
    float *scratch = p.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats;
    unsigned long long decisions = 0;
    unsigned long long encoded = 0;
    unsigned long long episodes = 0;
    const std::uint32_t total_chunks = p.chunk_start[p.population];

    for (std::uint32_t chunk = blockIdx.x; chunk < total_chunks; chunk += gridDim.x) {
        // ---- chunk -> (individual, class, slice) ----
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
        if (st.stop) {
            break;
        }
        const int cls = st.cls;
        const std::uint32_t ind = static_cast<std::uint32_t>(st.individual);
        const std::uint32_t w = static_cast<std::uint32_t>(st.cell_words);
        const __half *gh = reinterpret_cast<const __half *>(p.slab + static_cast<std::size_t>(st.slot) * p.pitch);

        // ---- episode set-up (evaluation_ops.cuh:203-237) ----
        if (tid < kChunkGames) {
            const int g = tid;
            st.episode[g] = -1;
            st.turns[g] = 0;
            st.done[g] = 1;
            st.won[g] = 0;
            for (int t = 0; t < kMaxTurns; ++t) {
                st.choice[t][g] = -1;
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
        // layer-1 accumulators start at the bias (the virgin-flag term of a non-virgin state adds a zero)
        for (int idx = tid; idx < kScratchFloats / 4; idx += kEvalThreads) {
            const int o = (idx * 4) / kChunkGames;
            const float b = H2F(gh, kTrB1 + o);
            reinterpret_cast<float4 *>(scratch)[idx] = make_float4(b, b, b, b);
        }
        __syncthreads();

        // ---- one encoder round: encode turn t of every game and append it to the layer-1 chains ----
        auto encode_round = [&](int t) {
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
#pragma unroll
            for (int i = 0; i < 8; ++i) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    enc[(tx * 4 + j) * kLd + RowOf(ty, i)] = acc[i][j];
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
        };

        if (cls == 1) {
            if (tid == 0) {
                int active = 0;
                for (int g = 0; g < kChunkGames; ++g) {
                    active += st.done[g] == 0;
                }
                st.active = active;
            }
            __syncthreads();
            if (st.active > 0) {
                encode_round(0);
                encode_round(1);
                encoded += tid == 0 ? 2ull * st.active : 0ull;
            }
        }

        for (int step = 0; step < kMaxTurns; ++step) {
            if (tid == 0) {
                int active = 0;
                for (int g = 0; g < kChunkGames; ++g) {
                    active += st.done[g] == 0;
                }
                st.active = active;
            }
            __syncthreads();
            if (st.active == 0) {
                break;
            }
            const int t = cls == 0 ? step : step + 2;  // turns already on every active grid
            if (step > 0) {
                encode_round(t - 1);  // the turn appended by the previous decision
                encoded += tid == 0 ? static_cast<unsigned long long>(st.active) : 0ull;
            }

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
            for (int i = 0; i < 8; ++i) {
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float v = acc[i][j];
                    h1[ColOf8(tx, j) * kLd + RowOf(ty, i)] = v < 0.0f ? 0.0f : v;
                }
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
            for (int i = 0; i < 8; ++i) {
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    pv[(tx * 4 + j) * kLd + RowOf(ty, i)] = pacc[i][j];
                }
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

            // ---- scoring and masked argmax over the action space ----
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

            // ---- append the chosen guess (wordle_grid.hpp:69-77) ----
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
                    st.turns[g] = static_cast<std::uint8_t>(turn + 1);
                    const bool won = code == st.secret[g];
                    st.won[g] = won ? 1 : 0;
                    st.done[g] = (won || turn + 1 >= kMaxTurns) ? 1 : 0;
                    ++decisions;
                }
            }
            __syncthreads();
        }

        // ---- episode scores (evaluation_ops.cuh:239-242), summed exactly as integers ----
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
            for (int off = 16; off > 0; off >>= 1) {
                score += __shfl_xor_sync(0xffffffffu, score, off);
            }
            if ((tid & 31) == 0 && score != 0) {
                atomicAdd(p.score_sum + ind, score);
            }
        }
        __syncthreads();
    }
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

}  // namespace

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
    static bool configured = false;
    if (!configured) {
        cudaError_t e = cudaFuncSetAttribute(EvalFp32Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kArenaFloats * static_cast<int>(sizeof(float)));
        if (e != cudaSuccess) {
            return e;
        }
        configured = true;
    }
    if (cta_count <= 0) {
        return cudaSuccess;
    }
    EvalFp32Kernel<<<cta_count, kEvalThreads, kArenaFloats * sizeof(float), stream>>>(params);
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
