// The exact FP32 encoder and trunk with streamed weights: the plain and the exact tensor-core-screened forms' policy
// path when a per-individual FP32 weight table is available.
//
// Every output is the same chain of fused multiply-adds, in the same input order, as eval_common.cuh's EncodeRound
// and TrunkForward (and the reference's dense_trunk.hpp:46-54: bias first, inputs ascending), so the results are
// bit-identical; only where the operands come from changes. Instead of restaging every weight block from the FP16
// genome with scalar loads and transposing stores between two barriers, each step streams the weights from a table
// built once per evaluation (BuildExactTrunkTables) that already holds them as FP32 in the [input][output] order the
// register-tiled micro-kernel reads, with 16-byte cp.async copies into double-buffered shared-memory tiles: the copies
// of the next K-chunk fly while the current one is multiplied, and each K-chunk costs one barrier.
#pragma once

#include "eval_common.cuh"

namespace nwg {
namespace evalx {

// Per-individual exact trunk table (bytes), every block 256-byte aligned:
constexpr int kXtWe1 = 0;                                               // FP16 [145 features][128 outputs]
constexpr int kXtWe2 = kXtWe1 + kTurnFeatures * kEncoderHidden * 2;     // FP32 [128 in][64 out]
constexpr int kXtW1 = kXtWe2 + kEncoderHidden * kEncoderOut * 4;        // FP32 5 x [64 in][256 out] (turn slots)
constexpr int kXtW1Turn = kEncoderOut * kHidden0 * 4;
constexpr int kXtW2 = kXtW1 + 5 * kXtW1Turn;                            // FP32 [256 in][128 out]
constexpr int kXtW3 = kXtW2 + kHidden0 * kHidden1 * 4;                  // FP32 [128 in][64 out]
constexpr int kXtBytes = kXtW3 + kHidden1 * kPolicy * 4;
static_assert(kXtBytes == 561408 && kXtBytes % 256 == 0, "exact trunk table layout");
static_assert(kXtWe2 % 256 == 0 && kXtW1 % 256 == 0 && kXtW2 % 256 == 0 && kXtW3 % 256 == 0, "table blocks align");

// 16-byte asynchronous global -> shared copy (bypassing L1), and its group bookkeeping.
__device__ __forceinline__ void CopyAsync16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(static_cast<std::uint32_t>(
                     __cvta_generic_to_shared(dst))),
                 "l"(src)
                 : "memory");
}
__device__ __forceinline__ void CopyAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void CopyAsyncWaitAll() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// rows x (cols floats, a multiple of 4) from global (row stride src_ld floats) to shared memory (row stride
// dst_ld floats), 16 bytes per copy, spread over the CTA. Returns nothing; the caller commits and waits.
__device__ __forceinline__ void CopyRowsAsync(float *dst, int dst_ld, const float *src, int src_ld, int rows,
                                              int cols) {
    const int per_row = cols / 4;
    for (int i = threadIdx.x; i < rows * per_row; i += kEvalThreads) {
        const int r = i / per_row;
        const int c = (i - r * per_row) * 4;
        CopyAsync16(dst + r * dst_ld + c, src + static_cast<std::size_t>(r) * src_ld + c);
    }
}

// acc[i][j] = fma(A[k][row i], B[k][col j], acc[i][j]) for k = 0..K-1 in ascending order (MmaChain with explicit
// leading dimensions): A is [K][128 games] with leading dimension lda, B is [K][8 * 16 or 4 * 16 outputs] with ldb.
template <int TN>
__device__ __forceinline__ void MmaChainLd(float (&acc)[8][TN], const float *As, int lda, const float *Bs, int ldb,
                                           int K, int ty, int tx) {
#pragma unroll 2
    for (int k = 0; k < K; ++k) {
        const float4 a0 = *reinterpret_cast<const float4 *>(As + k * lda + ty * 4);
        const float4 a1 = *reinterpret_cast<const float4 *>(As + k * lda + 64 + ty * 4);
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

__device__ __forceinline__ void CopyAsyncWaitAllButOne() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Shared-memory plan of the streamed encoder round (floats of the 25,344-float arena).
constexpr int kXeWs = 0;                 // W_e1 as FP16 [145 features][128 outputs]
constexpr int kXeBe = 9280;              // W_e2 [128 in][64 out]
constexpr int kXeAh = kXeBe + 8192;      // one quarter of the hidden layer, [32][kLd] (games)
constexpr int kXeEnc = 0;                // the encoded turn, [64][kLd] (after the encoder's last barrier)
constexpr int kXeB0 = kXeEnc + 64 * kLd;  // W1 slot of the turn, outputs 0-127: [64 in][128 out]
constexpr int kXeB1 = kXeB0 + 64 * 128;   // outputs 128-255
static_assert(kXeWs * 4 + kTurnFeatures * kEncoderHidden * 2 <= kXeBe * 4, "W_e1 before W_e2");
static_assert(kXeAh + 32 * kLd <= kArenaFloats && kXeB1 + 64 * 128 <= kArenaFloats, "encoder arena");

// EncodeRound with streamed weights (same chains, same order). xt is the individual's exact trunk table.
template <bool kMaskByTurns = false>
__device__ __forceinline__ void EncodeRoundX(ChunkState &st, const __half *gh, const std::uint8_t *xt, float *arena,
                                             float *scratch, int t) {
    const int tid = threadIdx.x;
    const int ty = tid >> 4;
    const int tx = tid & 15;
    __half *ws = reinterpret_cast<__half *>(arena + kXeWs);
    const float *be = arena + kXeBe;
    float *ah = arena + kXeAh;
    CopyRowsAsync(arena + kXeWs, 64, reinterpret_cast<const float *>(xt + kXtWe1), 64, kTurnFeatures, 64);
    CopyRowsAsync(arena + kXeBe, 64, reinterpret_cast<const float *>(xt + kXtWe2), 64, kEncoderHidden, 64);
    CopyAsyncCommit();
    float acc[8][4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float b = H2F(gh, kEncB2 + tx * 4 + j);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            acc[i][j] = b;
        }
    }
    // Each lane owns two adjacent hidden outputs of a quarter (one 4-byte read of W_e1 gives both) and a half-warp
    // one game, so a warp gathers two games at a time. Their biases are read while the weights stream in.
    const int pair = tid & 15;
    const int half_warp = (tid >> 4) & 1;
    float bias_q[4][2];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        bias_q[q][0] = H2F(gh, kEncB1 + q * 32 + 2 * pair);
        bias_q[q][1] = H2F(gh, kEncB1 + q * 32 + 2 * pair + 1);
    }
    CopyAsyncWaitAll();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        __syncthreads();
        // hidden[o] = relu(b1[o] + w[o][letter features] + w[o][tile features]) in ascending feature order
        const int o0 = q * 32 + 2 * pair;
        // Four games per pass (games 2 w + half, then + 16, + 32, + 48; then + 64 ...): their weight reads are
        // issued before any of the pass's stores, which the compiler could not move them past, and the eight
        // ten-add chains interleave.
        constexpr int kWarps = kEvalThreads / 32;
        for (int g0 = 2 * (tid >> 5) + half_warp; g0 < kChunkGames; g0 += 8 * kWarps) {
            float h[4][2];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int g = g0 + j * 2 * kWarps;
                const std::uint32_t code = st.guess[t][g];
                const std::uint32_t tiles = st.tiles[t][g];
                float h0 = bias_q[q][0];
                float h1 = bias_q[q][1];
#pragma unroll
                for (int pos = 0; pos < kWordLength; ++pos) {
                    const int f = pos * kAlphabet + static_cast<int>(WordLetter(code, pos));
                    const float2 w = __half22float2(*reinterpret_cast<const __half2 *>(ws + f * kEncoderHidden + o0));
                    h0 = __fmaf_rn(w.x, 1.0f, h0);
                    h1 = __fmaf_rn(w.y, 1.0f, h1);
                }
#pragma unroll
                for (int pos = 0; pos < kWordLength; ++pos) {
                    const int f = kWordLength * kAlphabet + pos * 3 + ((tiles >> (2 * pos)) & 3);
                    const float2 w = __half22float2(*reinterpret_cast<const __half2 *>(ws + f * kEncoderHidden + o0));
                    h0 = __fmaf_rn(w.x, 1.0f, h0);
                    h1 = __fmaf_rn(w.y, 1.0f, h1);
                }
                h[j][0] = h0;
                h[j][1] = h1;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int g = g0 + j * 2 * kWarps;
                ah[(2 * pair) * kLd + g] = h[j][0] < 0.0f ? 0.0f : h[j][0];
                ah[(2 * pair + 1) * kLd + g] = h[j][1] < 0.0f ? 0.0f : h[j][1];
            }
        }
        __syncthreads();
        MmaChainLd<4>(acc, ah, kLd, be + q * 32 * kEncoderOut, kEncoderOut, 32, ty, tx);
    }
    __syncthreads();
    // trunk layer 1: chains continue with inputs 1 + 64t .. 64 + 64t; both halves of the turn's W1 slot stream in
    // while the encoded turn is written and the accumulators are fetched
    const float *w1 = reinterpret_cast<const float *>(xt + kXtW1 + t * kXtW1Turn);
    CopyRowsAsync(arena + kXeB0, 128, w1, kHidden0, kEncoderOut, 128);
    CopyAsyncCommit();
    CopyRowsAsync(arena + kXeB1, 128, w1 + 128, kHidden0, kEncoderOut, 128);
    CopyAsyncCommit();
    float *enc = arena + kXeEnc;  // [64][kLd] encoded turn, k-major
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
    for (int nh = 0; nh < 2; ++nh) {
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
        if (nh == 0) {
            CopyAsyncWaitAllButOne();
        } else {
            CopyAsyncWaitAll();
        }
        __syncthreads();
        MmaChainLd<8>(a1, enc, kLd, arena + (nh == 0 ? kXeB0 : kXeB1), 128, kEncoderOut, ty, tx);
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

// Shared-memory plan of the streamed trunk (floats): layer 2 streams K-chunks of 32 inputs, A (the layer-1
// activations) and B (W2) double-buffered; W3 arrives with the first chunk; h1 and then the policy reuse the start.
constexpr int kXfKc = 32;
constexpr int kXfA0 = 0;
constexpr int kXfA1 = kXfA0 + kXfKc * 128;
constexpr int kXfB0 = kXfA1 + kXfKc * 128;
constexpr int kXfB1 = kXfB0 + kXfKc * 128;
constexpr int kXfW3 = kHidden1 * kLd;  // after h1 ([128][kLd])
constexpr int kXfVirgin = kXfB1 + kXfKc * 128;  // [256] layer-1 outputs with no turn, between B1 and W3
static_assert(kXfB1 + kXfKc * 128 <= kXfW3 && kXfW3 + kHidden1 * kPolicy <= kArenaFloats, "trunk arena");
static_assert(kXfVirgin + kHidden0 <= kXfW3, "the no-turn layer-1 outputs fit before W3");

// TrunkForward with streamed weights (same chains, same order): leaves the FP32 policy vectors in arena[0 .. kTile)
// as [64 k][kLd games] and records them in the trace when one is requested.
__device__ __forceinline__ void TrunkForwardX(const EvalParams &p, ChunkState &st, const __half *gh,
                                              const std::uint8_t *xt, float *arena, const float *scratch, int t,
                                              int step, std::uint32_t ind) {
    const int tid = threadIdx.x;
    const int ty = tid >> 4;
    const int tx = tid & 15;
    auto abuf = [&](int b) { return arena + kXfA0 + b * (kXfA1 - kXfA0); };
    auto bbuf = [&](int b) { return arena + kXfB0 + b * (kXfB1 - kXfB0); };
    const float *w2 = reinterpret_cast<const float *>(xt + kXtW2);
    auto issue = [&](int kc, int b) {
        if (t > 0) {  // layer-1 activations (before the ReLU) from the CTA's accumulators
            CopyRowsAsync(abuf(b), 128, scratch + kc * kXfKc * kChunkGames, kChunkGames, kXfKc, 128);
        }
        CopyRowsAsync(bbuf(b), 128, w2 + kc * kXfKc * kHidden1, kHidden1, kXfKc, 128);
        CopyAsyncCommit();
    };
    // layer 3's biases, read while layer 2 runs
    float b3[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        b3[j] = H2F(gh, kTrB3 + tx * 4 + j);
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
    CopyRowsAsync(arena + kXfW3, kPolicy, reinterpret_cast<const float *>(xt + kXtW3), kPolicy, kHidden1, kPolicy);
    issue(0, 0);
    // no turn on the board: every game's layer-1 output is relu(b1 + W1[:, 0]), one value per output
    float *virgin = arena + kXfVirgin;
    if (t == 0) {
        for (int o = tid; o < kHidden0; o += kEvalThreads) {
            const float v = __fmaf_rn(H2F(gh, kTrW1 + o * kModelInput), 1.0f, H2F(gh, kTrB1 + o));
            virgin[o] = v < 0.0f ? 0.0f : v;
        }
        __syncthreads();
    }
    constexpr int kChunks = kHidden0 / kXfKc;
    for (int kc = 0; kc < kChunks; ++kc) {
        const int b = kc & 1;
        CopyAsyncWaitAll();
        if (t > 0) {
            // the ReLU, by each thread on the 16-byte pieces it copied itself
            for (int i = tid; i < kXfKc * 32; i += kEvalThreads) {
                float4 *v = reinterpret_cast<float4 *>(abuf(b) + (i >> 5) * 128 + (i & 31) * 4);
                float4 x = *v;
                x.x = x.x < 0.0f ? 0.0f : x.x;
                x.y = x.y < 0.0f ? 0.0f : x.y;
                x.z = x.z < 0.0f ? 0.0f : x.z;
                x.w = x.w < 0.0f ? 0.0f : x.w;
                *v = x;
            }
        } else {
            for (int idx = tid; idx < kXfKc * kChunkGames; idx += kEvalThreads) {
                const int k = idx >> 7;
                abuf(b)[k * 128 + (idx & 127)] = virgin[kc * kXfKc + k];
            }
        }
        __syncthreads();
        if (kc + 1 < kChunks) {
            issue(kc + 1, b ^ 1);
        }
        MmaChainLd<8>(acc, abuf(b), 128, bbuf(b), 128, kXfKc, ty, tx);
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
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            pacc[i][j] = b3[j];
        }
    }
    __syncthreads();
    MmaChainLd<4>(pacc, h1, kLd, arena + kXfW3, kPolicy, kHidden1, ty, tx);
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

}  // namespace evalx
}  // namespace nwg
