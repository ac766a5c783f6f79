// Helpers shared by the tensor-core evaluation forms: ordered score keys, bulk copies into shared memory,
// per-thread top-4 chunk lists and the exact FP32 re-scoring of one 32-action chunk.
#pragma once

#include <cuda_fp16.h>

#include "eval_common.cuh"
#include "umma.cuh"

namespace nwg {
namespace tcx {

using namespace evalx;

constexpr int kTopK = 4;  // chunk maxima kept per thread (per game half)

__device__ __forceinline__ std::uint32_t OrderedBits(float f) {
    const std::uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float FromOrderedBits(std::uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// Larger key = larger score, then lower action index; 0 means "no action".
__device__ __forceinline__ unsigned long long PackKey(float score, std::uint32_t action) {
    return (static_cast<unsigned long long>(OrderedBits(score)) << 32) | (0xFFFFFFFFu - action);
}

__device__ __forceinline__ float KeyScore(unsigned long long key) {
    return FromOrderedBits(static_cast<std::uint32_t>(key >> 32));
}

__device__ __forceinline__ int KeyAction(unsigned long long key) {
    return static_cast<int>(0xFFFFFFFFu - static_cast<std::uint32_t>(key & 0xFFFFFFFFull));
}

// One bulk copy global -> shared memory, completing on `mbar` (which expects `bytes` more transaction bytes).
__device__ __forceinline__ void BulkLoad(void *dst, const void *src, std::uint32_t bytes, std::uint64_t *mbar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(umma::SmemAddress(mbar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            umma::SmemAddress(dst)),
        "l"(src), "r"(bytes), "r"(umma::SmemAddress(mbar))
        : "memory");
}

// Three-input maximum (one sm_100 instruction).
__device__ __forceinline__ float Max3(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Maximum of v[base .. base + 31] in 16 three-input steps.
__device__ __forceinline__ float Max32(const float (&v)[64], int base) {
    float m[12];
#pragma unroll
    for (int j = 0; j < 10; ++j) {
        m[j] = Max3(v[base + 3 * j], v[base + 3 * j + 1], v[base + 3 * j + 2]);
    }
    m[10] = v[base + 30];
    m[11] = v[base + 31];
    const float a = Max3(m[0], m[1], m[2]);
    const float b = Max3(m[3], m[4], m[5]);
    const float c = Max3(m[6], m[7], m[8]);
    const float d = Max3(m[9], m[10], m[11]);
    return fmaxf(Max3(a, b, c), d);
}

// Insert x (chunk id xi) into the descending list v[0..3].
__device__ __forceinline__ void InsertTop4(float (&v)[kTopK], int (&id)[kTopK], float x, int xi) {
#pragma unroll
    for (int j = 0; j < kTopK; ++j) {
        const bool c = x > v[j];
        const float tv = c ? v[j] : x;
        const int ti = c ? id[j] : xi;
        v[j] = c ? x : v[j];
        id[j] = c ? xi : id[j];
        x = tv;
        xi = ti;
    }
}

// Exact FP32 score of action a for the policy vector pv[k * ld] (the plain form's chain:
// output_embedding.hpp:98-119). All 64 embedding values are loaded before the chain starts.
__device__ __forceinline__ float ExactScore(const EvalParams &p, const float *pv, int ld, const __half *tail,
                                            std::uint32_t a) {
    float e[kPolicy];
#pragma unroll
    for (int k = 0; k < kFixedDim; ++k) {
        e[k] = p.fixed_t[static_cast<std::size_t>(k) * p.action_pad + a];
    }
    const __half2 *row = reinterpret_cast<const __half2 *>(tail + static_cast<std::size_t>(a) * kTailDim);
#pragma unroll
    for (int j = 0; j < kTailDim / 2; ++j) {
        const float2 f = __half22float2(row[j]);
        e[kFixedDim + 2 * j] = f.x;
        e[kFixedDim + 2 * j + 1] = f.y;
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kPolicy; ++k) {
        s = __fmaf_rn(pv[k * ld], e[k], s);
    }
    return s;
}

// Exact key of this lane's action in 32-action chunk `chunk` for game g, whose policy vector is pv[k * ld]: the
// packed (score, action) key, or 0 for a guessed word (word equality) or an action past the end. The score is
// formed before the mask is known, so the action's code and its embedding values are loaded together.
__device__ __forceinline__ unsigned long long ChunkKey(const EvalParams &p, const ChunkState &cs, const float *pv,
                                                       int ld, const __half *tail, int g, int chunk, int turns) {
    const std::uint32_t a = static_cast<std::uint32_t>(chunk) * 32u + (threadIdx.x & 31);
    if (a >= p.action_count) {
        return 0;
    }
    const std::uint32_t code = p.codes[a];
    const float s = ExactScore(p, pv, ld, tail, a);
    bool masked = false;
    for (int u = 0; u < turns; ++u) {
        masked |= cs.guess[u][g] == code;
    }
    return masked ? 0ull : PackKey(s, a);
}

// Action a's row of a 16-bit embedding table (64 values in eight 16-byte pieces of the K-major operand tile layout,
// 128 actions per 16 KB tile).
__device__ __forceinline__ void LoadEmbedRow(const std::uint8_t *embed, std::uint32_t a, uint4 (&e)[8]) {
    const std::uint8_t *erow = embed + static_cast<std::size_t>(a >> 7) * (128 * kPolicy * 2) +
                               umma::TileOffset(a & 127u, 0, kPolicy);
#pragma unroll
    for (int kg = 0; kg < 8; ++kg) {
        e[kg] = __ldg(reinterpret_cast<const uint4 *>(erow + kg * 128));
    }
}

// Exact keys of this lane's action in two (game, 32-action chunk) tasks, read from an FP16 embedding table. The
// FP16 table holds every embedding value exactly (the fixed features are small integers, the tail rows are the
// genome's own FP16 values), so each FP32 chain -- fma(p_k, e_k, s) for k = 0..63 in ascending order, the plain
// form's and the reference's (output_embedding.hpp:98-119) -- gives ExactScore's bits. kPvLd is the stride of a
// game's policy values (1: a contiguous, 16-byte aligned row, read four values per load). Both tasks' rows and codes
// are loaded before either chain starts, and the two chains run interleaved. key1 is computed for every lane; the
// caller ignores it when it has no second task.
template <int kPvLd>
__device__ __forceinline__ void ChunkKeyPairFp16(const EvalParams &p, const ChunkState &cs, const std::uint8_t *embed,
                                                 const float *pv0, int g0, int chunk0, const float *pv1, int g1,
                                                 int chunk1, int turns, unsigned long long &key0,
                                                 unsigned long long &key1) {
    const std::uint32_t lane = threadIdx.x & 31;
    const std::uint32_t a0 = static_cast<std::uint32_t>(chunk0) * 32u + lane;
    const std::uint32_t a1 = static_cast<std::uint32_t>(chunk1) * 32u + lane;
    const bool v0 = a0 < p.action_count;
    const bool v1 = a1 < p.action_count;
    uint4 e0[8];
    uint4 e1[8];
    LoadEmbedRow(embed, v0 ? a0 : 0u, e0);
    LoadEmbedRow(embed, v1 ? a1 : 0u, e1);
    const std::uint32_t code0 = v0 ? __ldg(p.codes + a0) : 0u;
    const std::uint32_t code1 = v1 ? __ldg(p.codes + a1) : 0u;
    float s0 = 0.0f;
    float s1 = 0.0f;
#pragma unroll
    for (int kg = 0; kg < 8; ++kg) {
        const std::uint32_t w0[4] = {e0[kg].x, e0[kg].y, e0[kg].z, e0[kg].w};
        const std::uint32_t w1[4] = {e1[kg].x, e1[kg].y, e1[kg].z, e1[kg].w};
        // the policy values k = 8 kg .. 8 kg + 7 of both games: two 16-byte loads each from a contiguous row
        float q0[8];
        float q1[8];
        if constexpr (kPvLd == 1) {
            const float4 x0 = *reinterpret_cast<const float4 *>(pv0 + kg * 8);
            const float4 y0 = *reinterpret_cast<const float4 *>(pv0 + kg * 8 + 4);
            const float4 x1 = *reinterpret_cast<const float4 *>(pv1 + kg * 8);
            const float4 y1 = *reinterpret_cast<const float4 *>(pv1 + kg * 8 + 4);
            q0[0] = x0.x, q0[1] = x0.y, q0[2] = x0.z, q0[3] = x0.w, q0[4] = y0.x, q0[5] = y0.y, q0[6] = y0.z,
            q0[7] = y0.w;
            q1[0] = x1.x, q1[1] = x1.y, q1[2] = x1.z, q1[3] = x1.w, q1[4] = y1.x, q1[5] = y1.y, q1[6] = y1.z,
            q1[7] = y1.w;
        } else {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                q0[i] = pv0[(kg * 8 + i) * kPvLd];
                q1[i] = pv1[(kg * 8 + i) * kPvLd];
            }
        }
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 f0 = __half22float2(*reinterpret_cast<const __half2 *>(&w0[i]));
            const float2 f1 = __half22float2(*reinterpret_cast<const __half2 *>(&w1[i]));
            s0 = __fmaf_rn(q0[2 * i], f0.x, s0);
            s1 = __fmaf_rn(q1[2 * i], f1.x, s1);
            s0 = __fmaf_rn(q0[2 * i + 1], f0.y, s0);
            s1 = __fmaf_rn(q1[2 * i + 1], f1.y, s1);
        }
    }
    bool m0 = !v0;
    bool m1 = !v1;
    for (int u = 0; u < turns; ++u) {
        m0 |= cs.guess[u][g0] == code0;
        m1 |= cs.guess[u][g1] == code1;
    }
    key0 = m0 ? 0ull : PackKey(s0, a0);
    key1 = m1 ? 0ull : PackKey(s1, a1);
}

// Folds a warp's keys (the masked argmax) into *best_key: the warp's largest 64-bit key as two 32-bit maximum
// reductions, the high words first, then the low words of the lanes that hold that high word.
__device__ __forceinline__ void FoldKeys(unsigned long long *best_key, unsigned long long key) {
    const std::uint32_t hi = static_cast<std::uint32_t>(key >> 32);
    const std::uint32_t top = __reduce_max_sync(0xffffffffu, hi);
    const std::uint32_t lo = __reduce_max_sync(0xffffffffu, hi == top ? static_cast<std::uint32_t>(key) : 0u);
    key = (static_cast<unsigned long long>(top) << 32) | lo;
    if ((threadIdx.x & 31) == 0 && key != 0) {
        atomicMax(best_key, key);
    }
}

// Warp-cooperative exact re-scoring of 32-action chunk `chunk` for game g, whose policy vector is
// pv[k * ld]; folds the masked argmax (guessed words excluded by word equality) into *best_key.
__device__ __forceinline__ void RescoreChunk(const EvalParams &p, const ChunkState &cs, unsigned long long *best_key,
                                             const float *pv, int ld, const __half *tail, int g, int chunk,
                                             int turns) {
    FoldKeys(best_key, ChunkKey(p, cs, pv, ld, tail, g, chunk, turns));
}

}  // namespace tcx
}  // namespace nwg
