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

// Folds a warp's keys (the masked argmax) into *best_key.
__device__ __forceinline__ void FoldKeys(unsigned long long *best_key, unsigned long long key) {
    for (int off = 16; off > 0; off >>= 1) {
        const unsigned long long other = __shfl_xor_sync(0xffffffffu, key, off);
        key = other > key ? other : key;
    }
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
