// Output-embedding injection for action-space growth: every child of a widening generation gets one new tail
// row per newly released catalog word (genotype_slab/device_runtime.cu:518-617, device/injection_ops.cuh:22-64,
// genetic_algorithm/output_embedding_injection.hpp:66-199).
//
// For a new word, the row is the mean of the child's 38 trainable policy outputs over the word's three hint grids
// (wordle/hint_grid.hpp: the all-yellow rotations of the word, then two 3-green/2-yellow letter swaps), rounded to
// FP16, then rescaled to the median norm of the child's existing rows. The reference runs the three forwards of
// every word one after another in a warp; here a CTA owns a child and runs its hint-grid states as chunks of up
// to 128 states with one turn count, through the plain form's exact FP32 encoder and trunk (eval_common.cuh), so
// each policy vector is the reference's FMA chain bit for bit. Chunks run grid by grid, so every word's three
// outputs are summed in the reference's order. The median is found by a 4-pass radix select over the norms'
// bit patterns (non-negative floats order like their bits), which gives the exact k-th value.
#include <cuda_fp16.h>

#include "eval_common.cuh"

namespace nwg {
namespace {

using namespace evalx;

struct InjectParams {
    std::uint8_t *slab;               // children's slab (their new pitch)
    std::size_t pitch;
    const std::uint32_t *child_slots; // slot of each child
    std::uint32_t child_count;
    std::uint32_t parent_action_count;
    std::uint32_t injection_count;
    const std::uint32_t *guess_codes; // [word][3 grids][4 turns] packed guesses
    const std::uint16_t *tiles;       // [word][3][4] packed feedback
    const int4 *chunks;               // {grid, turns, first entry of `order`, states}
    const std::uint32_t *order;       // words of grid 0, then grid 1, then grid 2, each grid sorted by turn count
    int chunk_count;
    float *scratch;                   // per CTA: layer-1 accumulators [256][128]
    float *sums;                      // per CTA: [injection_count][38] feature sums
    int *status;
};

// Exact k-th smallest (0-based) of n non-negative floats given as bit patterns, over the whole CTA.
__device__ float SelectKth(const unsigned *bits, int n, unsigned k, unsigned *hist, unsigned *shared) {
    unsigned prefix = 0;
    unsigned mask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) {
            hist[b] = 0;
        }
        __syncthreads();
        for (int a = threadIdx.x; a < n; a += blockDim.x) {
            const unsigned v = bits[a];
            if ((v & mask) == prefix) {
                atomicAdd(&hist[(v >> shift) & 255u], 1u);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            unsigned cumulative = 0;
            for (unsigned b = 0; b < 256; ++b) {
                if (cumulative + hist[b] > k) {
                    shared[0] = prefix | (b << shift);
                    shared[1] = k - cumulative;
                    break;
                }
                cumulative += hist[b];
            }
        }
        __syncthreads();
        prefix = shared[0];
        k = shared[1];
        mask |= 255u << shift;
        __syncthreads();
    }
    return __uint_as_float(prefix);
}

// output_embedding_injection.hpp:66-75 (the device build contracts `sum += v * v`).
__device__ __forceinline__ float RowNorm(const __half *row) {
    float sum = 0.0f;
    for (int k = 0; k < kTailDim; ++k) {
        const float v = __half2float(row[k]);
        sum = __fmaf_rn(v, v, sum);
    }
    return sqrtf(sum);
}

__global__ void __launch_bounds__(kEvalThreads, 2) InjectKernel(const InjectParams q) {
    extern __shared__ __align__(16) float arena[];
    __shared__ ChunkState cs;
    __shared__ unsigned hist[256];
    __shared__ unsigned select_state[2];
    const int tid = threadIdx.x;
    EvalParams ep{};  // no trace
    float *scratch = q.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats;
    float *sums = q.sums + static_cast<std::size_t>(blockIdx.x) * q.injection_count * kTailDim;
    const int n_inj = static_cast<int>(q.injection_count);
    for (std::uint32_t child = blockIdx.x; child < q.child_count; child += gridDim.x) {
        std::uint8_t *image = q.slab + static_cast<std::size_t>(q.child_slots[child]) * q.pitch;
        const __half *gh = reinterpret_cast<const __half *>(image);
        __half *tails = reinterpret_cast<__half *>(image + kTailOffsetBytes);

        // ---- hint-grid policy forwards, summed per word in grid order ----
        for (int ck = 0; ck < q.chunk_count; ++ck) {
            const int4 c = q.chunks[ck];
            const int grid = c.x;
            const int turns = c.y;
            const int begin = c.z;
            const int states = c.w;
            if (tid < kChunkGames) {
                const int g = tid;
                const std::uint32_t word = g < states ? q.order[begin + g] : 0u;
                for (int u = 0; u < kMaxTurns; ++u) {
                    const bool live = g < states && u < turns;
                    cs.guess[u][g] = live ? q.guess_codes[(word * 3 + grid) * 4 + u] : 0u;
                    cs.tiles[u][g] = live ? q.tiles[(word * 3 + grid) * 4 + u] : std::uint16_t{0};
                }
            }
            for (int idx = tid; idx < kScratchFloats / 4; idx += kEvalThreads) {
                const float b = H2F(gh, kTrB1 + (idx * 4) / kChunkGames);
                reinterpret_cast<float4 *>(scratch)[idx] = make_float4(b, b, b, b);
            }
            __syncthreads();
            for (int u = 0; u < turns; ++u) {
                EncodeRound(cs, gh, arena, scratch, u);
            }
            TrunkForward(ep, cs, gh, arena, scratch, turns, 0, 0);
            for (int idx = tid; idx < states * kTailDim; idx += kEvalThreads) {
                const int g = idx / kTailDim;
                const int f = idx - g * kTailDim;
                const std::uint32_t word = q.order[begin + g];
                const float v = arena[(kFixedDim + f) * kLd + g];
                float &s = sums[word * kTailDim + f];
                s = grid == 0 ? v : s + v;  // ((0 + p0) + p1) + p2
            }
            __syncthreads();
        }

        // ---- target norm: median of the child's existing rows ----
        unsigned *norm_bits = reinterpret_cast<unsigned *>(arena);
        const int n_rows = static_cast<int>(q.parent_action_count);
        for (int a = tid; a < n_rows; a += kEvalThreads) {
            norm_bits[a] = __float_as_uint(RowNorm(tails + static_cast<std::size_t>(a) * kTailDim));
        }
        __syncthreads();
        const unsigned upper_rank = static_cast<unsigned>(n_rows / 2);
        const float upper = SelectKth(norm_bits, n_rows, upper_rank, hist, select_state);
        float target = upper;
        if ((n_rows % 2) == 0) {
            const float lower = SelectKth(norm_bits, n_rows, upper_rank - 1u, hist, select_state);
            target = 0.5f * (lower + upper);
        }

        // ---- seed and rescale the new rows ----
        const float third = 1.0f / 3.0f;
        for (int i = tid; i < n_inj; i += kEvalThreads) {
            __half *row = tails + static_cast<std::size_t>(q.parent_action_count + i) * kTailDim;
            __half seed[kTailDim];
            for (int k = 0; k < kTailDim; ++k) {
                seed[k] = __float2half(sums[i * kTailDim + k] * third);
            }
            float scale = 0.0f;
            if (target > 1.0e-6f) {
                const float current = RowNorm(seed);
                if (!(current > 1.0e-6f)) {
                    SetStatus(q.status, kOutputEmbeddingInjectionFailed);
                }
                scale = current > 1.0e-6f ? target / current : 0.0f;
            }
            for (int k = 0; k < kTailDim; ++k) {
                row[k] = __float2half(__half2float(seed[k]) * scale);
            }
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t LaunchInject(std::uint8_t *slab, std::size_t pitch, const std::uint32_t *child_slots,
                         std::uint32_t child_count, std::uint32_t parent_action_count, std::uint32_t injection_count,
                         const std::uint32_t *guess_codes, const std::uint16_t *tiles, const int4 *chunks,
                         const std::uint32_t *order, int chunk_count, float *scratch, float *sums, int cta_count,
                         int *status, cudaStream_t stream) {
    const int arena_bytes = kArenaFloats * static_cast<int>(sizeof(float));
    static std::atomic<unsigned long long> configured{0};
    if (const cudaError_t e = RaiseSharedLimit(InjectKernel, arena_bytes, configured);
        e != cudaSuccess) {
        return e;
    }
    if (child_count == 0 || cta_count <= 0) {
        return cudaSuccess;
    }
    InjectParams q{};
    q.slab = slab;
    q.pitch = pitch;
    q.child_slots = child_slots;
    q.child_count = child_count;
    q.parent_action_count = parent_action_count;
    q.injection_count = injection_count;
    q.guess_codes = guess_codes;
    q.tiles = tiles;
    q.chunks = chunks;
    q.order = order;
    q.chunk_count = chunk_count;
    q.scratch = scratch;
    q.sums = sums;
    q.status = status;
    InjectKernel<<<cta_count, kEvalThreads, arena_bytes, stream>>>(q);
    return cudaGetLastError();
}

}  // namespace nwg
