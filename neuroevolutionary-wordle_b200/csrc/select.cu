// Cellular rank-roulette parent selection, one thread per child.
//
// Replaces BuildSlabAssemblyPlanKernel (genetic_algorithm/device/slab_runtime.cu:633-675) and
// TrySelectCellularParentPairDevice (genetic_algorithm/device/selection_ops.cuh:218-263). The child's
// Philox stream is (seed ^ 0xA341316C, uint32(child + generation * 8191)) and is consumed in the same
// order (two 32-bit outputs for the tie-break seed, one uniform for the threshold, per parent). The
// neighbourhood is the deduplicated Moore list for radius <= 2 (spatial/grid.hpp:181-218) and every cell
// within the toroidal Chebyshev radius, in index order, above that (selection_ops.cuh:163-216). A row band of a
// larger grid selects for its own children only (child_first = the band's first cell), over the whole grid's
// fitness, with the same streams as a single-population run.
#include <curand_kernel.h>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr std::uint64_t kNone = ~0ull;
constexpr int kMaxMoore = 25;

// selection_ops.cuh:32-37: splitmix64 finaliser for the rank tie-break keys.
__device__ __forceinline__ std::uint64_t MixKey(std::uint64_t v) {
    v += 0x9E3779B97F4A7C15ULL;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ULL;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBULL;
    return v ^ (v >> 31);
}

// selection_ops.cuh:43-57: lower fitness ranks first; equal fitness by seeded key, then by index.
__device__ __forceinline__ bool RanksBefore(float lf, std::uint64_t li, float rf, std::uint64_t ri,
                                            std::uint64_t seed) {
    if (lf < rf) {
        return true;
    }
    if (lf > rf) {
        return false;
    }
    const std::uint64_t lk = MixKey(seed ^ li);
    const std::uint64_t rk = MixKey(seed ^ ri);
    return lk < rk || (lk == rk && li < ri);
}

__device__ __forceinline__ std::uint64_t Chebyshev(std::uint64_t rows, std::uint64_t cols, std::uint64_t a,
                                                   std::uint64_t b) {
    auto axis = [](std::uint64_t x, std::uint64_t y, std::uint64_t side) {
        const std::uint64_t f = x >= y ? x - y : y - x;
        const std::uint64_t w = side - f;
        return f < w ? f : w;
    };
    const std::uint64_t dr = axis(a / cols, b / cols, rows);
    const std::uint64_t dc = axis(a % cols, b % cols, cols);
    return dr > dc ? dr : dc;
}

__device__ __forceinline__ std::uint64_t NextTieSeed(curandStatePhilox4_32_10_t &state) {
    const std::uint64_t high = curand(&state);
    const std::uint64_t low = curand(&state);
    return (high << 32) ^ low;
}

// selection_ops.cuh:115-161 over an explicit candidate list.
__device__ bool SelectFromList(const float *f, const std::uint8_t *has, const std::uint32_t *cand, int count,
                               curandStatePhilox4_32_10_t &state, float exponent, std::uint64_t excluded,
                               std::uint64_t &selected) {
    const std::uint64_t seed = NextTieSeed(state);
    float weight[kMaxMoore];
    float total = 0.0f;
    bool found = false;
    std::uint64_t fallback = 0;
    for (int k = 0; k < count; ++k) {
        const std::uint64_t c = cand[k];
        weight[k] = 0.0f;
        if (c == excluded || has[c] == 0) {
            continue;
        }
        std::uint32_t rank = 1;
        for (int k2 = 0; k2 < count; ++k2) {
            const std::uint64_t c2 = cand[k2];
            if (c2 == c || c2 == excluded || has[c2] == 0) {
                continue;
            }
            rank += RanksBefore(f[c2], c2, f[c], c, seed) ? 1u : 0u;
        }
        weight[k] = powf(static_cast<float>(rank), exponent);
        total += weight[k];
        fallback = c;
        found = true;
    }
    if (!found || total <= 0.0f) {
        return false;
    }
    const float threshold = curand_uniform(&state) * total;
    float cumulative = 0.0f;
    for (int k = 0; k < count; ++k) {
        const std::uint64_t c = cand[k];
        if (c == excluded || has[c] == 0) {
            continue;
        }
        cumulative += weight[k];
        if (threshold <= cumulative) {
            selected = c;
            return true;
        }
    }
    selected = fallback;
    return true;
}

// selection_ops.cuh:91-113 and :163-216: scan of the whole grid for radius > 2.
__device__ bool SelectFromRadius(const float *f, const std::uint8_t *has, std::uint64_t rows, std::uint64_t cols,
                                 std::uint64_t focal, std::uint64_t radius, curandStatePhilox4_32_10_t &state,
                                 float exponent, std::uint64_t excluded, std::uint64_t &selected) {
    const std::uint64_t cells = rows * cols;
    const std::uint64_t seed = NextTieSeed(state);
    auto eligible = [&](std::uint64_t c) {
        return c != excluded && has[c] != 0 && Chebyshev(rows, cols, focal, c) <= radius;
    };
    auto rank_of = [&](std::uint64_t c) {
        std::uint32_t rank = 1;
        for (std::uint64_t c2 = 0; c2 < cells; ++c2) {
            if (c2 == c || !eligible(c2)) {
                continue;
            }
            rank += RanksBefore(f[c2], c2, f[c], c, seed) ? 1u : 0u;
        }
        return rank;
    };
    float total = 0.0f;
    bool found = false;
    std::uint64_t fallback = 0;
    for (std::uint64_t c = 0; c < cells; ++c) {
        if (!eligible(c)) {
            continue;
        }
        total += powf(static_cast<float>(rank_of(c)), exponent);
        fallback = c;
        found = true;
    }
    if (!found || total <= 0.0f) {
        return false;
    }
    const float threshold = curand_uniform(&state) * total;
    float cumulative = 0.0f;
    for (std::uint64_t c = 0; c < cells; ++c) {
        if (!eligible(c)) {
            continue;
        }
        cumulative += powf(static_cast<float>(rank_of(c)), exponent);
        if (threshold <= cumulative) {
            selected = c;
            return true;
        }
    }
    selected = fallback;
    return true;
}

__global__ void SelectKernel(const SelectParams p) {
    const std::uint32_t local = blockIdx.x * blockDim.x + threadIdx.x;
    if (local >= p.child_count) {
        return;
    }
    const std::uint32_t child = p.child_first + local;  // the child's index in the whole grid
    const std::uint64_t rows = p.rows;
    const std::uint64_t cols = p.cols;
    // the child keeps its (row, column) in the current grid (selection_ops.cuh:233-235)
    const std::uint64_t focal = (child / cols) * cols + (child % cols);
    curandStatePhilox4_32_10_t state;
    curand_init(static_cast<unsigned long long>(p.planning_seed),
                static_cast<unsigned long long>(static_cast<std::uint32_t>(child + p.generation_index * 8191u)), 0ULL,
                &state);
    std::uint64_t first = 0;
    std::uint64_t second = 0;
    bool ok;
    if (p.radius <= 2) {
        std::uint32_t cand[kMaxMoore];
        int count = 0;
        const long long r = static_cast<long long>(p.radius);
        const long long fr = static_cast<long long>(focal / cols);
        const long long fc = static_cast<long long>(focal % cols);
        for (long long dr = -r; dr <= r; ++dr) {
            for (long long dc = -r; dc <= r; ++dc) {
                long long nr = (fr + dr) % static_cast<long long>(rows);
                nr += nr < 0 ? static_cast<long long>(rows) : 0;
                long long nc = (fc + dc) % static_cast<long long>(cols);
                nc += nc < 0 ? static_cast<long long>(cols) : 0;
                const std::uint32_t idx = static_cast<std::uint32_t>(nr * static_cast<long long>(cols) + nc);
                bool dup = false;
                for (int k = 0; k < count; ++k) {
                    dup |= cand[k] == idx;
                }
                if (!dup) {
                    cand[count++] = idx;
                }
            }
        }
        ok = SelectFromList(p.fitness, p.has_fitness, cand, count, state, p.rank_exponent, kNone, first) &&
             SelectFromList(p.fitness, p.has_fitness, cand, count, state, p.rank_exponent, first, second);
    } else {
        ok = SelectFromRadius(p.fitness, p.has_fitness, rows, cols, focal, p.radius, state, p.rank_exponent, kNone,
                              first) &&
             SelectFromRadius(p.fitness, p.has_fitness, rows, cols, focal, p.radius, state, p.rank_exponent, first,
                              second);
    }
    if (!ok) {
        SetStatus(p.status, kParentSelectionFailed);
        return;
    }
    p.pairs[2 * local] = static_cast<std::uint32_t>(first);
    p.pairs[2 * local + 1] = static_cast<std::uint32_t>(second);
}

}  // namespace

cudaError_t LaunchSelect(const SelectParams &params, cudaStream_t stream) {
    if (params.child_count == 0) {
        return cudaSuccess;
    }
    SelectKernel<<<(params.child_count + 127) / 128, 128, 0, stream>>>(params);
    return cudaGetLastError();
}

}  // namespace nwg
