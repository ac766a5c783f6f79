// Shard-release statistics on the GPU: the per-generation fitness telemetry and the genetic-convergence metrics the
// reference's adaptive training-shard release reads (cli/run_genetic_algorithm.cu:1080-1186 fitness row,
// :886-1054 convergence sample gather, :1199-1282 release decision; genetic_algorithm/genetic_convergence.hpp:49-196
// sample plan and metrics), and the release decision itself.
//
// The reference computes both on the host after copying the data down: a std::sort of the fitness values, then
// sequential double sums; and sequential float sums over a 256 x 8,192 sample of genome values. Its host build
// has no fused multiply-add (x86-64 baseline, SSE arithmetic), so every product and sum is rounded on its own.
// Here the data stays on the device: one CTA sorts the fitness keys in shared memory (bitonic, float bits mapped to
// order-preserving integers) and walks the sorted values in the reference's order with explicitly rounded double
// operations (__dadd_rn, __dmul_rn, ...); the convergence sample is gathered straight from the slab and reduced
// in the reference's loop order with explicitly rounded float operations, parallel only across independent
// loops (centroid per weight, distance per organism, distance per pair). The results equal the reference's bit
// for bit. The sample plan is drawn on the host with the same standard-library engine and distributions as the
// reference (std::mt19937_64 seeded by the splitmix mix of seed and generation; std::uniform_int_distribution),
// which makes it the reference's plan wherever both are built with the same C++ library.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <random>
#include <unordered_set>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

using namespace nwg;

namespace {

constexpr int kTelemetryThreads = 1024;
constexpr std::size_t kMaxTelemetryPopulation = 32768;  // sort keys fit in 128 KB of shared memory
constexpr std::size_t kSampleOrganisms = 256;           // genetic_convergence.hpp:18-20
constexpr std::size_t kSampleWeights = 8192;
constexpr std::size_t kSamplePairs = 512;
constexpr std::size_t kPolicyScalars = kTailOffsetBytes / 2;  // the policy's FP16 values precede the tail

struct FitnessTelemetryDevice {
    float min, mean, median, p90, p99, max, stddev;
    unsigned long long distinct;
    unsigned long long childless, one_child, more_children;
    int status;
};

__device__ __forceinline__ std::uint32_t OrderKey(std::uint32_t bits) {
    return bits ^ ((bits >> 31) != 0u ? 0xFFFFFFFFu : 0x80000000u);
}

__device__ __forceinline__ float FromOrderKey(std::uint32_t key) {
    return __uint_as_float(key ^ ((key >> 31) != 0u ? 0x80000000u : 0xFFFFFFFFu));
}

// TryCollectGenerationFitnessTelemetry's fitness statistics (run_genetic_algorithm.cu:1100-1146).
__global__ void __launch_bounds__(kTelemetryThreads) FitnessTelemetryKernel(const float *fitness,
                                                                            const std::uint8_t *has_fitness,
                                                                            std::uint32_t n, std::uint32_t padded,
                                                                            FitnessTelemetryDevice *out) {
    extern __shared__ std::uint32_t keys[];
    __shared__ unsigned long long distinct_total;
    __shared__ int missing;
    const int tid = threadIdx.x;
    if (tid == 0) {
        distinct_total = 0;
        missing = 0;
    }
    __syncthreads();
    for (std::uint32_t i = tid; i < padded; i += kTelemetryThreads) {
        if (i < n) {
            keys[i] = OrderKey(__float_as_uint(fitness[i]));
            if (has_fitness[i] == 0) {
                missing = 1;
            }
        } else {
            keys[i] = 0xFFFFFFFFu;
        }
    }
    __syncthreads();
    if (missing != 0) {
        if (tid == 0) {
            out->status = kPopulationNotEvaluated;
        }
        return;
    }
    for (std::uint32_t size = 2; size <= padded; size <<= 1) {
        for (std::uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (std::uint32_t i = tid; i < padded; i += kTelemetryThreads) {
                const std::uint32_t j = i ^ stride;
                if (j > i) {
                    const bool ascending = (i & size) == 0;
                    const std::uint32_t a = keys[i];
                    const std::uint32_t b = keys[j];
                    if ((a > b) == ascending) {
                        keys[i] = b;
                        keys[j] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
    unsigned long long distinct = 0;
    for (std::uint32_t i = tid + 1; i < n; i += kTelemetryThreads) {
        distinct += FromOrderKey(keys[i]) != FromOrderKey(keys[i - 1]) ? 1ull : 0ull;
    }
    atomicAdd(&distinct_total, distinct);
    __syncthreads();
    if (tid != 0) {
        return;
    }
    // the reference's sequential double sums over the sorted values
    double sum = 0.0;
    for (std::uint32_t i = 0; i < n; ++i) {
        sum = __dadd_rn(sum, static_cast<double>(FromOrderKey(keys[i])));
    }
    const double mean = __ddiv_rn(sum, static_cast<double>(n));
    double squares = 0.0;
    for (std::uint32_t i = 0; i < n; ++i) {
        const double delta = __dsub_rn(static_cast<double>(FromOrderKey(keys[i])), mean);
        squares = __dadd_rn(squares, __dmul_rn(delta, delta));
    }
    const std::uint32_t mid = n / 2;
    const float median = (n % 2 == 0)
                             ? __fmul_rn(__fadd_rn(FromOrderKey(keys[mid - 1]), FromOrderKey(keys[mid])), 0.5f)
                             : FromOrderKey(keys[mid]);
    const auto nearest_rank = [&](double percentile) {
        const double rank = ceil(__dmul_rn(__ddiv_rn(percentile, 100.0), static_cast<double>(n)));
        const std::uint32_t r = static_cast<std::uint32_t>(rank);
        const std::uint32_t index = r == 0 ? 0 : r - 1;
        return FromOrderKey(keys[index < n ? index : n - 1]);
    };
    out->min = FromOrderKey(keys[0]);
    out->max = FromOrderKey(keys[n - 1]);
    out->mean = __double2float_rn(mean);
    out->median = median;
    out->p90 = nearest_rank(90.0);
    out->p99 = nearest_rank(99.0);
    out->stddev = __double2float_rn(__dsqrt_rn(__ddiv_rn(squares, static_cast<double>(n))));
    out->distinct = distinct_total + 1;
    out->status = kOk;
}

// The breeding metrics of the same row (run_genetic_algorithm.cu:1147-1183): children per parent.
__global__ void ParentChildCountKernel(const std::uint32_t *pairs, std::uint32_t child_count, std::uint32_t n,
                                       std::uint32_t *per_parent, FitnessTelemetryDevice *out) {
    for (std::uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < child_count; c += gridDim.x * blockDim.x) {
        const std::uint32_t a = pairs[2 * c];
        const std::uint32_t b = pairs[2 * c + 1];
        if (a >= n || b >= n) {
            atomicCAS(&out->status, kOk, kInvalidAssemblyPlan);
            continue;
        }
        atomicAdd(&per_parent[a], 1u);
        atomicAdd(&per_parent[b], 1u);
    }
}

__global__ void ParentClassKernel(const std::uint32_t *per_parent, std::uint32_t n, FitnessTelemetryDevice *out) {
    unsigned long long counts[3] = {0, 0, 0};
    for (std::uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const std::uint32_t c = per_parent[i];
        counts[c == 0 ? 0 : (c == 1 ? 1 : 2)] += 1;
    }
    atomicAdd(&out->childless, counts[0]);
    atomicAdd(&out->one_child, counts[1]);
    atomicAdd(&out->more_children, counts[2]);
}

// GatherGeneticConvergenceSamplesKernel with GeneticConvergenceTrainableValueAt (run_genetic_algorithm.cu:886-939):
// trainable scalar w of an organism is policy half w, then tail row (w - P) / 38, feature (w - P) % 38.
__global__ void GatherConvergenceSampleKernel(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                              const std::uint32_t *organisms, std::uint32_t sample_organisms,
                                              const std::uint32_t *weights, std::uint32_t sample_weights,
                                              std::size_t action_count, float *values) {
    const std::size_t total = static_cast<std::size_t>(sample_organisms) * sample_weights;
    for (std::size_t flat = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; flat < total;
         flat += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const std::size_t o = flat / sample_weights;
        const std::uint32_t w = weights[flat - o * sample_weights];
        const __half *genome = reinterpret_cast<const __half *>(slab + slots[organisms[o]] * pitch);
        float v = 0.0f;
        if (w < kPolicyScalars) {
            v = __half2float(genome[w]);
        } else if (w - kPolicyScalars < action_count * kTailDim) {
            v = __half2float(genome[w]);  // the tail rows follow the policy halfs contiguously
        }
        values[flat] = v;
    }
}

// TryComputeMetrics (genetic_convergence.hpp:121-194), loop by loop.
__global__ void CentroidKernel(const float *values, std::uint32_t organisms, std::uint32_t weights, float *centroid) {
    const float inverse = __fdiv_rn(1.0f, static_cast<float>(organisms));
    for (std::uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < weights; w += gridDim.x * blockDim.x) {
        float c = 0.0f;
        for (std::uint32_t o = 0; o < organisms; ++o) {
            c = __fadd_rn(c, values[static_cast<std::size_t>(o) * weights + w]);
        }
        centroid[w] = __fmul_rn(c, inverse);
    }
}

__global__ void DistanceKernel(const float *values, std::uint32_t weights, const float *centroid,
                               std::uint32_t organisms, const std::uint32_t *pairs, std::uint32_t pair_count,
                               float *distances) {
    const std::uint32_t jobs = organisms + pair_count;
    for (std::uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < jobs; j += gridDim.x * blockDim.x) {
        const float *a = values + static_cast<std::size_t>(j < organisms ? j : pairs[2 * (j - organisms)]) * weights;
        const float *b = j < organisms ? centroid : values + static_cast<std::size_t>(pairs[2 * (j - organisms) + 1]) * weights;
        float squared = 0.0f;
        for (std::uint32_t w = 0; w < weights; ++w) {
            const float delta = __fsub_rn(a[w], b[w]);
            squared = __fadd_rn(squared, __fmul_rn(delta, delta));
        }
        distances[j] = __fsqrt_rn(squared);
    }
}

struct ConvergenceDevice {
    float centroid_mean, centroid_min, centroid_max, pair_mean, pair_min, pair_max;
};

__global__ void ConvergenceFinalizeKernel(const float *distances, std::uint32_t organisms, std::uint32_t pair_count,
                                          ConvergenceDevice *out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) {
        return;
    }
    const float inverse = __fdiv_rn(1.0f, static_cast<float>(organisms));
    float sum = 0.0f, lo = FLT_MAX, hi = 0.0f;
    for (std::uint32_t o = 0; o < organisms; ++o) {
        const float d = distances[o];
        sum = __fadd_rn(sum, d);
        lo = d < lo ? d : lo;
        hi = d > hi ? d : hi;
    }
    out->centroid_mean = __fmul_rn(sum, inverse);
    out->centroid_min = lo;
    out->centroid_max = hi;
    if (pair_count == 0) {
        out->pair_mean = 0.0f;
        out->pair_min = 0.0f;
        out->pair_max = 0.0f;
        return;
    }
    sum = 0.0f;
    lo = FLT_MAX;
    hi = 0.0f;
    for (std::uint32_t p = 0; p < pair_count; ++p) {
        const float d = distances[organisms + p];
        sum = __fadd_rn(sum, d);
        lo = d < lo ? d : lo;
        hi = d > hi ? d : hi;
    }
    out->pair_mean = __fdiv_rn(sum, static_cast<float>(pair_count));
    out->pair_min = lo;
    out->pair_max = hi;
}

// MixSamplingSeed (genetic_convergence.hpp:52-61): a splitmix-style finalizer of seed and generation.
std::uint64_t SamplingSeed(std::uint32_t run_seed, std::size_t generation) {
    std::uint64_t v = 0x9e3779b97f4a7c15ULL ^ static_cast<std::uint64_t>(run_seed);
    v ^= static_cast<std::uint64_t>(generation) + 0xbf58476d1ce4e5b9ULL + (v << 6U) + (v >> 2U);
    v ^= v >> 30U;
    v *= 0xbf58476d1ce4e5b9ULL;
    v ^= v >> 27U;
    v *= 0x94d049bb133111ebULL;
    v ^= v >> 31U;
    return v;
}

// SampleUniqueIndices (genetic_convergence.hpp:63-84): Floyd's sampling of distinct indices, in draw order.
std::vector<std::size_t> DistinctSample(std::size_t universe, std::size_t requested, std::mt19937_64 &engine) {
    const std::size_t count = requested < universe ? requested : universe;
    std::vector<std::size_t> out;
    out.reserve(count);
    if (count == universe) {
        out.resize(count);
        std::iota(out.begin(), out.end(), std::size_t{0});
        return out;
    }
    std::unordered_set<std::size_t> taken;
    taken.reserve(count * 2U);
    for (std::size_t top = universe - count; top < universe; ++top) {
        std::uniform_int_distribution<std::size_t> pick(0, top);
        const std::size_t candidate = pick(engine);
        const std::size_t chosen = taken.count(candidate) != 0 ? top : candidate;
        taken.insert(chosen);
        out.push_back(chosen);
    }
    return out;
}

}  // namespace

extern "C" {

// MakeSamplePlan (genetic_convergence.hpp:86-119).
int nwg_convergence_sample_plan(size_t organism_count, size_t trainable_count, uint32_t run_seed, size_t generation,
                                uint32_t *organisms, size_t *organism_count_out, uint32_t *weights,
                                size_t *weight_count_out, uint32_t *pairs, size_t *pair_count_out) {
    if (organism_count == 0 || trainable_count == 0 || trainable_count > 0xFFFFFFFFull || organisms == nullptr ||
        weights == nullptr || pairs == nullptr) {
        return kInvalidGeneration;
    }
    std::mt19937_64 engine(SamplingSeed(run_seed, generation));
    const std::vector<std::size_t> o = DistinctSample(organism_count, kSampleOrganisms, engine);
    const std::vector<std::size_t> w = DistinctSample(trainable_count, kSampleWeights, engine);
    for (std::size_t i = 0; i < o.size(); ++i) {
        organisms[i] = static_cast<std::uint32_t>(o[i]);
    }
    for (std::size_t i = 0; i < w.size(); ++i) {
        weights[i] = static_cast<std::uint32_t>(w[i]);
    }
    std::size_t pair_count = 0;
    if (o.size() >= 2) {
        std::uniform_int_distribution<std::size_t> first_pick(0, o.size() - 1U);
        std::uniform_int_distribution<std::size_t> second_pick(0, o.size() - 2U);
        for (; pair_count < kSamplePairs; ++pair_count) {
            const std::size_t first = first_pick(engine);
            std::size_t second = second_pick(engine);
            second += second >= first ? 1U : 0U;
            pairs[2 * pair_count] = static_cast<std::uint32_t>(first);
            pairs[2 * pair_count + 1] = static_cast<std::uint32_t>(second);
        }
    }
    *organism_count_out = o.size();
    *weight_count_out = w.size();
    *pair_count_out = pair_count;
    return kOk;
}

int nwg_fitness_telemetry_collect(const nwg_runtime *rt, const nwg_runtime_word_counts *counts, bool with_breeding,
                                  nwg_fitness_telemetry *row) {
    GenerationView v{};
    if (row == nullptr || ReadGenerationView(rt, &v) != kOk) {
        return kInvalidRuntimeConfig;
    }
    std::memset(row, 0, sizeof(*row));
    const std::size_t n = v.generation_size;
    if (n == 0) {
        return kInvalidGeneration;
    }
    if (n > kMaxTelemetryPopulation) {
        return kUnsupported;
    }
    if (with_breeding && v.planned_children == 0) {
        return kInvalidAssemblyPlan;
    }
    std::uint32_t padded = 1;
    while (padded < n) {
        padded <<= 1;
    }
    FitnessTelemetryDevice *d = nullptr;
    std::uint32_t *per_parent = nullptr;
    FitnessTelemetryDevice h{};
    const int smem = static_cast<int>(padded * sizeof(std::uint32_t));
    bool ok = cudaFuncSetAttribute(FitnessTelemetryKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) ==
                  cudaSuccess &&
              cudaMalloc(&d, sizeof(FitnessTelemetryDevice)) == cudaSuccess &&
              cudaMalloc(&per_parent, n * sizeof(std::uint32_t)) == cudaSuccess &&
              cudaMemsetAsync(d, 0, sizeof(FitnessTelemetryDevice), v.stream) == cudaSuccess &&
              cudaMemsetAsync(per_parent, 0, n * sizeof(std::uint32_t), v.stream) == cudaSuccess;
    if (ok) {
        FitnessTelemetryKernel<<<1, kTelemetryThreads, smem, v.stream>>>(v.fitness, v.has_fitness,
                                                                         static_cast<std::uint32_t>(n), padded, d);
        ok = cudaGetLastError() == cudaSuccess;
    }
    if (ok && with_breeding) {
        ParentChildCountKernel<<<64, 256, 0, v.stream>>>(v.pairs, static_cast<std::uint32_t>(v.planned_children),
                                                         static_cast<std::uint32_t>(n), per_parent, d);
        ParentClassKernel<<<64, 256, 0, v.stream>>>(per_parent, static_cast<std::uint32_t>(n), d);
        ok = cudaGetLastError() == cudaSuccess;
    }
    ok = ok && cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, v.stream) == cudaSuccess &&
         cudaStreamSynchronize(v.stream) == cudaSuccess;
    cudaFree(d);
    cudaFree(per_parent);
    if (!ok) {
        return kCudaFailure;
    }
    if (h.status != kOk) {
        return h.status;
    }
    row->generation = v.generation_index;
    row->population_size = n;
    row->training_word_count = counts != nullptr ? counts->training_word_count : 0;
    row->fitness_min = h.min;
    row->fitness_mean = h.mean;
    row->fitness_median = h.median;
    row->fitness_p90 = h.p90;
    row->fitness_p99 = h.p99;
    row->fitness_max = h.max;
    row->fitness_stddev = h.stddev;
    row->distinct_fitness_count = h.distinct;
    if (with_breeding) {
        row->has_breeding_metrics = true;
        row->parent_childless_count = h.childless;
        row->parent_one_child_count = h.one_child;
        row->parent_multiple_children_count = h.more_children;
    }
    return kOk;
}

int nwg_convergence_telemetry_collect(const nwg_runtime *rt, uint32_t run_seed, nwg_convergence_telemetry *row) {
    GenerationView v{};
    if (row == nullptr || ReadGenerationView(rt, &v) != kOk) {
        return kInvalidRuntimeConfig;
    }
    std::memset(row, 0, sizeof(*row));
    if (v.generation_size == 0) {
        return kInvalidGeneration;
    }
    std::vector<std::uint32_t> organisms(kSampleOrganisms), weights(kSampleWeights), pairs(2 * kSamplePairs);
    std::size_t n_org = 0, n_w = 0, n_pairs = 0;
    int st = nwg_convergence_sample_plan(v.generation_size, kPolicyScalars + v.action_count * kTailDim, run_seed,
                                         v.generation_index, organisms.data(), &n_org, weights.data(), &n_w,
                                         pairs.data(), &n_pairs);
    if (st != kOk) {
        return st;
    }
    // sampled organisms must hold a live slot (run_genetic_algorithm.cu:969-984)
    std::vector<std::uint32_t> slots(v.generation_size);
    if (cudaStreamSynchronize(v.stream) != cudaSuccess ||
        cudaMemcpy(slots.data(), v.slots, slots.size() * sizeof(std::uint32_t), cudaMemcpyDeviceToHost) !=
            cudaSuccess) {
        return kCudaFailure;
    }
    for (std::size_t i = 0; i < n_org; ++i) {
        if (slots[organisms[i]] == 0xFFFFFFFFu) {
            return kInvalidGeneration;
        }
    }
    std::uint32_t *d_org = nullptr, *d_w = nullptr, *d_pairs = nullptr;
    float *values = nullptr, *centroid = nullptr, *distances = nullptr;
    ConvergenceDevice *d_out = nullptr;
    ConvergenceDevice h{};
    cudaEvent_t begin = nullptr, end = nullptr;
    bool ok = cudaMalloc(&d_org, n_org * 4) == cudaSuccess && cudaMalloc(&d_w, n_w * 4) == cudaSuccess &&
              cudaMalloc(&d_pairs, (2 * n_pairs + 2) * 4) == cudaSuccess &&
              cudaMalloc(&values, n_org * n_w * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&centroid, n_w * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&distances, (n_org + n_pairs) * sizeof(float)) == cudaSuccess &&
              cudaMalloc(&d_out, sizeof(ConvergenceDevice)) == cudaSuccess &&
              cudaEventCreate(&begin) == cudaSuccess && cudaEventCreate(&end) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_org, organisms.data(), n_org * 4, cudaMemcpyHostToDevice, v.stream) == cudaSuccess &&
         cudaMemcpyAsync(d_w, weights.data(), n_w * 4, cudaMemcpyHostToDevice, v.stream) == cudaSuccess &&
         cudaMemcpyAsync(d_pairs, pairs.data(), 2 * n_pairs * 4 + 4, cudaMemcpyHostToDevice, v.stream) == cudaSuccess;
    if (ok) {
        cudaEventRecord(begin, v.stream);
        GatherConvergenceSampleKernel<<<256, 256, 0, v.stream>>>(v.slab, v.pitch, v.slots, d_org,
                                                                 static_cast<std::uint32_t>(n_org), d_w,
                                                                 static_cast<std::uint32_t>(n_w), v.action_count,
                                                                 values);
        CentroidKernel<<<32, 256, 0, v.stream>>>(values, static_cast<std::uint32_t>(n_org),
                                                 static_cast<std::uint32_t>(n_w), centroid);
        DistanceKernel<<<(static_cast<unsigned>(n_org + n_pairs) + 127) / 128, 128, 0, v.stream>>>(
            values, static_cast<std::uint32_t>(n_w), centroid, static_cast<std::uint32_t>(n_org), d_pairs,
            static_cast<std::uint32_t>(n_pairs), distances);
        ConvergenceFinalizeKernel<<<1, 32, 0, v.stream>>>(distances, static_cast<std::uint32_t>(n_org),
                                                          static_cast<std::uint32_t>(n_pairs), d_out);
        cudaEventRecord(end, v.stream);
        ok = cudaGetLastError() == cudaSuccess &&
             cudaMemcpyAsync(&h, d_out, sizeof(h), cudaMemcpyDeviceToHost, v.stream) == cudaSuccess &&
             cudaStreamSynchronize(v.stream) == cudaSuccess;
    }
    float ms = 0.0f;
    if (ok) {
        cudaEventElapsedTime(&ms, begin, end);
    }
    cudaFree(d_org);
    cudaFree(d_w);
    cudaFree(d_pairs);
    cudaFree(values);
    cudaFree(centroid);
    cudaFree(distances);
    cudaFree(d_out);
    if (begin != nullptr) {
        cudaEventDestroy(begin);
    }
    if (end != nullptr) {
        cudaEventDestroy(end);
    }
    if (!ok) {
        return kCudaFailure;
    }
    row->generation = v.generation_index;
    row->sample_organisms = n_org;
    row->sample_weights = n_w;
    row->pair_count = n_pairs;
    row->centroid_distance_mean = h.centroid_mean;
    row->centroid_distance_min = h.centroid_min;
    row->centroid_distance_max = h.centroid_max;
    row->pairwise_distance_mean = h.pair_mean;
    row->pairwise_distance_min = h.pair_min;
    row->pairwise_distance_max = h.pair_max;
    row->elapsed_ms = ms;
    return kOk;
}

// TryMaybeReleaseTrainingDataShard (cli/run_genetic_algorithm.cu:1199-1282) with TryRecordTrainingDataShardRelease
// (training_folder/training_data.hpp:119-133).
int nwg_maybe_release_training_shard(const nwg_runtime *rt, const nwg_runtime_word_counts *counts,
                                     const nwg_shard_release_policy *policy, size_t catalog_word_count,
                                     uint32_t run_seed, nwg_shard_release_history *history,
                                     nwg_pending_injection *pending, size_t *next_word_count,
                                     nwg_fitness_telemetry *fitness_row, nwg_convergence_telemetry *convergence_row) {
    GenerationView v{};
    if (counts == nullptr || policy == nullptr || history == nullptr || pending == nullptr ||
        next_word_count == nullptr || ReadGenerationView(rt, &v) != kOk) {
        return kInvalidRuntimeConfig;
    }
    std::memset(pending, 0, sizeof(*pending));
    *next_word_count = counts->action_space_word_count;
    if (history->release_count == 0) {
        return kInvalidTrainingShard;  // no foundation release record
    }
    if (counts->action_space_word_count >= catalog_word_count || counts->training_word_schedule.word_count_step == 0) {
        return kOk;
    }
    const std::size_t latest = history->release_count - 1;
    const std::size_t release_generation = v.generation_index + 1;
    const std::size_t previous = history->release_generations[latest];
    const std::size_t since = release_generation >= previous ? release_generation - previous : 0;
    if ((history->release_count == 1 && release_generation < policy->first_new_release_generation) ||
        since < policy->min_gap_generations) {
        return kOk;
    }
    nwg_fitness_telemetry f{};
    nwg_convergence_telemetry c{};
    int st = nwg_fitness_telemetry_collect(rt, counts, false, &f);
    if (st == kOk) {
        st = nwg_convergence_telemetry_collect(rt, run_seed, &c);
    }
    if (st != kOk) {
        return st;
    }
    if (fitness_row != nullptr) {
        *fitness_row = f;
    }
    if (convergence_row != nullptr) {
        *convergence_row = c;
    }
    if (!(c.centroid_distance_mean <= policy->centroid_distance_threshold) ||
        !(f.fitness_p99 > policy->fitness_p99_threshold)) {
        return kOk;
    }
    const std::size_t first = counts->action_space_word_count;
    const std::size_t remaining = catalog_word_count - first;
    const std::size_t step = counts->training_word_schedule.word_count_step;
    const std::size_t injection = remaining < step ? remaining : step;
    if (history->release_count >= NWG_CATALOG_CAPACITY ||
        release_generation <= history->release_generations[history->release_count - 1]) {
        return kInvalidTrainingShard;
    }
    history->release_generations[history->release_count] = release_generation;
    history->release_fitness_p99[history->release_count] = f.fitness_p99;
    ++history->release_count;
    pending->enabled = true;
    pending->first_catalog_word_index = first;
    pending->injection_count = injection;
    *next_word_count = first + injection;
    return kOk;
}

}  // extern "C"
