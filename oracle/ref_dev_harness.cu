// Device-side harness around the reference's own device functions.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/libref_dev.so by oracle/build.py,
// compiled for sm_100a from the reference's headers where they lie; nothing is copied).
// Each kernel here calls the reference's __device__ functions in the order its own
// kernels do, so the GPU parity tests can compare the new kernels with the
// reference's arithmetic and random streams bit for bit on the same B200:
//   - refdev_evaluate:  slab_runtime.cu:452-549 (warp per episode) with the guesses
//                       and policy vectors of every decision recorded;
//   - refdev_evaluate_csr: the same episode loop over explicit per-individual word
//                       lists (CSR); only the word lookup of TryInitializeEpisodeGrid
//                       (evaluation_ops.cuh:203-237) is restated, everything the policy,
//                       grid and score code does is the reference's own;
//   - refdev_select:    slab_runtime.cu:633-675 (BuildSlabAssemblyPlanKernel body);
//   - refdev_breed:     genotype_slab/device_runtime.cu:448-516 (breed + mutate body);
//   - refdev_bootstrap: genotype_slab/device_runtime.cu:258-314 (initialisation body);
//   - refdev_inject:    genotype_slab/device_runtime.cu:594-599 (output-embedding injection of a bred child,
//                       device/injection_ops.cuh:22-64), one warp per genome.
// The reference's slab allocator (free-list spin lock) is never called: children and
// organisms are written to caller-provided slots.
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "genetic_algorithm/device/evaluation_ops.cuh"
#include "genetic_algorithm/device/genome_ops.cuh"
#include "genetic_algorithm/device/injection_ops.cuh"
#include "genetic_algorithm/device/selection_ops.cuh"
#include "training_folder/training_data.cu"

namespace {

namespace ga = neuroevolution::genetic_algorithm;
namespace tf = neuroevolution::training_folder;
using ga::device_evaluation_ops::DeviceGenomeEvaluationStatusCode;
using ga::device_evaluation_ops::GenomeEvaluationWarpScratch;
using ga::device_evaluation_ops::ScoreCompletedEpisode;
using ga::device_evaluation_ops::TryCountLocalTrainingWords;
using ga::device_evaluation_ops::TryInitializeEpisodeGrid;
using neuroevolution::inference::dynamic_policy::DynamicInferenceStatusCode;
using neuroevolution::inference::dynamic_policy::SelectNextGuessFromDynamicGenomeConcurrently;
using neuroevolution::model::output_embedding::SelectedAction;
using neuroevolution::spatial::CellularGridShape;

constexpr int kWarps = 4;

__global__ void EvaluateKernel(const std::uint8_t *slab, std::size_t pitch, std::size_t population,
                               std::size_t action_count, const tf::TrainingDataShardRuntime *shards,
                               std::size_t shard_count, CellularGridShape shape, std::size_t max_episodes,
                               float *scores, int *turns, int *choices, float *policy_trace, int *status) {
    __shared__ GenomeEvaluationWarpScratch<32> scratch[kWarps];
    const std::size_t individual = blockIdx.x;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const std::size_t episode = static_cast<std::size_t>(blockIdx.y) * kWarps + warp;
    if (individual >= population) {
        return;
    }
    std::size_t local_words = 0;
    if (TryCountLocalTrainingWords(shards, shard_count, shape, individual, local_words) !=
        DeviceGenomeEvaluationStatusCode::kOk) {
        if (lane == 0) {
            atomicCAS(status, 0, 1);
        }
        return;
    }
    if (episode >= 3 * local_words || episode >= max_episodes) {
        return;
    }
    const std::uint8_t *genome = slab + individual * pitch;
    const std::size_t slot = individual * max_episodes + episode;
    auto &s = scratch[warp];
    if (lane == 0) {
        s.status = static_cast<int>(TryInitializeEpisodeGrid(tf::DeviceTrainingWordCatalog(), shards, shard_count,
                                                             shape, individual, episode, local_words, s.grid));
    }
    __syncwarp();
    if (s.status != 0) {
        if (lane == 0) {
            atomicCAS(status, 0, 100 + s.status);
        }
        return;
    }
    int step = 0;
    while (!s.grid.IsFinished()) {
        SelectedAction selected{};
        const DynamicInferenceStatusCode st = SelectNextGuessFromDynamicGenomeConcurrently<32>(
            s.grid, tf::DeviceTrainingWordCatalog(), genome, action_count, s.dynamic_policy, selected);
        if (st != DynamicInferenceStatusCode::kOk) {
            if (lane == 0) {
                atomicCAS(status, 0, 200 + static_cast<int>(st));
            }
            return;
        }
        if (policy_trace != nullptr) {
            for (int k = lane; k < 64; k += 32) {
                policy_trace[(slot * 6 + step) * 64 + k] = s.dynamic_policy.model.policy_vector[k];
            }
        }
        if (lane == 0) {
            choices[slot * 6 + step] = static_cast<int>(selected.action_index);
            s.status = neuroevolution::wordle::TryAppendGuess(s.grid, selected.word) ? 0 : 2;
        }
        __syncwarp();
        if (s.status != 0) {
            if (lane == 0) {
                atomicCAS(status, 0, 300);
            }
            return;
        }
        ++step;
    }
    if (lane == 0) {
        scores[slot] = ScoreCompletedEpisode(s.grid);
        turns[slot] = static_cast<int>(s.grid.turn_count);
    }
}

// evaluation_ops.cuh:171-237 with the shard walk replaced by a lookup in the individual's own word list:
// secret = list[e / 3]; variant 1 prefills list[(e/3 + 1) % W], list[(e/3 + 2) % W]; variant 2 the words at
// +3 and +4. The grid rules (MakeWordleGrid, TryAppendGuess) are the reference's.
__device__ bool InitializeCsrEpisode(const std::uint32_t *list, std::size_t w, std::size_t episode,
                                     neuroevolution::wordle::WordleGrid &grid) {
    const tf::TrainingWordCatalog &catalog = tf::DeviceTrainingWordCatalog();
    const std::size_t entry = episode / 3;
    const std::size_t variant = episode % 3;
    if (w == 0 || list[entry] >= catalog.word_count) {
        return false;
    }
    grid = neuroevolution::wordle::MakeWordleGrid(catalog.words[list[entry]]);
    if (variant == 0) {
        return true;
    }
    const std::size_t first = variant == 1 ? entry + 1 : entry + 3;
    const std::uint32_t a = list[first % w];
    const std::uint32_t b = list[(first + 1) % w];
    if (a >= catalog.word_count || b >= catalog.word_count) {
        return false;
    }
    return neuroevolution::wordle::TryAppendGuess(grid, catalog.words[a]) &&
           neuroevolution::wordle::TryAppendGuess(grid, catalog.words[b]);
}

// One warp per episode (slab_runtime.cu:452-549); individual i's genome at slab + slots[i] * pitch and its
// words at cell_words[cell_offsets[i] .. cell_offsets[i + 1]).
__global__ void EvaluateCsrKernel(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                  std::size_t population, std::size_t action_count,
                                  const std::uint32_t *cell_offsets, const std::uint32_t *cell_words,
                                  std::size_t max_episodes, float *scores, int *turns, int *choices,
                                  float *policy_trace, int *status) {
    __shared__ GenomeEvaluationWarpScratch<32> scratch[kWarps];
    const std::size_t individual = blockIdx.x;
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const std::size_t episode = static_cast<std::size_t>(blockIdx.y) * kWarps + warp;
    if (individual >= population) {
        return;
    }
    const std::size_t w = cell_offsets[individual + 1] - cell_offsets[individual];
    if (episode >= 3 * w || episode >= max_episodes) {
        return;
    }
    const std::uint8_t *genome = slab + static_cast<std::size_t>(slots[individual]) * pitch;
    const std::size_t slot = individual * max_episodes + episode;
    auto &s = scratch[warp];
    if (lane == 0) {
        s.status = InitializeCsrEpisode(cell_words + cell_offsets[individual], w, episode, s.grid) ? 0 : 1;
    }
    __syncwarp();
    if (s.status != 0) {
        if (lane == 0) {
            atomicCAS(status, 0, 101);
        }
        return;
    }
    int step = 0;
    while (!s.grid.IsFinished()) {
        SelectedAction selected{};
        const DynamicInferenceStatusCode st = SelectNextGuessFromDynamicGenomeConcurrently<32>(
            s.grid, tf::DeviceTrainingWordCatalog(), genome, action_count, s.dynamic_policy, selected);
        if (st != DynamicInferenceStatusCode::kOk) {
            if (lane == 0) {
                atomicCAS(status, 0, 200 + static_cast<int>(st));
            }
            return;
        }
        if (policy_trace != nullptr) {
            for (int k = lane; k < 64; k += 32) {
                policy_trace[(slot * 6 + step) * 64 + k] = s.dynamic_policy.model.policy_vector[k];
            }
        }
        if (lane == 0) {
            choices[slot * 6 + step] = static_cast<int>(selected.action_index);
            s.status = neuroevolution::wordle::TryAppendGuess(s.grid, selected.word) ? 0 : 2;
        }
        __syncwarp();
        if (s.status != 0) {
            if (lane == 0) {
                atomicCAS(status, 0, 300);
            }
            return;
        }
        ++step;
    }
    if (lane == 0) {
        scores[slot] = ScoreCompletedEpisode(s.grid);
        turns[slot] = static_cast<int>(s.grid.turn_count);
    }
}

__global__ void SelectKernel(const float *fitness, const std::uint8_t *has_fitness, std::size_t population,
                             std::size_t child_count, std::size_t columns, std::size_t generation_index,
                             ga::ParentSelectionConfig config, std::uint32_t planning_seed, std::uint32_t *pairs,
                             int *ok) {
    const std::size_t child = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (child >= child_count) {
        return;
    }
    CellularGridShape current{};
    CellularGridShape next{};
    if (!neuroevolution::spatial::TryMakeCellularGridShapeForColumnCount(population, columns, current) ||
        !neuroevolution::spatial::TryMakeCellularGridShapeForColumnCount(child_count, columns, next)) {
        ok[child] = 0;
        return;
    }
    auto state = ga::device_genome_ops::MakeDeviceRandomState(
        planning_seed, static_cast<std::uint32_t>(child + (generation_index * 8191U)));
    ga::ParentPair pair{};
    ok[child] = ga::device_selection_ops::TrySelectCellularParentPairDevice(fitness, has_fitness, current, next, child,
                                                                           state, config, pair)
                    ? 1
                    : 0;
    pairs[2 * child] = static_cast<std::uint32_t>(pair.first_parent_index);
    pairs[2 * child + 1] = static_cast<std::uint32_t>(pair.second_parent_index);
}

__global__ void BreedKernel(const std::uint8_t *parents, std::size_t parent_pitch, std::uint8_t *children,
                            std::size_t child_pitch, const std::uint32_t *pairs, std::size_t child_count,
                            std::size_t action_count, std::uint32_t generation_seed, std::size_t generation_index,
                            ga::BreedingConfig breeding, ga::MutationConfig mutation) {
    const std::size_t child = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (child >= child_count) {
        return;
    }
    auto state = ga::device_genome_ops::MakeDeviceRandomState(
        generation_seed, static_cast<std::uint32_t>(child + (generation_index * 4099U)));
    ga::device_genome_ops::BreedAndMutateGenome(parents + pairs[2 * child] * parent_pitch,
                                                parents + pairs[2 * child + 1] * parent_pitch, action_count,
                                                children + child * child_pitch, state, breeding, mutation);
}

__global__ void BootstrapKernel(std::uint8_t *slab, std::size_t pitch, std::size_t population,
                                std::size_t generation_index, std::uint32_t seed, std::size_t action_count) {
    const std::size_t organism = blockIdx.x;
    if (organism >= population) {
        return;
    }
    const std::uint64_t stream =
        ((static_cast<std::uint64_t>(generation_index) * population + organism) * blockDim.x) + threadIdx.x;
    auto state = ga::device_genome_ops::MakeDeviceRandomState(seed, stream);
    ga::device_genome_ops::InitializeRandomGenome(slab + organism * pitch, action_count, state, threadIdx.x,
                                                  blockDim.x);
}

__global__ void InjectKernel(std::uint8_t *genomes, std::size_t pitch, std::size_t count,
                             std::size_t parent_action_count, std::size_t first, std::size_t injection_count,
                             int *status) {
    __shared__ ga::OutputEmbeddingInjectionWarpScratch<32> scratch;
    const std::size_t genome = blockIdx.x;
    if (genome >= count) {
        return;
    }
    const auto result = ga::device_injection_ops::TryInjectExpandedOutputEmbeddingTailsConcurrently<32>(
        genomes + genome * pitch, parent_action_count, first, injection_count, scratch);
    if (threadIdx.x == 0) {
        status[genome] = static_cast<int>(result);
    }
}

} // namespace

extern "C" {

int refdev_upload_catalog(const std::uint8_t *letters, std::size_t count) {
    static tf::TrainingWordCatalog catalog{};
    catalog = {};
    if (count > tf::kTrainingWordCatalogCapacity) {
        return 0;
    }
    for (std::size_t w = 0; w < count; ++w) {
        for (std::size_t p = 0; p < 5; ++p) {
            catalog.words[w].letter_indices[p] = letters[5 * w + p];
        }
    }
    catalog.word_count = count;
    return tf::UploadTrainingWordCatalogToDeviceConstantMemory(catalog) ? 1 : 0;
}

// shards: host array of 48-byte TrainingDataShardRuntime records (training_data.hpp:35-42).
int refdev_evaluate(const void *slab, std::size_t pitch, std::size_t population, std::size_t columns,
                    std::size_t action_count, const void *host_shards, std::size_t shard_count,
                    std::size_t max_episodes, float *scores, int *turns, int *choices, float *policy_trace,
                    int *status, void *stream) {
    static_assert(sizeof(tf::TrainingDataShardRuntime) == 48, "shard record layout");
    tf::TrainingDataShardRuntime *shards = nullptr;
    if (cudaMalloc(&shards, shard_count * sizeof(*shards)) != cudaSuccess) {
        return 0;
    }
    cudaMemcpy(shards, host_shards, shard_count * sizeof(*shards), cudaMemcpyHostToDevice);
    CellularGridShape shape{};
    if (!neuroevolution::spatial::TryMakeCellularGridShapeForColumnCount(population, columns, shape)) {
        cudaFree(shards);
        return 0;
    }
    dim3 grid(static_cast<unsigned>(population), static_cast<unsigned>((max_episodes + kWarps - 1) / kWarps));
    EvaluateKernel<<<grid, 32 * kWarps, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const std::uint8_t *>(slab), pitch, population, action_count, shards, shard_count, shape,
        max_episodes, scores, turns, choices, policy_trace, status);
    const bool ok = cudaGetLastError() == cudaSuccess && cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) ==
                                                             cudaSuccess;
    cudaFree(shards);
    return ok ? 1 : 0;
}

// Explicit per-individual word lists; every pointer is a device pointer (policy_trace may be null).
int refdev_evaluate_csr(const void *slab, std::size_t pitch, const std::uint32_t *slots, std::size_t population,
                        std::size_t action_count, const std::uint32_t *cell_offsets, const std::uint32_t *cell_words,
                        std::size_t max_episodes, float *scores, int *turns, int *choices, float *policy_trace,
                        int *status, void *stream) {
    if (population == 0 || max_episodes == 0) {
        return 0;
    }
    dim3 grid(static_cast<unsigned>(population), static_cast<unsigned>((max_episodes + kWarps - 1) / kWarps));
    EvaluateCsrKernel<<<grid, 32 * kWarps, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const std::uint8_t *>(slab), pitch, slots, population, action_count, cell_offsets, cell_words,
        max_episodes, scores, turns, choices, policy_trace, status);
    return cudaGetLastError() == cudaSuccess &&
                   cudaStreamSynchronize(static_cast<cudaStream_t>(stream)) == cudaSuccess
               ? 1
               : 0;
}

int refdev_select(const float *fitness, const std::uint8_t *has_fitness, std::size_t population,
                  std::size_t child_count, std::size_t columns, std::size_t generation_index, std::size_t radius,
                  float rank_exponent, std::uint32_t planning_seed, std::uint32_t *pairs, int *ok, void *stream) {
    ga::ParentSelectionConfig config{};
    config.cellular_breeding_radius = radius;
    config.rank_exponent = rank_exponent;
    SelectKernel<<<static_cast<unsigned>((child_count + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        fitness, has_fitness, population, child_count, columns, generation_index, config, planning_seed, pairs, ok);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

int refdev_breed(const void *parents, std::size_t parent_pitch, void *children, std::size_t child_pitch,
                 const std::uint32_t *pairs, std::size_t child_count, std::size_t action_count,
                 std::uint32_t generation_seed, std::size_t generation_index, float l1, float l2, float l3,
                 float mutation_probability, float mutation_sigma, float row_scale_probability, void *stream) {
    ga::BreedingConfig breeding{};
    breeding.crossover_temperature_level1 = l1;
    breeding.crossover_temperature_level2 = l2;
    breeding.crossover_temperature_level3 = l3;
    ga::MutationConfig mutation{};
    mutation.mutation_probability = mutation_probability;
    mutation.mutation_sigma = mutation_sigma;
    mutation.output_tail_row_scale_mutation_probability = row_scale_probability;
    BreedKernel<<<static_cast<unsigned>((child_count + 31) / 32), 32, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<const std::uint8_t *>(parents), parent_pitch, static_cast<std::uint8_t *>(children), child_pitch,
        pairs, child_count, action_count, generation_seed, generation_index, breeding, mutation);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

int refdev_bootstrap(void *slab, std::size_t pitch, std::size_t population, std::size_t generation_index,
                     std::uint32_t seed, std::size_t action_count, void *stream) {
    BootstrapKernel<<<static_cast<unsigned>(population), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<std::uint8_t *>(slab), pitch, population, generation_index, seed, action_count);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

int refdev_inject(void *genomes, std::size_t pitch, std::size_t count, std::size_t parent_action_count,
                  std::size_t first, std::size_t injection_count, int *status, void *stream) {
    InjectKernel<<<static_cast<unsigned>(count), 32, 0, static_cast<cudaStream_t>(stream)>>>(
        static_cast<std::uint8_t *>(genomes), pitch, count, parent_action_count, first, injection_count, status);
    return cudaGetLastError() == cudaSuccess ? 1 : 0;
}

} // extern "C"
