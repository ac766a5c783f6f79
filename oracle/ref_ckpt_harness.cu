// Test infrastructure only: the reference's runtime-checkpoint code (genetic_algorithm/device/slab_runtime.cu)
// and its device runtime, compiled from the reference's own sources where they lie, behind a small C ABI for the
// parity tests. Built by oracle/build.py into oracle/_ref/libref_ckpt.so; nothing from the reference is copied.
//
// Host-only entry points (no GPU needed):
//   refckpt_roundtrip      TryReadRuntimeCheckpoint then TryWriteRuntimeCheckpointAtomically
//   refckpt_write_synthetic a RuntimeCheckpoint of seeded content (padding bytes of the padded records set to 0xA5)
//                          sealed with ComputeRuntimeCheckpointChecksum and written by the reference writer
//   refckpt_identity_hash  the training-data identity hash, mixed by the reference's helpers in the order
//                          TryDownloadBoundaryCheckpointPayload uses (slab_runtime.cu:1283-1297)
//   refart_write / refart_read TryWriteWinnerArtifactToPaths / TryReadWinnerArtifact (model_artifact/)
//   refconv_plan / refconv_metrics MakeSamplePlan / TryComputeMetrics (genetic_algorithm/genetic_convergence.hpp)
//   refsm_select_many      TryCreateSingleModelDeviceRuntime + TrySelectNextGuessWithSingleModelDeviceRuntime per
//                          grid (GPU)
// Device entry points (drive the reference's whole runtime on the GPU):
//   refckpt_runtime_capture create, bootstrap, TryCreatePrebreedingCheckpointOnDevice, write
//   refckpt_runtime_evaluate create, bootstrap, TryEvaluateCurrentGenerationFitnessOnDevice, fitness arrays
//   refckpt_time_evaluation create, bootstrap, TryEvaluateCurrentGenerationFitnessOnDevice timed per call
//   refckpt_runtime_resume  read, TryRestorePrebreedingCheckpointToDevice, TryResumeGenerationFromCheckpointOnDevice,
//                          then the new generation's genomes in individual order
#include "genetic_algorithm/device/slab_runtime.cu"
#include "genetic_algorithm/genotype_slab/device_runtime.cu"
#include "genetic_algorithm/genotype_slab/slab_allocator.cpp"
#include "training_folder/training_data.cu"
#include "model_artifact/winner_artifact.cpp"
#include "model_artifact/winner_artifact_reader.cpp"
#include "genetic_algorithm/genetic_convergence.hpp"
#include "inference/single_model_device_runtime.cu"

#include <chrono>
#include <cstring>
#include <random>

namespace {

namespace sd = neuroevolution::genetic_algorithm::slab_device;
namespace ga = neuroevolution::genetic_algorithm;
namespace tf = neuroevolution::training_folder;
namespace gs = neuroevolution::genetic_algorithm::genotype_slab;

bool MakeCatalog(const std::uint8_t *letters, std::size_t count, tf::TrainingWordCatalog &catalog) {
    catalog = {};
    if (letters == nullptr || count == 0 || count > tf::kTrainingWordCatalogCapacity) {
        return false;
    }
    for (std::size_t w = 0; w < count; ++w) {
        for (std::size_t p = 0; p < 5; ++p) {
            catalog.words[w].letter_indices[p] = letters[w * 5 + p];
        }
    }
    catalog.word_count = count;
    return true;
}

}  // namespace

extern "C" {

// The reference's reader keeps reading after a failed check and can then size an allocation from misaligned
// bytes, which throws; a throw counts as a rejection here.
int refckpt_roundtrip(const char *in, const char *out) {
    try {
        sd::RuntimeCheckpoint c{};
        if (!sd::TryReadRuntimeCheckpoint(in, c)) {
            return 0;
        }
        return sd::TryWriteRuntimeCheckpointAtomically(c, out) ? 1 : 0;
    } catch (...) {
        return 0;
    }
}

int refckpt_write_synthetic(const char *path, std::uint32_t seed, std::size_t individuals, std::size_t children,
                            std::size_t action_count, std::size_t releases, int injection) {
    std::mt19937_64 rng(seed);
    const auto u = [&](std::uint64_t bound) { return static_cast<std::size_t>(rng() % bound); };
    sd::RuntimeCheckpoint c{};
    c.training_data_identity_hash = rng();
    c.generation_seed = static_cast<std::uint32_t>(rng());
    c.runtime_word_counts.training_word_count = u(5000);
    c.runtime_word_counts.action_space_word_count = u(5000);
    c.runtime_word_counts.training_word_schedule.initial_word_count = u(100);
    c.runtime_word_counts.training_word_schedule.word_count_step = u(100);
    c.runtime_word_counts.training_word_schedule.word_count_step_period_generations = u(100);
    c.runtime_word_counts.shard_initial_radius = u(10);
    c.runtime_word_counts.shard_radius_growth_period_generations = u(10);
    c.training_shard_release_history.release_count = releases;
    for (std::size_t i = 0; i < releases; ++i) {
        c.training_shard_release_history.release_generations[i] = u(1000);
        c.training_shard_release_history.release_fitness_p99[i] = static_cast<float>(u(1000)) / 1000.0f;
    }
    // padded records: non-zero padding, which the format carries as stored
    std::memset(static_cast<void *>(&c.assembly_config), 0xA5, sizeof(c.assembly_config));
    c.assembly_config.parent_selection.cellular_breeding_radius = 1 + u(3);
    c.assembly_config.parent_selection.rank_exponent = 0.5f;
    c.assembly_config.breeding.crossover_temperature_level1 = 0.02f;
    c.assembly_config.breeding.crossover_temperature_level2 = 0.01f;
    c.assembly_config.breeding.crossover_temperature_level3 = 0.005f;
    c.assembly_config.mutation.mutation_probability = 0.001f;
    c.assembly_config.mutation.mutation_sigma = 0.02f;
    c.assembly_config.mutation.output_tail_row_scale_mutation_probability = 0.0f;
    std::memset(static_cast<void *>(&c.pending_output_embedding_injection), 0xA5,
                sizeof(c.pending_output_embedding_injection));
    c.pending_output_embedding_injection.enabled = injection != 0;
    c.pending_output_embedding_injection.first_catalog_word_index = injection != 0 ? action_count - 3 : 0;
    c.pending_output_embedding_injection.injection_count = injection != 0 ? 3 : 0;
    const std::size_t stride = gs::ComputeSlabSlotStrideBytes(action_count);
    c.slab_layout.action_count = action_count;
    c.slab_layout.slot_stride_bytes = stride;
    c.slab_layout.slot_count = 2 * individuals;
    c.slab_layout.slab_bytes = 2 * individuals * stride;
    c.runtime_config.genotype_slab_byte_budget_bytes = c.slab_layout.slab_bytes;
    c.runtime_config.generation_byte_budget_bytes = individuals * stride;
    c.runtime_config.action_count = action_count;
    c.runtime_config.population_size_ceiling = individuals;
    c.runtime_config.grid_column_count = 4;
    c.current_grid_shape = {individuals / 4, 4, individuals};
    c.next_grid_shape = {children / 4, 4, children};
    c.epicenter_grid_shape = {individuals / 4, 4, individuals};
    if (!gs::TryCreateSlabGeneration(c.current_generation, individuals, u(50)) ||
        !gs::TryCreateSlabAssemblyPlan(c.assembly_plan, children)) {
        return 0;
    }
    for (std::size_t i = 0; i < individuals; ++i) {
        const bool live = u(4) != 0;
        c.current_generation.slot_indices[i] = live ? static_cast<std::uint32_t>(i) : gs::kInvalidSlabSlotIndex;
        c.current_generation.fitness[i] = static_cast<float>(u(100000)) / 100000.0f;
        c.current_generation.evaluation_counts[i] = static_cast<std::uint32_t>(u(40));
        c.current_generation.has_fitness[i] = static_cast<std::uint8_t>(u(2));
        if (live) {
            sd::RuntimeCheckpointGenotypeRecord record{};
            record.organism_index = static_cast<std::uint32_t>(i);
            record.genome_bytes.resize(stride);
            for (std::size_t b = 0; b < stride; ++b) {
                record.genome_bytes[b] = static_cast<std::uint8_t>(rng());
            }
            c.live_genotypes.push_back(std::move(record));
        }
    }
    for (std::size_t k = 0; k < children; ++k) {
        c.assembly_plan.parent_pairs[k].first_parent_index = static_cast<std::uint32_t>(u(individuals));
        c.assembly_plan.parent_pairs[k].second_parent_index = static_cast<std::uint32_t>(u(individuals));
    }
    c.checksum = sd::ComputeRuntimeCheckpointChecksum(c);
    return sd::TryWriteRuntimeCheckpointAtomically(c, path) ? 1 : 0;
}

std::uint64_t refckpt_identity_hash(const void *counts, const void *history, const std::uint8_t *letters,
                                    std::size_t count) {
    std::uint64_t hash = 1469598103934665603ULL;
    sd::MixCheckpointBytes(hash, counts, sizeof(sd::RuntimeWordCounts));
    if (history != nullptr) {
        sd::MixTrainingShardReleaseHistory(hash, *static_cast<const tf::TrainingDataShardReleaseHistory *>(history));
    }
    if (letters != nullptr) {
        static tf::TrainingWordCatalog catalog{};
        if (!MakeCatalog(letters, count, catalog)) {
            return 0;
        }
        sd::MixCheckpointValue(hash, catalog.word_count);
        for (std::size_t w = 0; w < catalog.word_count; ++w) {
            sd::MixCheckpointBytes(hash, &catalog.words[w], sizeof(catalog.words[w]));
        }
    }
    return hash;
}

// meta: best_fitness (float bits in u64), generation_index, best_index, best_slot_index, action_count,
// genome_byte_count, seed
int refart_write(const char *binary_path, const char *metadata_path, const std::uint8_t *genome,
                 const std::uint8_t *letters, std::size_t catalog_count, const std::uint64_t *meta,
                 const char *action_space_path) {
    try {
        static tf::TrainingWordCatalog catalog{};
        if (!MakeCatalog(letters, catalog_count, catalog)) {
            return 0;
        }
        neuroevolution::model_artifact::WinnerArtifactMetadata m{};
        std::uint32_t bits = static_cast<std::uint32_t>(meta[0]);
        std::memcpy(&m.best_fitness, &bits, 4);
        m.generation_index = meta[1];
        m.best_index = meta[2];
        m.best_slot_index = static_cast<std::uint32_t>(meta[3]);
        m.action_count = meta[4];
        m.genome_byte_count = meta[5];
        m.seed = static_cast<std::uint32_t>(meta[6]);
        m.action_space_path = action_space_path;
        neuroevolution::model_artifact::WinnerArtifactPaths paths{};
        return neuroevolution::model_artifact::TryWriteWinnerArtifactToPaths(binary_path, metadata_path, genome,
                                                                             catalog, m, paths)
                   ? 1
                   : 0;
    } catch (...) {
        return 0;
    }
}

int refart_read(const char *binary_path, const char *metadata_path, std::uint64_t *meta, std::uint8_t *genome,
                std::size_t capacity, std::uint8_t *letters, std::size_t *catalog_count, char *path_out,
                std::size_t path_capacity) {
    try {
        neuroevolution::model_artifact::LoadedWinnerArtifact a{};
        if (!neuroevolution::model_artifact::TryReadWinnerArtifact(binary_path, metadata_path, a) ||
            a.metadata.genome_byte_count > capacity) {
            return 0;
        }
        std::uint32_t bits = 0;
        std::memcpy(&bits, &a.metadata.best_fitness, 4);
        meta[0] = bits;
        meta[1] = a.metadata.generation_index;
        meta[2] = a.metadata.best_index;
        meta[3] = a.metadata.best_slot_index;
        meta[4] = a.metadata.action_count;
        meta[5] = a.metadata.genome_byte_count;
        meta[6] = a.metadata.seed;
        std::memcpy(genome, a.genome_bytes.get(), a.metadata.genome_byte_count);
        for (std::size_t w = 0; w < a.action_space_words.word_count; ++w) {
            for (std::size_t k = 0; k < 5; ++k) {
                letters[w * 5 + k] = a.action_space_words.words[w].letter_indices[k];
            }
        }
        *catalog_count = a.action_space_words.word_count;
        const std::string path = a.metadata.action_space_path.string();
        if (path.size() + 1 > path_capacity) {
            return 0;
        }
        std::memcpy(path_out, path.c_str(), path.size() + 1);
        return 1;
    } catch (...) {
        return 0;
    }
}

int refconv_plan(std::size_t organisms, std::size_t trainable, std::uint32_t seed, std::size_t generation,
                 std::uint64_t *org_out, std::size_t *n_org, std::uint64_t *w_out, std::size_t *n_w,
                 std::uint64_t *pairs_out, std::size_t *n_pairs) {
    namespace gc = neuroevolution::genetic_algorithm::genetic_convergence;
    const gc::GeneticConvergenceSamplePlan plan = gc::MakeSamplePlan(organisms, trainable, seed, generation);
    for (std::size_t i = 0; i < plan.organism_indices.size(); ++i) {
        org_out[i] = plan.organism_indices[i];
    }
    for (std::size_t i = 0; i < plan.weight_indices.size(); ++i) {
        w_out[i] = plan.weight_indices[i];
    }
    for (std::size_t i = 0; i < plan.pairs.size(); ++i) {
        pairs_out[2 * i] = plan.pairs[i].first;
        pairs_out[2 * i + 1] = plan.pairs[i].second;
    }
    *n_org = plan.organism_indices.size();
    *n_w = plan.weight_indices.size();
    *n_pairs = plan.pairs.size();
    return 1;
}

// out: centroid mean, min, max, pairwise mean, min, max
int refconv_metrics(const float *values, std::size_t organisms, std::size_t weights, const std::uint64_t *pairs,
                    std::size_t pair_count, float *out) {
    namespace gc = neuroevolution::genetic_algorithm::genetic_convergence;
    std::vector<float> v(values, values + organisms * weights);
    std::vector<gc::GeneticConvergencePair> p(pair_count);
    for (std::size_t i = 0; i < pair_count; ++i) {
        p[i].first = pairs[2 * i];
        p[i].second = pairs[2 * i + 1];
    }
    gc::GeneticConvergenceMetrics m{};
    if (!gc::TryComputeMetrics(v, organisms, weights, p, m)) {
        return 0;
    }
    out[0] = m.centroid_distance_mean;
    out[1] = m.centroid_distance_min;
    out[2] = m.centroid_distance_max;
    out[3] = m.pairwise_distance_mean;
    out[4] = m.pairwise_distance_min;
    out[5] = m.pairwise_distance_max;
    return 1;
}

// grids: guesses[n][6][5], feedback[n][6][5] (0 green, 1 yellow, 2 grey), turns[n]; per grid the reference's
// status, action index and score.
int refsm_select_many(const std::uint8_t *genome, std::size_t genome_bytes, const std::uint8_t *letters,
                      std::size_t catalog_count, const std::uint8_t *guesses, const std::uint8_t *feedback,
                      const std::uint8_t *turns, std::size_t n, int *status, std::uint64_t *index, float *score) {
    namespace inf = neuroevolution::inference;
    namespace wd = neuroevolution::wordle;
    static tf::TrainingWordCatalog catalog{};
    if (!MakeCatalog(letters, catalog_count, catalog)) {
        return 0;
    }
    inf::SingleModelDeviceRuntime runtime{};
    if (!inf::TryCreateSingleModelDeviceRuntime(genome, genome_bytes, catalog, runtime)) {
        return 0;
    }
    for (std::size_t g = 0; g < n; ++g) {
        wd::WordleGrid grid{};
        grid.turn_count = turns[g];
        for (std::size_t u = 0; u < turns[g] && u < wd::kMaxTurnCount; ++u) {
            for (std::size_t k = 0; k < 5; ++k) {
                grid.turns[u].guess.letter_indices[k] = guesses[(g * 6 + u) * 5 + k];
                grid.turns[u].feedback.values[k] = static_cast<wd::TileFeedback>(feedback[(g * 6 + u) * 5 + k]);
            }
        }
        neuroevolution::model::output_embedding::SelectedAction action{};
        inf::SingleModelDeviceRuntimeStatusCode st = inf::SingleModelDeviceRuntimeStatusCode::kInvalidRuntime;
        (void)inf::TrySelectNextGuessWithSingleModelDeviceRuntime(runtime, grid, action, &st);
        status[g] = static_cast<int>(st);
        index[g] = action.action_index;
        score[g] = action.score;
    }
    inf::DestroySingleModelDeviceRuntime(runtime);
    return 1;
}

// Records the POD layouts the C ABI relies on.
int refckpt_layouts(std::size_t *out) {
    out[0] = sizeof(sd::RuntimeWordCounts);
    out[1] = sizeof(tf::TrainingDataShardReleaseHistory);
    out[2] = sizeof(ga::GenerationAssemblyConfig);
    out[3] = sizeof(sd::PendingOutputEmbeddingInjection);
    out[4] = sizeof(sd::DeviceSlabGARuntimeConfig);
    out[5] = sizeof(gs::GenotypeSlabLayout);
    out[6] = sizeof(neuroevolution::spatial::CellularGridShape);
    out[7] = sizeof(neuroevolution::wordle::Word);
    return 8;
}

int refckpt_runtime_capture(const void *config, const std::uint8_t *letters, std::size_t catalog_count,
                            std::size_t generation_size, std::uint32_t bootstrap_seed, std::size_t generation_index,
                            std::uint32_t generation_seed,
                            const void *counts, const void *assembly, const void *pending, const void *history,
                            int hash_catalog, const char *path) {
    tf::TrainingWordCatalog *catalog = new tf::TrainingWordCatalog{};
    if (!MakeCatalog(letters, catalog_count, *catalog) || !tf::UploadTrainingWordCatalogToDeviceConstantMemory(*catalog)) {
        delete catalog;
        return 0;
    }
    sd::DeviceSlabGARuntimeBuffers buffers{};
    sd::RuntimeCheckpoint checkpoint{};
    const auto *h = static_cast<const tf::TrainingDataShardReleaseHistory *>(history);
    bool ok = sd::TryCreateDeviceSlabGARuntimeBuffers(buffers, *static_cast<const sd::DeviceSlabGARuntimeConfig *>(config)) &&
              sd::TryBootstrapRandomCurrentGenerationOnDevice(buffers, generation_size, bootstrap_seed, generation_index) &&
              sd::TryCreatePrebreedingCheckpointOnDevice(
                  buffers, generation_seed, *static_cast<const sd::RuntimeWordCounts *>(counts),
                  *static_cast<const ga::GenerationAssemblyConfig *>(assembly),
                  *static_cast<const sd::PendingOutputEmbeddingInjection *>(pending), checkpoint,
                  hash_catalog != 0 ? catalog : nullptr, false, {}, {}, h) &&
              sd::TryWriteRuntimeCheckpointAtomically(checkpoint, path);
    sd::DestroyDeviceSlabGARuntimeBuffers(buffers);
    delete catalog;
    return ok ? 1 : 0;
}

// TryCreateDeviceSlabGARuntimeBuffers, TryBootstrapRandomCurrentGenerationOnDevice,
// TryEvaluateCurrentGenerationFitnessOnDevice, then the generation's fitness arrays and the summary.
int refckpt_runtime_evaluate(const void *config, const std::uint8_t *letters, std::size_t catalog_count,
                             std::size_t generation_size, std::uint32_t bootstrap_seed, std::size_t generation_index,
                             const void *counts, const void *history, float *fitness, std::uint32_t *evaluation_counts,
                             std::uint8_t *has_fitness, void *summary) {
    tf::TrainingWordCatalog *catalog = new tf::TrainingWordCatalog{};
    const bool have_catalog =
        MakeCatalog(letters, catalog_count, *catalog) && tf::UploadTrainingWordCatalogToDeviceConstantMemory(*catalog);
    delete catalog;
    if (!have_catalog) {
        return 0;
    }
    sd::DeviceSlabGARuntimeBuffers buffers{};
    gs::SlabGeneration generation{};
    sd::PopulationFitnessSummary s{};
    bool ok = sd::TryCreateDeviceSlabGARuntimeBuffers(buffers, *static_cast<const sd::DeviceSlabGARuntimeConfig *>(config)) &&
              sd::TryBootstrapRandomCurrentGenerationOnDevice(buffers, generation_size, bootstrap_seed, generation_index) &&
              sd::TryEvaluateCurrentGenerationFitnessOnDevice(
                  buffers, *static_cast<const sd::RuntimeWordCounts *>(counts),
                  static_cast<const tf::TrainingDataShardReleaseHistory *>(history)) &&
              sd::TryDownloadCurrentGenerationFromDevice(buffers, generation) &&
              sd::TryReadPopulationFitnessSummaryFromDevice(buffers, s);
    for (std::size_t i = 0; ok && i < generation.active_individual_count; ++i) {
        fitness[i] = generation.fitness[i];
        evaluation_counts[i] = generation.evaluation_counts[i];
        has_fitness[i] = generation.has_fitness[i];
    }
    if (ok) {
        std::memcpy(summary, &s, sizeof(s));
    }
    sd::DestroyDeviceSlabGARuntimeBuffers(buffers);
    return ok ? 1 : 0;
}

// The reference's evaluation timed through its public API: create, bootstrap, then `repeats` calls of
// TryEvaluateCurrentGenerationFitnessOnDevice (each synchronises the device before it returns), each timed on the
// host clock around the call; ms_out[r] is call r's time, then the fitness of the last call.
int refckpt_time_evaluation(const void *config, const std::uint8_t *letters, std::size_t catalog_count,
                            std::size_t generation_size, std::uint32_t bootstrap_seed, std::size_t generation_index,
                            const void *counts, std::size_t repeats, double *ms_out, float *fitness) {
    tf::TrainingWordCatalog *catalog = new tf::TrainingWordCatalog{};
    const bool have_catalog =
        MakeCatalog(letters, catalog_count, *catalog) && tf::UploadTrainingWordCatalogToDeviceConstantMemory(*catalog);
    delete catalog;
    if (!have_catalog) {
        return 0;
    }
    sd::DeviceSlabGARuntimeBuffers buffers{};
    gs::SlabGeneration generation{};
    bool ok = sd::TryCreateDeviceSlabGARuntimeBuffers(buffers, *static_cast<const sd::DeviceSlabGARuntimeConfig *>(config)) &&
              sd::TryBootstrapRandomCurrentGenerationOnDevice(buffers, generation_size, bootstrap_seed, generation_index);
    for (std::size_t r = 0; ok && r < repeats; ++r) {
        const auto t0 = std::chrono::steady_clock::now();
        ok = sd::TryEvaluateCurrentGenerationFitnessOnDevice(buffers, *static_cast<const sd::RuntimeWordCounts *>(counts),
                                                             nullptr) &&
             cudaDeviceSynchronize() == cudaSuccess;
        const auto t1 = std::chrono::steady_clock::now();
        ms_out[r] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    }
    ok = ok && sd::TryDownloadCurrentGenerationFromDevice(buffers, generation);
    for (std::size_t i = 0; ok && i < generation.active_individual_count; ++i) {
        fitness[i] = generation.fitness[i];
    }
    sd::DestroyDeviceSlabGARuntimeBuffers(buffers);
    return ok ? 1 : 0;
}

int refckpt_runtime_resume(const char *path, const std::uint8_t *letters, std::size_t catalog_count,
                           std::uint8_t *genomes, std::size_t capacity_bytes, std::size_t *count_out,
                           std::size_t *stride_out) {
    tf::TrainingWordCatalog *catalog = new tf::TrainingWordCatalog{};
    const bool have_catalog =
        MakeCatalog(letters, catalog_count, *catalog) && tf::UploadTrainingWordCatalogToDeviceConstantMemory(*catalog);
    delete catalog;
    if (!have_catalog) {
        return 0;
    }
    sd::RuntimeCheckpoint checkpoint{};
    sd::DeviceSlabGARuntimeBuffers buffers{};
    gs::SlabGeneration generation{};
    bool ok = sd::TryReadRuntimeCheckpoint(path, checkpoint) &&
              sd::TryRestorePrebreedingCheckpointToDevice(checkpoint, buffers) &&
              sd::TryResumeGenerationFromCheckpointOnDevice(buffers, checkpoint, false) &&
              sd::TryDownloadCurrentGenerationFromDevice(buffers, generation);
    std::size_t stride = 0;
    if (ok) {
        stride = buffers.genotype_slab.slab_layout.slot_stride_bytes;
        ok = generation.active_individual_count * stride <= capacity_bytes;
    }
    for (std::size_t i = 0; ok && i < generation.active_individual_count; ++i) {
        std::unique_ptr<std::uint8_t[]> bytes;
        std::size_t n = 0;
        ok = sd::TryDownloadSlabSlotBytesFromDevice(buffers, generation.slot_indices[i], bytes, n) && n == stride;
        if (ok) {
            std::memcpy(genomes + i * stride, bytes.get(), stride);
        }
    }
    *count_out = ok ? generation.active_individual_count : 0;
    *stride_out = stride;
    sd::DestroyDeviceSlabGARuntimeBuffers(buffers);
    return ok ? 1 : 0;
}

}  // extern "C"
