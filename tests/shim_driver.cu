// Test program: a caller written against the reference's device GA runtime API
// (neuroevolution::genetic_algorithm::slab_device, slab_runtime.hpp:119-186), linked against libnwg.so through
// include/nwg_slab_device_shim.hpp. It walks the calls the reference's CLI makes (cli/run_genetic_algorithm.cu:
// catalog upload, create, bootstrap, evaluate, summary, advance with both callbacks, checkpoint with an
// asynchronous write then resume on the same buffers, restore from the file and resume) and prints what it saw,
// one "key value..." line each, for tests/test_shim.py to compare with the reference's own runtime.
//
// usage: shim_driver CATALOG_FILE ACTIONS INJECTED SLOTS POPULATION COLUMNS BOOT_SEED BOOT_INDEX SEED CHECKPOINT
//   CATALOG_FILE holds ACTIONS + INJECTED rows of 5 letter indices.
#define NWG_SLAB_DEVICE_SHIM_IMPLEMENTATION
#include "nwg_slab_device_shim.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace sd = neuroevolution::genetic_algorithm::slab_device;
namespace ga = neuroevolution::genetic_algorithm;
namespace gs = neuroevolution::genetic_algorithm::genotype_slab;
namespace tf = neuroevolution::training_folder;

namespace {

std::uint64_t Fnv(const std::uint8_t *bytes, std::size_t n) {
    std::uint64_t h = 1469598103934665603ULL;
    for (std::size_t i = 0; i < n; ++i) {
        h = (h ^ bytes[i]) * 1099511628211ULL;
    }
    return h;
}

// Prints the current generation: index, size, then one FNV-1a hash per individual's genome image.
bool PrintGeneration(const char *key, const sd::DeviceSlabGARuntimeBuffers &b) {
    gs::SlabGeneration g{};
    if (!sd::TryDownloadCurrentGenerationFromDevice(b, g)) {
        return false;
    }
    std::printf("%s %zu %zu", key, g.generation_index, g.active_individual_count);
    for (std::size_t i = 0; i < g.active_individual_count; ++i) {
        std::unique_ptr<std::uint8_t[]> bytes;
        std::size_t n = 0;
        if (!sd::TryDownloadSlabSlotBytesFromDevice(b, g.slot_indices[i], bytes, n)) {
            return false;
        }
        std::printf(" %016llx", static_cast<unsigned long long>(Fnv(bytes.get(), n)));
    }
    std::printf("\n");
    return true;
}

// RuntimeCheckpoint is move-only; the CLI hands the writer a clone (cli/run_genetic_algorithm.cu:1948-1953).
bool Clone(const sd::RuntimeCheckpoint &in, sd::RuntimeCheckpoint &out) {
    out = {};
    const gs::SlabGeneration &g = in.current_generation;
    if (!gs::TryCreateSlabGeneration(out.current_generation, g.active_individual_count, g.generation_index) ||
        !gs::TryCreateSlabAssemblyPlan(out.assembly_plan, in.assembly_plan.child_count)) {
        return false;
    }
    out.schema_version = in.schema_version;
    out.genome_layout_version = in.genome_layout_version;
    out.resume_phase = in.resume_phase;
    out.checksum = in.checksum;
    out.training_data_identity_hash = in.training_data_identity_hash;
    out.generation_seed = in.generation_seed;
    out.runtime_word_counts = in.runtime_word_counts;
    out.training_shard_release_history = in.training_shard_release_history;
    std::memcpy(static_cast<void *>(&out.assembly_config), &in.assembly_config, sizeof(in.assembly_config));
    std::memcpy(static_cast<void *>(&out.pending_output_embedding_injection), &in.pending_output_embedding_injection,
                sizeof(in.pending_output_embedding_injection));
    out.runtime_config = in.runtime_config;
    out.slab_layout = in.slab_layout;
    out.current_grid_shape = in.current_grid_shape;
    out.next_grid_shape = in.next_grid_shape;
    out.epicenter_grid_shape = in.epicenter_grid_shape;
    const std::size_t n = g.active_individual_count;
    std::memcpy(out.current_generation.slot_indices.get(), g.slot_indices.get(), n * sizeof(std::uint32_t));
    std::memcpy(out.current_generation.fitness.get(), g.fitness.get(), n * sizeof(float));
    std::memcpy(out.current_generation.evaluation_counts.get(), g.evaluation_counts.get(), n * sizeof(std::uint32_t));
    std::memcpy(out.current_generation.has_fitness.get(), g.has_fitness.get(), n);
    std::memcpy(out.assembly_plan.parent_pairs.get(), in.assembly_plan.parent_pairs.get(),
                in.assembly_plan.child_count * sizeof(gs::SlabParentPair));
    out.live_genotypes.resize(in.live_genotypes.size());
    for (std::size_t k = 0; k < in.live_genotypes.size(); ++k) {
        out.live_genotypes[k].organism_index = in.live_genotypes[k].organism_index;
        out.live_genotypes[k].genome_bytes = in.live_genotypes[k].genome_bytes;
    }
    return true;
}

int Fail(const char *what) {
    std::printf("FAIL %s\n", what);
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc != 11) {
        return Fail("usage");
    }
    const std::size_t actions = std::strtoull(argv[2], nullptr, 10);
    const std::size_t injected = std::strtoull(argv[3], nullptr, 10);
    const std::size_t slots = std::strtoull(argv[4], nullptr, 10);
    const std::size_t population = std::strtoull(argv[5], nullptr, 10);
    const std::size_t columns = std::strtoull(argv[6], nullptr, 10);
    const std::uint32_t boot_seed = static_cast<std::uint32_t>(std::strtoul(argv[7], nullptr, 10));
    const std::size_t boot_index = std::strtoull(argv[8], nullptr, 10);
    const std::uint32_t seed = static_cast<std::uint32_t>(std::strtoul(argv[9], nullptr, 10));
    const char *checkpoint_path = argv[10];

    static tf::TrainingWordCatalog catalog{};
    std::FILE *f = std::fopen(argv[1], "rb");
    if (f == nullptr) {
        return Fail("catalog file");
    }
    std::vector<std::uint8_t> letters((actions + injected) * 5);
    const bool read_ok = std::fread(letters.data(), 1, letters.size(), f) == letters.size();
    std::fclose(f);
    if (!read_ok) {
        return Fail("catalog read");
    }
    for (std::size_t w = 0; w < actions + injected; ++w) {
        for (std::size_t k = 0; k < 5; ++k) {
            catalog.words[w].letter_indices[k] = letters[w * 5 + k];
        }
    }
    catalog.word_count = actions + injected;
    if (!nwg_shim::UploadTrainingWordCatalog(catalog)) {
        return Fail("catalog upload");
    }

    const std::size_t stride = gs::ComputeSlabSlotStrideBytes(actions);
    sd::DeviceSlabGARuntimeConfig config{};
    config.genotype_slab_byte_budget_bytes = slots * stride;
    config.generation_byte_budget_bytes = population * stride;
    config.action_count = actions;
    config.population_size_ceiling = population;
    config.grid_column_count = columns;
    sd::DeviceSlabGARuntimeBuffers buffers{};
    if (!sd::TryCreateDeviceSlabGARuntimeBuffers(buffers, config) ||
        !sd::TryBootstrapRandomCurrentGenerationOnDevice(buffers, population, boot_seed, boot_index)) {
        return Fail("create/bootstrap");
    }
    std::printf("layout %zu %zu %zu %zu %zu\n", buffers.genotype_slab.slab_layout.action_count,
                buffers.genotype_slab.slab_layout.slot_stride_bytes, buffers.genotype_slab.slab_layout.slot_count,
                buffers.max_generation_size, buffers.grid_column_count);

    sd::RuntimeWordCounts counts{};
    counts.training_word_count = actions;
    counts.action_space_word_count = actions;
    counts.training_word_schedule.initial_word_count = actions;
    counts.training_word_schedule.word_count_step = 0;
    counts.training_word_schedule.word_count_step_period_generations = 1;
    if (!sd::TryEvaluateCurrentGenerationFitnessOnDevice(buffers, counts)) {
        return Fail("evaluate");
    }
    gs::SlabGeneration evaluated{};
    sd::PopulationFitnessSummary summary{};
    if (!sd::TryDownloadCurrentGenerationFromDevice(buffers, evaluated) ||
        !sd::TryReadPopulationFitnessSummaryFromDevice(buffers, summary)) {
        return Fail("download fitness");
    }
    std::printf("fitness");
    for (std::size_t i = 0; i < evaluated.active_individual_count; ++i) {
        std::uint32_t bits = 0;
        std::memcpy(&bits, &evaluated.fitness[i], 4);
        std::printf(" %08x", bits);
    }
    std::printf("\nsummary %a %a %zu %zu %zu\n", summary.best_fitness, summary.average_fitness, summary.best_index,
                summary.generation_index, summary.population_size);

    // one advance with both callbacks; the shard-release callback asks for the injection
    ga::GenerationAssemblyConfig assembly{};
    assembly.parent_selection.cellular_breeding_radius = 1;
    assembly.mutation.mutation_probability = 0.01f;
    assembly.mutation.mutation_sigma = 0.02f;
    int post_calls = 0, release_calls = 0;
    std::size_t seen_planned = 0;
    const sd::PostFitnessEvaluationCallback post = [&](const sd::DeviceSlabGARuntimeBuffers &b,
                                                       const sd::RuntimeWordCounts &) {
        ++post_calls;
        seen_planned = b.genotype_slab.planned_child_count;
        return true;
    };
    const sd::TrainingShardReleaseCallback release = [&](const sd::DeviceSlabGARuntimeBuffers &,
                                                         const sd::RuntimeWordCounts &,
                                                         sd::PendingOutputEmbeddingInjection &pending) {
        ++release_calls;
        if (injected > 0) {
            pending.enabled = true;
            pending.first_catalog_word_index = actions;
            pending.injection_count = injected;
        }
        return true;
    };
    if (!sd::TryAdvanceGenerationOnDevice(buffers, seed, counts, assembly, {}, false, post, release)) {
        return Fail("advance");
    }
    std::printf("callbacks %d %d %zu\n", post_calls, release_calls, seen_planned);
    std::printf("grown %zu\n", buffers.genotype_slab.slab_layout.action_count);
    if (!PrintGeneration("advanced", buffers)) {
        return Fail("advanced generation");
    }

    // checkpoint at the next boundary, write it asynchronously, resume on the same buffers
    sd::RuntimeWordCounts grown = counts;
    grown.action_space_word_count = buffers.genotype_slab.slab_layout.action_count;
    sd::RuntimeCheckpoint checkpoint{};
    if (!sd::TryCreatePrebreedingCheckpointOnDevice(buffers, seed + 1, grown, assembly, {}, checkpoint, &catalog)) {
        return Fail("checkpoint");
    }
    sd::RuntimeCheckpointAsyncWriter writer{};
    sd::RuntimeCheckpoint for_write{};
    if (!Clone(checkpoint, for_write) || !writer.TryStartWrite(std::move(for_write), checkpoint_path) ||
        !writer.TryWaitForWrite()) {
        return Fail("checkpoint write");
    }
    std::printf("checkpoint %zu %zu %zu %016llx\n", checkpoint.current_generation.generation_index,
                checkpoint.assembly_plan.child_count, checkpoint.live_genotypes.size(),
                static_cast<unsigned long long>(checkpoint.checksum));
    if (!sd::TryResumeGenerationFromCheckpointOnDevice(buffers, checkpoint) || !PrintGeneration("resumed", buffers)) {
        return Fail("resume");
    }

    sd::RuntimeCheckpoint loaded{};
    sd::DeviceSlabGARuntimeBuffers restored{};
    if (!sd::TryReadRuntimeCheckpoint(checkpoint_path, loaded) ||
        !sd::TryRestorePrebreedingCheckpointToDevice(loaded, restored) ||
        !sd::TryResumeGenerationFromCheckpointOnDevice(restored, loaded) || !PrintGeneration("restored", restored)) {
        return Fail("restore");
    }
    sd::DeviceSlabGARuntimeStatusCode status{};
    if (!sd::TryReadDeviceSlabGARuntimeStatus(restored, status)) {
        return Fail("status");
    }
    std::printf("status %d %s\n", static_cast<int>(status), sd::DeviceSlabGARuntimeStatusCodeString(status));
    sd::DestroyDeviceSlabGARuntimeBuffers(restored);
    sd::DestroyDeviceSlabGARuntimeBuffers(buffers);
    std::printf("ok\n");
    return 0;
}
