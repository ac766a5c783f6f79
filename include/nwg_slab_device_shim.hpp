// nwg_slab_device_shim.hpp -- the reference's device GA runtime API implemented on this library's C ABI.
//
// The reference's callers (its CLI and tests) program against neuroevolution::genetic_algorithm::slab_device
// (src/genetic_algorithm/device/slab_runtime.hpp:119-186). This header keeps those declarations (it includes the
// reference's slab_runtime.hpp) and supplies their definitions on top of nwg_capi.h, so the callers link against
// libnwg.so instead of the reference's slab_runtime.cu without a source change.
//
// Single header: include it where the declarations are needed; in exactly one translation unit define
// NWG_SLAB_DEVICE_SHIM_IMPLEMENTATION before including it, and link that unit with libnwg.so in place of
// slab_runtime.cu. The reference's host-side genotype_slab code (slab_allocator.cpp) stays linked as before.
//
// How the reference's objects map onto the runtime:
//   - the runtime handle rides in DeviceSlabGARuntimeBuffers::status (the reference's device status int*, read
//     only by the runtime itself). Each call refreshes the buffers' host-side fields from nwg_get_info (slab
//     layout, generation indices and sizes, planned children, budgets, epicenter shape), so code reading them
//     sees the reference's values.
//   - the reference's device pointers stay null: slots sit at a 256-byte pitch, so genome images are read with
//     TryDownloadSlabSlotBytesFromDevice or TryDownloadSlabFromDevice, never by address.
//   - std::function callbacks run through C trampolines with the caller's buffers object; an exception from a
//     callback counts as a false return. The verbose flags print nothing.
//   - RuntimeCheckpoint converts to and from nwg_checkpoint field for field; files are the same bytes.
#pragma once

#include <chrono>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <future>
#include <memory>
#include <utility>
#include <vector>

#include "genetic_algorithm/device/slab_runtime.hpp"
#include "nwg_capi.h"

namespace nwg_shim {

// The one line a caller adds beside UploadTrainingWordCatalogToDeviceConstantMemory (cli/run_genetic_algorithm.cu:1579,
// and the tests' catalog set-up): the runtime evaluates with its own device copy of the catalog.
inline bool UploadTrainingWordCatalog(const neuroevolution::training_folder::TrainingWordCatalog &catalog) {
    static_assert(sizeof(neuroevolution::wordle::Word) == 5, "a catalog word is 5 letter indices");
    return nwg_upload_catalog(reinterpret_cast<const std::uint8_t *>(&catalog.words[0]), catalog.word_count) == NWG_OK;
}

}  // namespace nwg_shim

#ifdef NWG_SLAB_DEVICE_SHIM_IMPLEMENTATION

namespace neuroevolution::genetic_algorithm::slab_device {

static_assert(sizeof(DeviceSlabGARuntimeConfig) == sizeof(nwg_runtime_config));
static_assert(sizeof(RuntimeWordCounts) == sizeof(nwg_runtime_word_counts));
static_assert(sizeof(training_folder::TrainingDataShardReleaseHistory) == sizeof(nwg_shard_release_history));
static_assert(sizeof(GenerationAssemblyConfig) == sizeof(nwg_generation_assembly_config));
static_assert(sizeof(PendingOutputEmbeddingInjection) == sizeof(nwg_pending_injection));
static_assert(sizeof(PopulationFitnessSummary) == sizeof(nwg_fitness_summary));
static_assert(sizeof(genotype_slab::GenotypeSlabLayout) == sizeof(nwg_slab_layout));
static_assert(sizeof(::neuroevolution::spatial::CellularGridShape) == sizeof(nwg_grid_shape));
static_assert(sizeof(genotype_slab::SlabParentPair) == 2 * sizeof(std::uint32_t));
static_assert(sizeof(wordle::Word) == 5);
static_assert(offsetof(PopulationFitnessSummary, best_slot_index) == offsetof(nwg_fitness_summary, best_slot_index));
static_assert(offsetof(PendingOutputEmbeddingInjection, injection_count) ==
              offsetof(nwg_pending_injection, injection_count));
static_assert(offsetof(RuntimeWordCounts, shard_radius_growth_period_generations) ==
              offsetof(nwg_runtime_word_counts, shard_radius_growth_period_generations));
static_assert(offsetof(training_folder::TrainingDataShardReleaseHistory, release_count) ==
              offsetof(nwg_shard_release_history, release_count));

namespace {

nwg_runtime *ShimHandle(const DeviceSlabGARuntimeBuffers &b) { return reinterpret_cast<nwg_runtime *>(b.status); }

void ShimMirror(DeviceSlabGARuntimeBuffers &b) {
    nwg_runtime_info i{};
    if (ShimHandle(b) == nullptr || nwg_get_info(ShimHandle(b), &i) != NWG_OK) {
        return;
    }
    genotype_slab::device::DeviceSlabRuntimeBuffers &g = b.genotype_slab;
    g.slab_layout.action_count = i.action_count;
    g.slab_layout.slot_stride_bytes = i.slot_stride_bytes;
    g.slab_layout.slot_count = i.slot_count;
    g.slab_layout.slab_bytes = i.slab_bytes;
    g.max_generation_size = i.max_generation_size;
    g.current_generation_index = i.current_generation_index;
    g.current_generation_size = i.current_generation_size;
    g.next_generation_index = i.next_generation_index;
    g.next_generation_size = i.next_generation_size;
    g.planned_child_count = i.planned_child_count;
    b.max_generation_size = i.max_generation_size;
    b.generation_byte_budget_bytes = i.generation_byte_budget_bytes;
    b.host_spillover_byte_budget_bytes = i.host_spillover_byte_budget_bytes;
    b.grid_column_count = i.grid_column_count;
    b.epicenter_grid_shape.row_count = i.epicenter_row_count;
    b.epicenter_grid_shape.column_count = i.grid_column_count;
    b.epicenter_grid_shape.cell_count = i.epicenter_row_count * i.grid_column_count;
    b.active_training_shard_capacity = NWG_CATALOG_CAPACITY;
}

struct ShimCallbacks {
    DeviceSlabGARuntimeBuffers *buffers;
    const PostFitnessEvaluationCallback *post_fitness;
    const TrainingShardReleaseCallback *shard_release;
};

bool ShimPostFitness(nwg_runtime *, const nwg_runtime_word_counts *counts, void *user) {
    auto *c = static_cast<ShimCallbacks *>(user);
    try {
        ShimMirror(*c->buffers);
        return (*c->post_fitness)(*c->buffers, *reinterpret_cast<const RuntimeWordCounts *>(counts));
    } catch (...) {
        return false;
    }
}

bool ShimShardRelease(nwg_runtime *, const nwg_runtime_word_counts *counts, nwg_pending_injection *pending,
                      void *user) {
    auto *c = static_cast<ShimCallbacks *>(user);
    try {
        ShimMirror(*c->buffers);
        return (*c->shard_release)(*c->buffers, *reinterpret_cast<const RuntimeWordCounts *>(counts),
                                   *reinterpret_cast<PendingOutputEmbeddingInjection *>(pending));
    } catch (...) {
        return false;
    }
}

// nwg_checkpoint views of a RuntimeCheckpoint: the scalars are copied, the arrays point into the checkpoint and
// into two staging vectors for the genotype records.
struct ShimCheckpointView {
    nwg_checkpoint c{};
    std::vector<std::uint32_t> organisms;
    std::vector<std::uint8_t> genomes;
};

bool ShimToC(const RuntimeCheckpoint &r, ShimCheckpointView &v) {
    nwg_checkpoint &c = v.c;
    std::memset(&c, 0, sizeof(c));
    c.schema_version = r.schema_version;
    c.genome_layout_version = r.genome_layout_version;
    c.resume_phase = static_cast<std::uint32_t>(r.resume_phase);
    c.checksum = r.checksum;
    c.training_data_identity_hash = r.training_data_identity_hash;
    c.generation_seed = r.generation_seed;
    std::memcpy(&c.runtime_word_counts, &r.runtime_word_counts, sizeof(c.runtime_word_counts));
    std::memcpy(&c.training_shard_release_history, &r.training_shard_release_history,
                sizeof(c.training_shard_release_history));
    std::memcpy(&c.assembly_config, &r.assembly_config, sizeof(c.assembly_config));
    std::memcpy(&c.pending_output_embedding_injection, &r.pending_output_embedding_injection,
                sizeof(c.pending_output_embedding_injection));
    std::memcpy(&c.runtime_config, &r.runtime_config, sizeof(c.runtime_config));
    std::memcpy(&c.slab_layout, &r.slab_layout, sizeof(c.slab_layout));
    std::memcpy(&c.current_grid_shape, &r.current_grid_shape, sizeof(c.current_grid_shape));
    std::memcpy(&c.next_grid_shape, &r.next_grid_shape, sizeof(c.next_grid_shape));
    std::memcpy(&c.epicenter_grid_shape, &r.epicenter_grid_shape, sizeof(c.epicenter_grid_shape));
    c.generation_index = r.current_generation.generation_index;
    c.individual_count = r.current_generation.active_individual_count;
    c.slot_indices = r.current_generation.slot_indices.get();
    c.fitness = r.current_generation.fitness.get();
    c.evaluation_counts = r.current_generation.evaluation_counts.get();
    c.has_fitness = r.current_generation.has_fitness.get();
    c.child_count = r.assembly_plan.child_count;
    c.parent_pairs = reinterpret_cast<std::uint32_t *>(r.assembly_plan.parent_pairs.get());
    const std::size_t stride = r.slab_layout.slot_stride_bytes;
    v.organisms.resize(r.live_genotypes.size());
    v.genomes.assign(r.live_genotypes.size() * stride, 0);
    for (std::size_t k = 0; k < r.live_genotypes.size(); ++k) {
        if (r.live_genotypes[k].genome_bytes.size() != stride) {
            return false;
        }
        v.organisms[k] = r.live_genotypes[k].organism_index;
        std::memcpy(v.genomes.data() + k * stride, r.live_genotypes[k].genome_bytes.data(), stride);
    }
    c.live_count = r.live_genotypes.size();
    c.live_organisms = v.organisms.data();
    c.live_genomes = v.genomes.data();
    return true;
}

bool ShimFromC(const nwg_checkpoint &c, RuntimeCheckpoint &r) {
    r = {};
    r.schema_version = c.schema_version;
    r.genome_layout_version = c.genome_layout_version;
    r.resume_phase = static_cast<RuntimeCheckpointResumePhase>(c.resume_phase);
    r.checksum = c.checksum;
    r.training_data_identity_hash = c.training_data_identity_hash;
    r.generation_seed = c.generation_seed;
    std::memcpy(&r.runtime_word_counts, &c.runtime_word_counts, sizeof(c.runtime_word_counts));
    std::memcpy(&r.training_shard_release_history, &c.training_shard_release_history,
                sizeof(c.training_shard_release_history));
    std::memcpy(&r.assembly_config, &c.assembly_config, sizeof(c.assembly_config));
    std::memcpy(&r.pending_output_embedding_injection, &c.pending_output_embedding_injection,
                sizeof(c.pending_output_embedding_injection));
    std::memcpy(&r.runtime_config, &c.runtime_config, sizeof(c.runtime_config));
    std::memcpy(&r.slab_layout, &c.slab_layout, sizeof(c.slab_layout));
    std::memcpy(&r.current_grid_shape, &c.current_grid_shape, sizeof(c.current_grid_shape));
    std::memcpy(&r.next_grid_shape, &c.next_grid_shape, sizeof(c.next_grid_shape));
    std::memcpy(&r.epicenter_grid_shape, &c.epicenter_grid_shape, sizeof(c.epicenter_grid_shape));
    if (!genotype_slab::TryCreateSlabGeneration(r.current_generation, c.individual_count, c.generation_index) ||
        !genotype_slab::TryCreateSlabAssemblyPlan(r.assembly_plan, c.child_count)) {
        r = {};
        return false;
    }
    const std::size_t n = c.individual_count;
    std::memcpy(r.current_generation.slot_indices.get(), c.slot_indices, n * sizeof(std::uint32_t));
    std::memcpy(r.current_generation.fitness.get(), c.fitness, n * sizeof(float));
    std::memcpy(r.current_generation.evaluation_counts.get(), c.evaluation_counts, n * sizeof(std::uint32_t));
    std::memcpy(r.current_generation.has_fitness.get(), c.has_fitness, n);
    std::memcpy(r.assembly_plan.parent_pairs.get(), c.parent_pairs, c.child_count * 2 * sizeof(std::uint32_t));
    const std::size_t stride = c.slab_layout.slot_stride_bytes;
    r.live_genotypes.resize(c.live_count);
    for (std::size_t k = 0; k < c.live_count; ++k) {
        r.live_genotypes[k].organism_index = c.live_organisms[k];
        r.live_genotypes[k].genome_bytes.assign(c.live_genomes + k * stride, c.live_genomes + (k + 1) * stride);
    }
    return true;
}

bool ShimDownloadGeneration(const DeviceSlabGARuntimeBuffers &b, bool current, genotype_slab::SlabGeneration &out) {
    out = {};
    nwg_runtime_info i{};
    if (ShimHandle(b) == nullptr || nwg_get_info(ShimHandle(b), &i) != NWG_OK) {
        return false;
    }
    const std::size_t n = current ? i.current_generation_size : i.next_generation_size;
    const std::size_t index = current ? i.current_generation_index : i.next_generation_index;
    if (!genotype_slab::TryCreateSlabGeneration(out, n, index)) {
        return false;
    }
    std::size_t count = 0, generation = 0;
    const auto fn = current ? nwg_download_current_generation : nwg_download_next_generation;
    if (fn(ShimHandle(b), out.slot_indices.get(), out.fitness.get(), out.evaluation_counts.get(), out.has_fitness.get(),
           n, &count, &generation) != NWG_OK) {
        out = {};
        return false;
    }
    return true;
}

}  // namespace

bool TryCreateDeviceSlabGARuntimeBuffers(DeviceSlabGARuntimeBuffers &buffers, const DeviceSlabGARuntimeConfig &config) {
    buffers = {};
    nwg_runtime *rt = nullptr;
    if (nwg_create(reinterpret_cast<const nwg_runtime_config *>(&config), &rt) != NWG_OK) {
        return false;
    }
    buffers.status = reinterpret_cast<int *>(rt);
    ShimMirror(buffers);
    return true;
}

void DestroyDeviceSlabGARuntimeBuffers(DeviceSlabGARuntimeBuffers &buffers) noexcept {
    nwg_destroy(ShimHandle(buffers));
    buffers = {};
}

bool TryBootstrapRandomCurrentGenerationOnDevice(DeviceSlabGARuntimeBuffers &buffers, const std::size_t generation_size,
                                                 const std::uint32_t generation_seed,
                                                 const std::size_t generation_index) {
    const bool ok = nwg_bootstrap(ShimHandle(buffers), generation_size, generation_seed, generation_index) == NWG_OK;
    ShimMirror(buffers);
    return ok;
}

bool TryDownloadSlabFromDevice(const DeviceSlabGARuntimeBuffers &buffers, genotype_slab::HostGenotypeSlab &host_buffer) {
    nwg_runtime_info i{};
    if (ShimHandle(buffers) == nullptr || nwg_get_info(ShimHandle(buffers), &i) != NWG_OK) {
        return false;
    }
    genotype_slab::GenotypeSlabLayout layout{};
    layout.action_count = i.action_count;
    layout.slot_stride_bytes = i.slot_stride_bytes;
    layout.slot_count = i.slot_count;
    layout.slab_bytes = i.slab_bytes;
    if (!genotype_slab::TryCreateHostGenotypeSlab(host_buffer, layout)) {
        return false;
    }
    for (std::size_t s = 0; s < i.slot_count; ++s) {
        std::size_t n = 0;
        if (nwg_download_slot(ShimHandle(buffers), static_cast<std::uint32_t>(s),
                              host_buffer.storage.get() + s * i.slot_stride_bytes, i.slot_stride_bytes,
                              &n) != NWG_OK) {
            host_buffer = {};
            return false;
        }
    }
    // the current generation's slots are the occupied ones; the free stack keeps the others in its order
    genotype_slab::SlabGeneration current{};
    if (i.current_generation_size > 0 && ShimDownloadGeneration(buffers, true, current)) {
        for (std::size_t k = 0; k < current.active_individual_count; ++k) {
            const std::uint32_t s = current.slot_indices[k];
            if (s < i.slot_count) {
                host_buffer.slot_states[s].occupied = true;
                host_buffer.slot_states[s].liveness_count = 1;
            }
        }
        std::uint32_t kept = 0;
        for (std::uint32_t k = 0; k < host_buffer.free_slot_count; ++k) {
            const std::uint32_t s = host_buffer.free_slot_stack[k];
            if (!host_buffer.slot_states[s].occupied) {
                host_buffer.free_slot_stack[kept++] = s;
            }
        }
        host_buffer.free_slot_count = kept;
    }
    return true;
}

bool TryDownloadSlabSlotBytesFromDevice(const DeviceSlabGARuntimeBuffers &buffers, const std::uint32_t slot_index,
                                        std::unique_ptr<std::uint8_t[]> &slot_bytes, std::size_t &slot_byte_count) {
    slot_bytes.reset();
    slot_byte_count = 0;
    nwg_runtime_info i{};
    if (ShimHandle(buffers) == nullptr || nwg_get_info(ShimHandle(buffers), &i) != NWG_OK) {
        return false;
    }
    std::unique_ptr<std::uint8_t[]> bytes(new (std::nothrow) std::uint8_t[i.slot_stride_bytes]);
    std::size_t n = 0;
    if (bytes == nullptr ||
        nwg_download_slot(ShimHandle(buffers), slot_index, bytes.get(), i.slot_stride_bytes, &n) != NWG_OK) {
        return false;
    }
    slot_bytes = std::move(bytes);
    slot_byte_count = n;
    return true;
}

bool TryDownloadCurrentGenerationFromDevice(const DeviceSlabGARuntimeBuffers &buffers,
                                            genotype_slab::SlabGeneration &generation) {
    return ShimDownloadGeneration(buffers, true, generation);
}

bool TryDownloadNextGenerationFromDevice(const DeviceSlabGARuntimeBuffers &buffers,
                                         genotype_slab::SlabGeneration &generation) {
    return ShimDownloadGeneration(buffers, false, generation);
}

bool TryEvaluateCurrentGenerationFitnessOnDevice(
    DeviceSlabGARuntimeBuffers &buffers, const RuntimeWordCounts &runtime_word_counts,
    const training_folder::TrainingDataShardReleaseHistory *training_shard_release_history) {
    const bool ok = nwg_evaluate(ShimHandle(buffers), reinterpret_cast<const nwg_runtime_word_counts *>(&runtime_word_counts),
                                 reinterpret_cast<const nwg_shard_release_history *>(training_shard_release_history)) ==
                    NWG_OK;
    ShimMirror(buffers);
    return ok;
}

bool TryReadPopulationFitnessSummaryFromDevice(const DeviceSlabGARuntimeBuffers &buffers,
                                               PopulationFitnessSummary &summary) {
    return nwg_read_summary(ShimHandle(buffers), reinterpret_cast<nwg_fitness_summary *>(&summary)) == NWG_OK;
}

bool TryAdvanceGenerationOnDevice(DeviceSlabGARuntimeBuffers &buffers, const std::uint32_t generation_seed,
                                  const RuntimeWordCounts &runtime_word_counts, const GenerationAssemblyConfig &config,
                                  const PendingOutputEmbeddingInjection &pending_output_embedding_injection,
                                  const bool /*verbose*/,
                                  const PostFitnessEvaluationCallback &post_fitness_evaluation_callback,
                                  const TrainingShardReleaseCallback &training_shard_release_callback,
                                  const training_folder::TrainingDataShardReleaseHistory *training_shard_release_history) {
    ShimCallbacks cb{&buffers, &post_fitness_evaluation_callback, &training_shard_release_callback};
    const bool ok =
        nwg_advance(ShimHandle(buffers), generation_seed,
                    reinterpret_cast<const nwg_runtime_word_counts *>(&runtime_word_counts),
                    reinterpret_cast<const nwg_generation_assembly_config *>(&config),
                    reinterpret_cast<const nwg_pending_injection *>(&pending_output_embedding_injection),
                    post_fitness_evaluation_callback ? ShimPostFitness : nullptr, &cb,
                    training_shard_release_callback ? ShimShardRelease : nullptr, &cb,
                    reinterpret_cast<const nwg_shard_release_history *>(training_shard_release_history)) == NWG_OK;
    ShimMirror(buffers);
    return ok;
}

bool TryCreatePrebreedingCheckpointOnDevice(DeviceSlabGARuntimeBuffers &buffers, const std::uint32_t generation_seed,
                                            const RuntimeWordCounts &runtime_word_counts,
                                            const GenerationAssemblyConfig &config,
                                            const PendingOutputEmbeddingInjection &pending_output_embedding_injection,
                                            RuntimeCheckpoint &checkpoint_out,
                                            const training_folder::TrainingWordCatalog *host_training_word_catalog,
                                            const bool /*verbose*/,
                                            const PostFitnessEvaluationCallback &post_fitness_evaluation_callback,
                                            const TrainingShardReleaseCallback &training_shard_release_callback,
                                            const training_folder::TrainingDataShardReleaseHistory *training_shard_release_history) {
    checkpoint_out = {};
    const std::uint8_t *letters = nullptr;
    std::size_t letter_count = 0;
    if (host_training_word_catalog != nullptr) {
        letters = reinterpret_cast<const std::uint8_t *>(&host_training_word_catalog->words[0]);
        letter_count = host_training_word_catalog->word_count;
    }
    ShimCallbacks cb{&buffers, &post_fitness_evaluation_callback, &training_shard_release_callback};
    nwg_checkpoint c{};
    const int st = nwg_checkpoint_capture(
        ShimHandle(buffers), generation_seed, reinterpret_cast<const nwg_runtime_word_counts *>(&runtime_word_counts),
        reinterpret_cast<const nwg_generation_assembly_config *>(&config),
        reinterpret_cast<const nwg_pending_injection *>(&pending_output_embedding_injection),
        post_fitness_evaluation_callback ? ShimPostFitness : nullptr, &cb,
        training_shard_release_callback ? ShimShardRelease : nullptr, &cb,
        reinterpret_cast<const nwg_shard_release_history *>(training_shard_release_history), letters, letter_count, &c);
    ShimMirror(buffers);
    const bool ok = st == NWG_OK && ShimFromC(c, checkpoint_out);
    nwg_checkpoint_free(&c);
    return ok;
}

bool TryRestorePrebreedingCheckpointToDevice(const RuntimeCheckpoint &checkpoint, DeviceSlabGARuntimeBuffers &buffers) {
    buffers = {};
    ShimCheckpointView v;
    nwg_runtime *rt = nullptr;
    if (!ShimToC(checkpoint, v) || nwg_checkpoint_restore(&v.c, &rt) != NWG_OK) {
        return false;
    }
    buffers.status = reinterpret_cast<int *>(rt);
    ShimMirror(buffers);
    return true;
}

bool TryResumeGenerationFromCheckpointOnDevice(DeviceSlabGARuntimeBuffers &buffers, const RuntimeCheckpoint &,
                                               const bool /*verbose*/) {
    const bool ok = nwg_checkpoint_resume(ShimHandle(buffers)) == NWG_OK;
    ShimMirror(buffers);
    return ok;
}

bool TryWriteRuntimeCheckpointAtomically(const RuntimeCheckpoint &checkpoint,
                                         const std::filesystem::path &checkpoint_path) {
    ShimCheckpointView v;
    std::error_code error{};
    if (checkpoint_path.has_parent_path()) {
        std::filesystem::create_directories(checkpoint_path.parent_path(), error);
    }
    return ShimToC(checkpoint, v) && nwg_checkpoint_write(&v.c, checkpoint_path.c_str()) == NWG_OK;
}

bool TryReadRuntimeCheckpoint(const std::filesystem::path &checkpoint_path, RuntimeCheckpoint &checkpoint_out) {
    checkpoint_out = {};
    nwg_checkpoint c{};
    if (nwg_checkpoint_read(checkpoint_path.c_str(), &c) != NWG_OK) {
        return false;
    }
    const bool ok = ShimFromC(c, checkpoint_out);
    nwg_checkpoint_free(&c);
    return ok;
}

// RuntimeCheckpointAsyncWriter (slab_runtime.hpp:169-178): one write in flight on a std::async thread; a new write
// starts only after the previous one has finished and succeeded.
bool RuntimeCheckpointAsyncWriter::IsWriteInProgress() {
    return pending_write_.valid() && pending_write_.wait_for(std::chrono::seconds(0)) != std::future_status::ready;
}

bool RuntimeCheckpointAsyncWriter::TryCollectFinishedWrite(bool &write_finished_out, bool &write_succeeded_out) {
    write_finished_out = false;
    write_succeeded_out = true;
    if (!pending_write_.valid() || IsWriteInProgress()) {
        return true;
    }
    write_finished_out = true;
    write_succeeded_out = pending_write_.get();
    return write_succeeded_out;
}

bool RuntimeCheckpointAsyncWriter::TryStartWrite(RuntimeCheckpoint checkpoint, std::filesystem::path checkpoint_path) {
    if (IsWriteInProgress() || (pending_write_.valid() && !pending_write_.get())) {
        return false;
    }
    pending_write_ = std::async(std::launch::async, [c = std::move(checkpoint), p = std::move(checkpoint_path)]() {
        return TryWriteRuntimeCheckpointAtomically(c, p);
    });
    return true;
}

bool RuntimeCheckpointAsyncWriter::TryWaitForWrite() { return !pending_write_.valid() || pending_write_.get(); }

void SwapDeviceSlabGenerationBuffers(DeviceSlabGARuntimeBuffers &buffers) noexcept {
    (void)nwg_swap_generations(ShimHandle(buffers));
    ShimMirror(buffers);
}

bool TryReadDeviceSlabGARuntimeStatus(const DeviceSlabGARuntimeBuffers &buffers,
                                      DeviceSlabGARuntimeStatusCode &status_code) {
    int status = 0;
    if (nwg_read_status(ShimHandle(buffers), &status) != NWG_OK) {
        return false;
    }
    status_code = static_cast<DeviceSlabGARuntimeStatusCode>(status);
    return true;
}

const char *DeviceSlabGARuntimeStatusCodeString(const DeviceSlabGARuntimeStatusCode status_code) noexcept {
    return nwg_status_string(static_cast<int>(status_code));
}

}  // namespace neuroevolution::genetic_algorithm::slab_device

#endif  // NWG_SLAB_DEVICE_SHIM_IMPLEMENTATION
