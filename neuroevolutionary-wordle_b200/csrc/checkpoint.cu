// Runtime checkpoints at the pre-breeding boundary (genetic_algorithm/device/slab_runtime.hpp:86-117,
// slab_runtime.cu:1182-1372 checksum and capture, :1707-1880 create, restore and resume, :1889-2073 file format).
//
// The file is the reference's byte for byte: a little-endian stream of the checkpoint's records in declaration
// order, each at its LP64 in-memory size (the assembly config and the pending injection carry padding, which is
// kept as read and zeroed when captured here), the current generation's per-individual arrays interleaved, the
// parent plan, then one record per live genome; an FNV-1a 64 checksum covers the same fields. Capture and restore
// work through the runtime's boundary (nwg_prepare_generation / nwg_assemble_prepared) rather than the reference's
// slot free list: capture marks the parents no child references as released (slot 0xFFFFFFFF, no genome record),
// as the reference's CollectZeroReferenceParentsKernel does before its capture, and restore places the genome
// records in slots 0, 1, 2, ... in record order, as TryAllocateSlabSlot does on the reference's fresh host slab.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

using namespace nwg;

namespace {

constexpr std::uint64_t kMagic = 0x4b4350474147524eULL;  // "NRGAGPCK" read as a little-endian u64
constexpr std::uint64_t kFnvOffset = 1469598103934665603ULL;
constexpr std::uint64_t kFnvPrime = 1099511628211ULL;
constexpr std::uint32_t kSchemaVersion = 3;
constexpr std::uint32_t kGenomeLayoutVersion = 1;
constexpr std::uint32_t kResumePreRecombinationPreMutation = 1;
constexpr std::uint32_t kReleasedSlot = 0xFFFFFFFFu;

static_assert(sizeof(nwg_generation_assembly_config) == 40, "assembly config record is 40 bytes on LP64");
static_assert(sizeof(nwg_pending_injection) == 24, "pending injection record is 24 bytes on LP64");
static_assert(sizeof(nwg_runtime_word_counts) == 56, "word-count record is 56 bytes on LP64");
static_assert(sizeof(nwg_runtime_config) == 48, "runtime config record is 48 bytes on LP64");
static_assert(sizeof(nwg_slab_layout) == 32, "slab layout record is 32 bytes on LP64");
static_assert(sizeof(nwg_grid_shape) == 24, "grid shape record is 24 bytes on LP64");

// The records with padding, written field by field into zeroed storage.
void Canonical(const nwg_generation_assembly_config &c, nwg_generation_assembly_config *out) {
    std::memset(out, 0, sizeof(*out));
    out->parent_selection.cellular_breeding_radius = c.parent_selection.cellular_breeding_radius;
    out->parent_selection.rank_exponent = c.parent_selection.rank_exponent;
    out->breeding = c.breeding;
    out->mutation = c.mutation;
}

void Canonical(const nwg_pending_injection &p, nwg_pending_injection *out) {
    std::memset(out, 0, sizeof(*out));
    out->enabled = p.enabled;
    out->first_catalog_word_index = p.first_catalog_word_index;
    out->injection_count = p.injection_count;
}

struct Fnv {
    std::uint64_t h = kFnvOffset;
    void Bytes(const void *data, std::size_t n) {
        const auto *b = static_cast<const unsigned char *>(data);
        for (std::size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= kFnvPrime;
        }
    }
    template <typename T>
    void Value(const T &v) {
        Bytes(&v, sizeof(T));
    }
};

void MixHistory(Fnv &f, const nwg_shard_release_history &h) {  // slab_runtime.cu:1198-1204
    f.Value(h.release_count);
    for (std::size_t i = 0; i < h.release_count && i < NWG_CATALOG_CAPACITY; ++i) {
        f.Value(h.release_generations[i]);
        f.Value(h.release_fitness_p99[i]);
    }
}

// One visitor for the checksum and the writer, so both walk the fields in the same order.
template <typename Sink>
void VisitFields(const nwg_checkpoint &c, Sink &sink, bool with_file_header) {
    if (with_file_header) {  // the file leads with the magic and puts the checksum before the identity hash
        sink.Value(kMagic);
        sink.Value(c.schema_version);
        sink.Value(c.genome_layout_version);
        sink.Value(c.checksum);
        sink.Value(c.training_data_identity_hash);
        sink.Value(c.resume_phase);
    } else {
        sink.Value(c.schema_version);
        sink.Value(c.genome_layout_version);
        sink.Value(c.resume_phase);
        sink.Value(c.training_data_identity_hash);
    }
    sink.Value(c.generation_seed);
    sink.Value(c.runtime_word_counts);
    const nwg_shard_release_history &h = c.training_shard_release_history;
    sink.Value(h.release_count);
    for (std::size_t i = 0; i < h.release_count && i < NWG_CATALOG_CAPACITY; ++i) {
        sink.Value(h.release_generations[i]);
        sink.Value(h.release_fitness_p99[i]);
    }
    sink.Value(c.assembly_config);
    sink.Value(c.pending_output_embedding_injection);
    sink.Value(c.runtime_config);
    sink.Value(c.slab_layout);
    sink.Value(c.current_grid_shape);
    sink.Value(c.next_grid_shape);
    sink.Value(c.epicenter_grid_shape);
    sink.Value(c.generation_index);
    sink.Value(c.individual_count);
    for (std::size_t i = 0; i < c.individual_count; ++i) {
        sink.Value(c.slot_indices[i]);
        sink.Value(c.fitness[i]);
        sink.Value(c.evaluation_counts[i]);
        sink.Value(c.has_fitness[i]);
    }
    sink.Value(c.child_count);
    if (c.child_count > 0) {
        sink.Bytes(c.parent_pairs, c.child_count * 2 * sizeof(std::uint32_t));
    }
    const std::uint64_t live = c.live_count;
    sink.Value(live);
    const std::size_t stride = c.slab_layout.slot_stride_bytes;
    for (std::size_t k = 0; k < c.live_count; ++k) {
        const std::uint64_t bytes = stride;
        sink.Value(c.live_organisms[k]);
        sink.Value(bytes);
        sink.Bytes(c.live_genomes + k * stride, stride);
    }
}

struct Writer {
    std::FILE *file;
    bool ok = true;
    void Bytes(const void *data, std::size_t n) {
        if (ok && n > 0) {
            ok = std::fwrite(data, 1, n, file) == n;
        }
    }
    template <typename T>
    void Value(const T &v) {
        Bytes(&v, sizeof(T));
    }
};

struct Reader {
    std::FILE *file;
    bool ok = true;
    void Bytes(void *data, std::size_t n) {
        if (ok && n > 0) {
            ok = std::fread(data, 1, n, file) == n;
        }
    }
    template <typename T>
    void Value(T &v) {
        Bytes(&v, sizeof(T));
    }
};

template <typename T>
T *Calloc(std::size_t n) {
    return static_cast<T *>(std::calloc(n + 1, sizeof(T)));  // +1: a valid pointer for n = 0
}

// IsValidGenotypeSlabLayout (genotype_slab/layout.hpp:66-71).
bool ValidLayout(const nwg_slab_layout &l) {
    const std::size_t stride = GenomeStrideBytes(l.action_count);
    return l.action_count > 0 && l.slot_count > 0 && l.slot_count < kReleasedSlot && l.slot_stride_bytes == stride &&
           l.slot_count == l.slab_bytes / stride && l.slab_bytes >= l.slot_count * stride;
}

// TryMakeCellularGridShapeForColumnCount (spatial/grid.hpp:97-106).
bool GridShape(std::size_t cells, std::size_t cols, nwg_grid_shape *out) {
    std::memset(out, 0, sizeof(*out));
    if (cells == 0 || cols == 0 || cells % cols != 0) {
        return false;
    }
    out->row_count = cells / cols;
    out->column_count = cols;
    out->cell_count = cells;
    return true;
}

}  // namespace

extern "C" {

uint64_t nwg_checkpoint_checksum(const nwg_checkpoint *c) {
    if (c == nullptr) {
        return 0;
    }
    Fnv f;
    VisitFields(*c, f, false);
    return f.h;
}

uint64_t nwg_checkpoint_identity_hash(const nwg_runtime_word_counts *counts, const nwg_shard_release_history *history,
                                      const uint8_t *catalog_letters, size_t catalog_count) {
    Fnv f;
    if (counts != nullptr) {
        f.Value(*counts);
    }
    if (history != nullptr) {
        MixHistory(f, *history);
    }
    if (catalog_letters != nullptr) {
        const std::size_t n = catalog_count;
        f.Value(n);
        f.Bytes(catalog_letters, catalog_count * 5);
    }
    return f.h;
}

void nwg_checkpoint_free(nwg_checkpoint *c) {
    if (c == nullptr) {
        return;
    }
    std::free(c->slot_indices);
    std::free(c->fitness);
    std::free(c->evaluation_counts);
    std::free(c->has_fitness);
    std::free(c->parent_pairs);
    std::free(c->live_organisms);
    std::free(c->live_genomes);
    c->slot_indices = nullptr;
    c->fitness = nullptr;
    c->evaluation_counts = nullptr;
    c->has_fitness = nullptr;
    c->parent_pairs = nullptr;
    c->live_organisms = nullptr;
    c->live_genomes = nullptr;
    c->individual_count = 0;
    c->child_count = 0;
    c->live_count = 0;
}

int nwg_checkpoint_write(const nwg_checkpoint *c, const char *path) {
    if (c == nullptr || path == nullptr) {
        return kInvalidCheckpoint;
    }
    if ((c->individual_count > 0 && (!c->slot_indices || !c->fitness || !c->evaluation_counts || !c->has_fitness)) ||
        (c->child_count > 0 && c->parent_pairs == nullptr) ||
        (c->live_count > 0 && (c->live_organisms == nullptr || c->live_genomes == nullptr)) ||
        c->training_shard_release_history.release_count > NWG_CATALOG_CAPACITY ||
        c->checksum != nwg_checkpoint_checksum(c)) {
        return kInvalidCheckpoint;
    }
    const std::string tmp = std::string(path) + ".tmp";
    Writer w{std::fopen(tmp.c_str(), "wb")};
    if (w.file == nullptr) {
        return kInvalidCheckpoint;
    }
    VisitFields(*c, w, true);
    const bool closed = std::fclose(w.file) == 0;
    if (!w.ok || !closed || std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        return kInvalidCheckpoint;
    }
    return kOk;
}

int nwg_checkpoint_read(const char *path, nwg_checkpoint *out) {
    if (path == nullptr || out == nullptr) {
        return kInvalidCheckpoint;
    }
    std::memset(out, 0, sizeof(*out));
    Reader r{std::fopen(path, "rb")};
    if (r.file == nullptr) {
        return kInvalidCheckpoint;
    }
    std::uint64_t magic = 0;
    r.Value(magic);
    r.ok = r.ok && magic == kMagic;
    r.Value(out->schema_version);
    r.Value(out->genome_layout_version);
    r.Value(out->checksum);
    r.Value(out->training_data_identity_hash);
    r.Value(out->resume_phase);
    r.Value(out->generation_seed);
    r.Value(out->runtime_word_counts);
    nwg_shard_release_history &h = out->training_shard_release_history;
    r.Value(h.release_count);
    r.ok = r.ok && h.release_count <= NWG_CATALOG_CAPACITY;
    for (std::size_t i = 0; r.ok && i < h.release_count; ++i) {
        r.Value(h.release_generations[i]);
        r.Value(h.release_fitness_p99[i]);
    }
    r.Value(out->assembly_config);
    r.Value(out->pending_output_embedding_injection);
    r.Value(out->runtime_config);
    r.Value(out->slab_layout);
    r.Value(out->current_grid_shape);
    r.Value(out->next_grid_shape);
    r.Value(out->epicenter_grid_shape);
    r.Value(out->generation_index);
    std::size_t individuals = 0;
    r.Value(individuals);
    // TryCreateSlabGeneration / TryCreateSlabAssemblyPlan refuse empty arrays; the caps bound a corrupt count
    // before it is allocated
    const std::size_t stride = out->slab_layout.slot_stride_bytes;
    r.ok = r.ok && individuals > 0 && individuals <= (std::size_t{1} << 26) && stride <= (std::size_t{1} << 30);
    if (r.ok) {
        out->individual_count = individuals;
        out->slot_indices = Calloc<std::uint32_t>(individuals);
        out->fitness = Calloc<float>(individuals);
        out->evaluation_counts = Calloc<std::uint32_t>(individuals);
        out->has_fitness = Calloc<std::uint8_t>(individuals);
        r.ok = out->slot_indices && out->fitness && out->evaluation_counts && out->has_fitness;
    }
    for (std::size_t i = 0; r.ok && i < individuals; ++i) {
        r.Value(out->slot_indices[i]);
        r.Value(out->fitness[i]);
        r.Value(out->evaluation_counts[i]);
        r.Value(out->has_fitness[i]);
    }
    std::size_t children = 0;
    r.Value(children);
    r.ok = r.ok && children > 0 && children <= (std::size_t{1} << 26);
    if (r.ok) {
        out->child_count = children;
        out->parent_pairs = Calloc<std::uint32_t>(2 * children);
        r.ok = out->parent_pairs != nullptr;
        r.Bytes(out->parent_pairs, children * 2 * sizeof(std::uint32_t));
    }
    std::uint64_t live = 0;
    r.Value(live);
    r.ok = r.ok && live <= individuals;
    if (r.ok) {
        out->live_count = static_cast<std::size_t>(live);
        out->live_organisms = Calloc<std::uint32_t>(out->live_count);
        out->live_genomes = Calloc<std::uint8_t>(out->live_count * stride);
        r.ok = out->live_organisms != nullptr && out->live_genomes != nullptr;
    }
    for (std::size_t k = 0; r.ok && k < out->live_count; ++k) {
        std::uint64_t bytes = 0;
        r.Value(out->live_organisms[k]);
        r.Value(bytes);
        r.ok = r.ok && bytes == stride;
        r.Bytes(out->live_genomes + k * stride, stride);
    }
    std::fclose(r.file);
    if (!r.ok || out->schema_version != kSchemaVersion || out->genome_layout_version != kGenomeLayoutVersion ||
        out->checksum != nwg_checkpoint_checksum(out)) {
        nwg_checkpoint_free(out);
        std::memset(out, 0, sizeof(*out));
        return kInvalidCheckpoint;
    }
    return kOk;
}

int nwg_checkpoint_capture(nwg_runtime *rt, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                           const nwg_generation_assembly_config *config, const nwg_pending_injection *pending,
                           nwg_post_fitness_fn post_fitness, void *post_fitness_user,
                           nwg_shard_release_fn shard_release, void *shard_release_user,
                           const nwg_shard_release_history *history, const uint8_t *catalog_letters,
                           size_t catalog_count, nwg_checkpoint *out) {
    if (out == nullptr) {
        return kInvalidCheckpoint;
    }
    std::memset(out, 0, sizeof(*out));
    int st = nwg_prepare_generation(rt, generation_seed, counts, config, pending, post_fitness, post_fitness_user,
                                    shard_release, shard_release_user, history);
    if (st != kOk) {
        return st;
    }
    BoundaryState b{};
    st = ReadBoundary(rt, &b);
    if (st != kOk) {
        return st;
    }
    // the layout the reference holds at this boundary: widened in place when an injection is pending
    // (TryPrepareSlabForExpandedActionCountOnDevice, genotype_slab/device_runtime.cu:1338-1432)
    nwg_slab_layout layout{};
    layout.action_count = b.injection.enabled ? b.next_action_count : b.action_count;
    layout.slot_stride_bytes = GenomeStrideBytes(layout.action_count);
    layout.slab_bytes = b.slab_bytes;
    layout.slot_count = b.injection.enabled ? b.slab_bytes / layout.slot_stride_bytes : b.slot_count;
    if (!ValidLayout(layout)) {
        return kSlabRepackFailed;
    }
    const std::size_t n = b.generation_size;
    const std::size_t children = b.planned_children;
    out->schema_version = kSchemaVersion;
    out->genome_layout_version = kGenomeLayoutVersion;
    out->resume_phase = kResumePreRecombinationPreMutation;
    out->generation_seed = b.seed;
    out->training_data_identity_hash = nwg_checkpoint_identity_hash(counts, history, catalog_letters, catalog_count);
    out->runtime_word_counts = *counts;
    if (history != nullptr) {
        out->training_shard_release_history = *history;
    }
    Canonical(config != nullptr ? *config : b.config, &out->assembly_config);
    Canonical(b.injection, &out->pending_output_embedding_injection);
    // slab_runtime.cu:1495-1502
    out->runtime_config.genotype_slab_byte_budget_bytes = layout.slab_bytes;
    out->runtime_config.generation_byte_budget_bytes = b.generation_byte_budget;
    out->runtime_config.host_spillover_byte_budget_bytes = b.host_spill_budget;
    out->runtime_config.action_count = layout.action_count;
    out->runtime_config.population_size_ceiling = b.max_generation_size;
    out->runtime_config.grid_column_count = b.grid_column_count;
    out->slab_layout = layout;
    out->epicenter_grid_shape.row_count = b.epicenter_rows;
    out->epicenter_grid_shape.column_count = b.grid_column_count;
    out->epicenter_grid_shape.cell_count = b.epicenter_rows * b.grid_column_count;
    if (!GridShape(n, b.grid_column_count, &out->current_grid_shape) ||
        !GridShape(children, b.grid_column_count, &out->next_grid_shape)) {
        std::memset(out, 0, sizeof(*out));
        return kInvalidGeneration;
    }
    out->individual_count = n;
    out->child_count = children;
    out->slot_indices = Calloc<std::uint32_t>(n);
    out->fitness = Calloc<float>(n);
    out->evaluation_counts = Calloc<std::uint32_t>(n);
    out->has_fitness = Calloc<std::uint8_t>(n);
    out->parent_pairs = Calloc<std::uint32_t>(2 * children);
    out->live_organisms = Calloc<std::uint32_t>(n);
    bool ok = out->slot_indices && out->fitness && out->evaluation_counts && out->has_fitness && out->parent_pairs &&
              out->live_organisms;
    std::size_t count = 0, generation_index = 0, plan_count = 0;
    ok = ok && nwg_download_current_generation(rt, out->slot_indices, out->fitness, out->evaluation_counts,
                                               out->has_fitness, n, &count, &generation_index) == kOk &&
         count == n;
    ok = ok && nwg_download_assembly_plan(rt, out->parent_pairs, children, &plan_count) == kOk && plan_count == children;
    out->generation_index = generation_index;
    // parents no child references are released before the reference's capture (slab_runtime.cu:1481-1491)
    std::vector<std::uint8_t> referenced(n, 0);
    for (std::size_t c = 0; ok && c < 2 * children; ++c) {
        ok = out->parent_pairs[c] < n;
        if (ok) {
            referenced[out->parent_pairs[c]] = 1;
        }
    }
    std::size_t live = 0;
    for (std::size_t i = 0; ok && i < n; ++i) {
        if (!referenced[i]) {
            out->slot_indices[i] = kReleasedSlot;
        } else {
            out->live_organisms[live++] = static_cast<std::uint32_t>(i);
        }
    }
    // genomes at the checkpoint's stride: a widened one keeps the parent's bytes and zero-fills the new rows
    // (genotype_slab/device_runtime.cu:953-961)
    out->live_count = live;
    out->live_genomes = ok ? Calloc<std::uint8_t>(live * layout.slot_stride_bytes) : nullptr;
    ok = ok && out->live_genomes != nullptr;
    for (std::size_t k = 0; ok && k < live; ++k) {
        std::size_t got = 0;
        const std::uint32_t slot = out->slot_indices[out->live_organisms[k]];
        ok = nwg_download_slot(rt, slot, out->live_genomes + k * layout.slot_stride_bytes, b.stride, &got) == kOk &&
             got == b.stride;
    }
    if (!ok) {
        nwg_checkpoint_free(out);
        std::memset(out, 0, sizeof(*out));
        return kCudaFailure;
    }
    out->checksum = nwg_checkpoint_checksum(out);
    return kOk;
}

int nwg_checkpoint_restore(const nwg_checkpoint *c, nwg_runtime **runtime_out) {
    if (runtime_out == nullptr) {
        return kInvalidCheckpoint;
    }
    *runtime_out = nullptr;
    // TryRestorePrebreedingCheckpointToDevice's checks (slab_runtime.cu:1734-1742)
    if (c == nullptr || c->schema_version != kSchemaVersion || c->genome_layout_version != kGenomeLayoutVersion ||
        c->resume_phase != kResumePreRecombinationPreMutation || c->individual_count == 0 || c->child_count == 0 ||
        !c->slot_indices || !c->fitness || !c->evaluation_counts || !c->has_fitness || !c->parent_pairs ||
        (c->live_count > 0 && (!c->live_organisms || !c->live_genomes)) ||
        c->training_shard_release_history.release_count > NWG_CATALOG_CAPACITY ||
        c->checksum != nwg_checkpoint_checksum(c) || !ValidLayout(c->slab_layout)) {
        return kInvalidCheckpoint;
    }
    const nwg_pending_injection &inj = c->pending_output_embedding_injection;
    if (inj.enabled && (inj.first_catalog_word_index == 0 || inj.injection_count == 0 ||
                        inj.first_catalog_word_index + inj.injection_count != c->slab_layout.action_count)) {
        return kInvalidCheckpoint;
    }
    const std::size_t n = c->individual_count;
    // the parents' own width: a widened checkpoint's genomes are the parents' images zero-padded, and breeding
    // reads only the parents' rows (slab_runtime.cu:1849-1852)
    const std::size_t parent_actions = inj.enabled ? inj.first_catalog_word_index : c->slab_layout.action_count;
    const std::size_t parent_stride = GenomeStrideBytes(parent_actions);
    const std::size_t parent_slots = c->slab_layout.slab_bytes / parent_stride;
    if (c->live_count > parent_slots || c->runtime_config.grid_column_count == 0) {
        return kInvalidCheckpoint;
    }
    std::vector<std::uint32_t> slots(n, kReleasedSlot);
    for (std::size_t k = 0; k < c->live_count; ++k) {  // slab_runtime.cu:1800-1819
        const std::uint32_t organism = c->live_organisms[k];
        if (organism >= n || slots[organism] != kReleasedSlot || c->slot_indices[organism] == kReleasedSlot) {
            return kInvalidCheckpoint;
        }
        slots[organism] = static_cast<std::uint32_t>(k);
    }
    for (std::size_t i = 0; i < 2 * c->child_count; ++i) {  // slab_runtime.cu:1821-1829
        if (c->parent_pairs[i] >= n || slots[c->parent_pairs[i]] == kReleasedSlot) {
            return kInvalidCheckpoint;
        }
    }
    RuntimeShape shape{};
    shape.action_count = parent_actions;
    shape.slot_count = parent_slots;
    shape.slab_bytes = c->slab_layout.slab_bytes;
    shape.max_generation_size = n > c->child_count ? n : c->child_count;
    shape.grid_column_count = c->runtime_config.grid_column_count;
    shape.generation_byte_budget = c->runtime_config.generation_byte_budget_bytes;
    shape.host_spill_budget = c->runtime_config.host_spillover_byte_budget_bytes;
    shape.epicenter_rows = c->epicenter_grid_shape.row_count;
    nwg_runtime *rt = nullptr;
    int st = CreateShapedRuntime(shape, &rt);
    if (st != kOk) {
        return st == kInvalidRuntimeConfig ? kInvalidCheckpoint : st;
    }
    for (std::size_t k = 0; st == kOk && k < c->live_count; ++k) {
        st = nwg_upload_slot(rt, static_cast<std::uint32_t>(k), c->live_genomes + k * c->slab_layout.slot_stride_bytes,
                             parent_stride);
    }
    if (st == kOk) {
        st = InstallBoundary(rt, slots.data(), c->fitness, c->evaluation_counts, c->has_fitness, n,
                             c->generation_index, c->parent_pairs, c->child_count, c->generation_seed,
                             c->assembly_config, inj, c->slab_layout.action_count);
    }
    if (st != kOk) {
        nwg_destroy(rt);
        return st;
    }
    *runtime_out = rt;
    return kOk;
}

int nwg_checkpoint_resume(nwg_runtime *rt) { return nwg_assemble_prepared(rt); }

}  // extern "C"
