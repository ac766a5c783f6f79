/*
 * nwg_capi.h -- C ABI of the B200 fitness-evaluation / generation-step runtime.
 *
 * Drop-in boundary for sam-bee/neuroevolutionary-wordle's device GA runtime
 * (src/genetic_algorithm/device/slab_runtime.hpp, namespace
 * neuroevolution::genetic_algorithm::slab_device). Every entry point below names the
 * reference function it replaces. Conventions:
 *   - plain pointers and sizes, no C++ or torch types;
 *   - every call returns an nwg status code: 0 is success, 1..16 are the reference's
 *     DeviceSlabGARuntimeStatusCode values (slab_runtime.hpp:21-39), 17..19 are
 *     additions (a bounded device wait that gave up; a feature this runtime rejects;
 *     a checkpoint that fails its checks, where the reference returns false);
 *   - the last failure is also kept as the runtime's sticky status, readable with
 *     nwg_read_status, as the reference keeps its device status int;
 *   - all device work of a runtime is issued on its stream (nwg_set_stream), and a call
 *     returns after that work has finished, like the reference's synchronous API.
 * Struct layouts equal the reference's POD structs on LP64 so a C++ shim can pass them
 * through unchanged.
 */
#ifndef NWG_CAPI_H
#define NWG_CAPI_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NWG_ABI_VERSION 4
#define NWG_CATALOG_CAPACITY 4739

enum {
    NWG_OK = 0,
    NWG_CUDA_FAILURE = 1,
    NWG_INVALID_RUNTIME_CONFIG = 2,
    NWG_INVALID_SLAB = 3,
    NWG_INVALID_GENERATION = 4,
    NWG_INVALID_TRAINING_SHARD = 5,
    NWG_GUESS_APPEND_FAILED = 6,
    NWG_POLICY_FORWARD_FAILED = 7,
    NWG_ACTION_SELECTION_FAILED = 8,
    NWG_POPULATION_NOT_EVALUATED = 9,
    NWG_INVALID_ASSEMBLY_CONFIG = 10,
    NWG_PARENT_SELECTION_FAILED = 11,
    NWG_INVALID_ASSEMBLY_PLAN = 12,
    NWG_INVALID_PARENT_INDEX = 13,
    NWG_SLAB_FULL = 14,
    NWG_OUTPUT_EMBEDDING_INJECTION_FAILED = 15,
    NWG_SLAB_REPACK_FAILED = 16,
    NWG_TIMEOUT = 17,
    NWG_UNSUPPORTED = 18,
    NWG_INVALID_CHECKPOINT = 19,
};

typedef struct nwg_runtime nwg_runtime;

/* DeviceSlabGARuntimeConfig (slab_runtime.hpp:41-48). */
typedef struct {
    size_t genotype_slab_byte_budget_bytes;
    size_t generation_byte_budget_bytes;
    size_t host_spillover_byte_budget_bytes;
    size_t action_count;
    size_t population_size_ceiling;
    size_t grid_column_count;
} nwg_runtime_config;

/* WordCountSchedule (training_folder/training_data.hpp:24-28). */
typedef struct {
    size_t initial_word_count;
    size_t word_count_step;
    size_t word_count_step_period_generations;
} nwg_word_count_schedule;

/* RuntimeWordCounts (genetic_algorithm/device/runtime_common.hpp:10-16). */
typedef struct {
    size_t training_word_count;
    size_t action_space_word_count;
    nwg_word_count_schedule training_word_schedule;
    size_t shard_initial_radius;
    size_t shard_radius_growth_period_generations;
} nwg_runtime_word_counts;

/* TrainingDataShardReleaseHistory (training_folder/training_data.hpp:49-53). */
typedef struct {
    size_t release_generations[NWG_CATALOG_CAPACITY];
    float release_fitness_p99[NWG_CATALOG_CAPACITY];
    size_t release_count;
} nwg_shard_release_history;

/* PopulationFitnessSummary (genetic_algorithm/device/runtime_common.hpp:18-26). */
typedef struct {
    float best_fitness;
    float average_fitness;
    size_t best_index;
    uint32_t best_slot_index;
    size_t generation_index;
    size_t action_count;
    size_t population_size;
} nwg_fitness_summary;

/* ParentSelectionConfig, BreedingConfig, MutationConfig, GenerationAssemblyConfig
 * (genetic_algorithm/selection.hpp:15-18, breeding.hpp:11-15, mutation.hpp:11-15,
 * generation_assembly.hpp:9-13). */
typedef struct {
    size_t cellular_breeding_radius;
    float rank_exponent;
} nwg_parent_selection_config;

typedef struct {
    float crossover_temperature_level1;
    float crossover_temperature_level2;
    float crossover_temperature_level3;
} nwg_breeding_config;

typedef struct {
    float mutation_probability;
    float mutation_sigma;
    float output_tail_row_scale_mutation_probability;
} nwg_mutation_config;

typedef struct {
    nwg_parent_selection_config parent_selection;
    nwg_breeding_config breeding;
    nwg_mutation_config mutation;
} nwg_generation_assembly_config;

/* PendingOutputEmbeddingInjection (genotype_slab/device_runtime.hpp:26-30). */
typedef struct {
    bool enabled;
    size_t first_catalog_word_index;
    size_t injection_count;
} nwg_pending_injection;

/* Statistics of the last evaluation, beyond the reference's summary. */
typedef struct {
    uint64_t game_steps;        /* policy decisions made (one forward + scoring + argmax + feedback each) */
    uint64_t episodes;          /* games played */
    uint64_t encoded_turns;     /* turns run through the shared encoder (each turn once) */
    double fitness_mean_fp64;   /* FP64 reductions for the adaptive shard-release statistics */
    double fitness_variance_fp64;
    double eval_kernel_ms;      /* device time of the last evaluation kernel (CUDA events on the runtime's stream) */
    uint64_t rescored_chunks;   /* tensor-core forms: 32-action chunks re-scored exactly in FP32 */
    uint64_t full_rescores;     /* tensor-core forms: game steps re-scored in FP32 over every action */
    uint64_t candidate_chunks;  /* tensor-core trunk forms: chunks re-scored from the 16-bit operands */
    uint64_t fallback_steps;    /* tensor-core trunk forms: game steps decided by the exact FP32 path */
} nwg_evaluation_stats;

/* Evaluation forms (nwg_set_evaluation_form). */
enum {
    NWG_FORM_FP32 = 0,          /* plain form: every score an FP32 fused-multiply-add chain (default) */
    NWG_FORM_TC_BF16 = 1,       /* scores on tcgen05 with BF16 operands, near-top chunks re-scored in FP32 */
    NWG_FORM_TC_FP16 = 2,       /* as above with FP16 operands (tighter bound, fewer re-scored chunks) */
    NWG_FORM_TC_TRUNK_BF16 = 3, /* encoder, trunk and scores on tcgen05 (BF16 operands), margin-guarded */
    NWG_FORM_TC_TRUNK_FP16 = 4, /* as above with FP16 operands (the genome's FP16 weights stay exact) */
};

typedef struct {
    size_t action_count;
    size_t slot_stride_bytes;   /* reference genome image size (dynamic_layout.hpp:30-36) */
    size_t slot_pitch_bytes;    /* device placement pitch of a slot (256-byte aligned) */
    size_t slot_count;
    size_t max_generation_size;
    size_t grid_column_count;
    size_t current_generation_index;
    size_t current_generation_size;
    size_t next_generation_index;       /* the generation being assembled (reference DeviceSlabRuntimeBuffers) */
    size_t next_generation_size;
    size_t planned_child_count;         /* children of the last plan */
    size_t slab_bytes;                  /* GenotypeSlabLayout::slab_bytes (slot_count x stride at creation) */
    size_t generation_byte_budget_bytes;
    size_t host_spillover_byte_budget_bytes;
    size_t epicenter_row_count;         /* rows of the epicenter grid (generation capacity / columns) */
    uint32_t prepared;                  /* 1 between nwg_prepare_generation (or a restore) and assembly */
} nwg_runtime_info;

/* Callbacks of TryAdvanceGenerationOnDevice (slab_runtime.hpp:81-84); return true to continue. */
typedef bool (*nwg_post_fitness_fn)(nwg_runtime *runtime, const nwg_runtime_word_counts *counts, void *user);
typedef bool (*nwg_shard_release_fn)(nwg_runtime *runtime, const nwg_runtime_word_counts *counts,
                                     nwg_pending_injection *pending, void *user);

/* DeviceSlabGARuntimeStatusCodeString (slab_runtime.hpp:186). */
const char *nwg_status_string(int status);

int nwg_abi_version(void);

/* UploadTrainingWordCatalogToDeviceConstantMemory (training_folder/training_data.hpp:375).
 * letters: word_count rows of 5 letter indices (0..25); process-wide, like the reference's catalog. */
int nwg_upload_catalog(const uint8_t *letters, size_t word_count);

/* TryCreateDeviceSlabGARuntimeBuffers / DestroyDeviceSlabGARuntimeBuffers (slab_runtime.hpp:119-121). */
int nwg_create(const nwg_runtime_config *config, nwg_runtime **runtime_out);
void nwg_destroy(nwg_runtime *runtime);

/* Issue this runtime's device work on `cuda_stream` (a cudaStream_t; NULL = legacy default stream). */
int nwg_set_stream(nwg_runtime *runtime, void *cuda_stream);

int nwg_get_info(const nwg_runtime *runtime, nwg_runtime_info *info);

/* Selects how nwg_evaluate / nwg_advance score actions (NWG_FORM_*). No reference counterpart. The two
 * tensor-core scoring forms keep the FP32 trunk, score on tcgen05 and re-score in FP32 every 32-action chunk
 * within a proven error bound of the best, so their guesses equal the plain form's. The two tensor-core trunk
 * forms also run the encoder and the trunk on tcgen05 and send uncertain steps through the exact FP32 path
 * (nwg_set_margin_guard). All four keep a 16-bit embedding table per individual on the device (about 128
 * bytes per action); the trunk forms add a 296 KB weight table per individual. */
int nwg_set_evaluation_form(nwg_runtime *runtime, int form);

/* Margin guard of the tensor-core trunk forms (NWG_FORM_TC_TRUNK_*). No reference counterpart. A game step whose
 * top-2 margin among unguessed actions, on the 16-bit scores, is not positive or is below tau * spread, with
 * spread = sqrt(sum_k p_k^2 var_a(e_ak)) the game's score scale (an estimate of the standard deviation of its
 * scores over the actions), is recomputed by the exact FP32 path (the plain form's chains), so its guess is the
 * plain form's. Default tau = 1e-3; tau = 0 keeps only the positive-margin test (uncertifiable steps still fall
 * back); a huge tau sends every step through the exact path. Negative or non-finite tau is rejected. */
int nwg_set_margin_guard(nwg_runtime *runtime, float tau);

/* Poll limit of every bounded mbarrier wait in the tensor-core evaluation kernels (default 2^26; no counterpart in
 * the reference, whose kernels have no such waits). A wait that reaches it gives up: the evaluation stops issuing
 * copies and tensor-core work, waits (bounded) for what is in flight, releases tensor memory and returns
 * NWG_TIMEOUT, the sticky-first-failure convention of slab_runtime.cu:288-290; the runtime stays usable. A limit
 * of 0 gives up at the first wait whose phase has not completed yet, which is how the tests exercise that path. */
int nwg_set_wait_limit(nwg_runtime *runtime, uint32_t polls);

/* TryBootstrapRandomCurrentGenerationOnDevice (slab_runtime.hpp:123-124). */
int nwg_bootstrap(nwg_runtime *runtime, size_t generation_size, uint32_t generation_seed, size_t generation_index);

/* Explicit per-cell training-word lists (CSR: cell c's words are words[offsets[c] .. offsets[c+1]),
 * catalog indices). No reference counterpart: while set, evaluation takes each cell's words from this
 * list instead of the reference shard set, so per-cell secret sets of any size can be expressed.
 * Passing cell_count = 0 returns to the shard set. */
int nwg_set_cell_words(nwg_runtime *runtime, const uint32_t *offsets, const uint32_t *words, size_t cell_count);

/* TryEvaluateCurrentGenerationFitnessOnDevice (slab_runtime.hpp:137-139). history may be NULL. */
int nwg_evaluate(nwg_runtime *runtime, const nwg_runtime_word_counts *counts,
                 const nwg_shard_release_history *history);

/* TryReadPopulationFitnessSummaryFromDevice (slab_runtime.hpp:141-142). */
int nwg_read_summary(const nwg_runtime *runtime, nwg_fitness_summary *summary);

int nwg_read_evaluation_stats(const nwg_runtime *runtime, nwg_evaluation_stats *stats);

/* Solve rate of each individual of the last evaluation: games won / games played (3 per local word), and their
 * mean. No reference counterpart (the reference reports fitness only). rates may be NULL. */
int nwg_read_solve_rates(const nwg_runtime *runtime, float *rates, size_t capacity, size_t *count_out,
                         double *mean_out);

/* TryAdvanceGenerationOnDevice (slab_runtime.hpp:144-150): evaluate, select, breed, mutate, swap.
 * config and pending may be NULL (reference defaults); callbacks may be NULL. */
int nwg_advance(nwg_runtime *runtime, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                const nwg_generation_assembly_config *config, const nwg_pending_injection *pending,
                nwg_post_fitness_fn post_fitness, void *post_fitness_user, nwg_shard_release_fn shard_release,
                void *shard_release_user, const nwg_shard_release_history *history);

/* Whether each word (5 letter indices 0..25) has the hint-grid group an injection needs (wordle/hint_grid.hpp:76-164;
 * output_embedding_injection.hpp:123-131 rejects an injection of a word without one). Host only: available[i] = 1
 * or 0. NWG_INVALID_RUNTIME_CONFIG for a letter out of range. */
int nwg_hint_groups_available(const uint8_t *letters, size_t count, uint8_t *available);

/* Graphed generation step (no reference counterpart): the same generation as nwg_advance without callbacks or
 * shard history, with its device work (evaluation, summary, selection, slot plan, breeding and mutation) captured
 * as one CUDA graph and launched once; the host then checks the status and swaps the generations. The graph is
 * captured from the same launch code every generation and updated into one executable graph, so the children
 * and fitness are those of nwg_advance bit for bit. A pending injection runs as nwg_advance (the widening
 * generation is not graphed). When the runtime's stream is the legacy default stream, the graph runs on a
 * stream of the runtime's own after the default stream has drained.
 * While tuning is on (the default), the first three generations at each (action width, form) try launch shapes in
 * turn (two or one persistent evaluation CTAs per SM, 4, 8 or 16 children per breeding CTA), timing each kernel
 * with CUDA events, and every later generation at that width uses the fastest; once one CTA per SM has lost by
 * more than 20% for a form, later widths time only two. The results do not depend on the shapes. */
int nwg_advance_graphed(nwg_runtime *runtime, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                        const nwg_generation_assembly_config *config, const nwg_pending_injection *pending);

typedef struct {
    size_t launches;        /* graph launches */
    size_t instantiations;  /* executable graphs built */
    size_t updates;         /* executable graph updated in place from a new capture */
} nwg_graph_info;

int nwg_read_graph_info(const nwg_runtime *runtime, nwg_graph_info *info);

typedef struct {
    int decided;          /* 1 once every candidate shape has been timed */
    int trials;           /* graphed generations run at this width and form */
    int eval_ctas;        /* persistent evaluation CTAs chosen (0: not decided) */
    int breed_warps;      /* children per breeding CTA chosen (0: not decided) */
    float eval_ms[2];     /* mean evaluation-kernel time at two and at one CTA per SM (0: not tried) */
    float breed_ms[3];    /* breeding-kernel time at 4, 8 and 16 children per CTA */
} nwg_launch_tuning;

/* The tuning state for one action width (the genome's action count) and evaluation form. */
int nwg_read_launch_tuning(const nwg_runtime *runtime, size_t action_width, int form, nwg_launch_tuning *out);
/* Turns the launch-shape tuning of nwg_advance_graphed on (default) or off (default shapes). */
int nwg_set_launch_tuning(nwg_runtime *runtime, int enabled);

/* The two halves of nwg_advance (TryPreparePrebreedingBoundaryOnDevice and TryAssemblePreparedGenerationOnDevice,
 * slab_runtime.cu:1374-1680). prepare evaluates the current generation, runs the callbacks, sizes the next
 * generation and plans its parents; assemble breeds (and, when an injection is pending, widens and injects) the
 * planned children and swaps them in. Between the two the runtime sits at the pre-breeding boundary that
 * checkpoints capture. assemble without a prepared generation returns NWG_INVALID_ASSEMBLY_PLAN. */
int nwg_prepare_generation(nwg_runtime *runtime, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                           const nwg_generation_assembly_config *config, const nwg_pending_injection *pending,
                           nwg_post_fitness_fn post_fitness, void *post_fitness_user,
                           nwg_shard_release_fn shard_release, void *shard_release_user,
                           const nwg_shard_release_history *history);
int nwg_assemble_prepared(nwg_runtime *runtime);

/* GenotypeSlabLayout (genotype_slab/layout.hpp:20-25). */
typedef struct {
    size_t action_count;
    size_t slot_stride_bytes;
    size_t slot_count;
    size_t slab_bytes;
} nwg_slab_layout;

/* CellularGridShape (spatial/grid.hpp:17-21). */
typedef struct {
    size_t row_count;
    size_t column_count;
    size_t cell_count;
} nwg_grid_shape;

/* RuntimeCheckpoint (slab_runtime.hpp:86-117) with its vectors as arrays: the pre-breeding boundary of one
 * generation step (evaluated, parents planned, nothing bred yet). Arrays filled by nwg_checkpoint_capture or
 * nwg_checkpoint_read are malloc-owned; release them with nwg_checkpoint_free. A caller-built checkpoint may
 * point anywhere (nwg_checkpoint_write and nwg_checkpoint_restore only read it). */
typedef struct {
    uint32_t schema_version;              /* 3 */
    uint32_t genome_layout_version;       /* 1 */
    uint32_t resume_phase;                /* 1: before recombination and mutation */
    uint64_t checksum;                    /* nwg_checkpoint_checksum */
    uint64_t training_data_identity_hash; /* nwg_checkpoint_identity_hash */
    uint32_t generation_seed;
    nwg_runtime_word_counts runtime_word_counts;
    nwg_shard_release_history training_shard_release_history;
    nwg_generation_assembly_config assembly_config;
    nwg_pending_injection pending_output_embedding_injection;
    nwg_runtime_config runtime_config;
    nwg_slab_layout slab_layout;
    nwg_grid_shape current_grid_shape;
    nwg_grid_shape next_grid_shape;
    nwg_grid_shape epicenter_grid_shape;
    size_t generation_index;
    size_t individual_count;
    uint32_t *slot_indices;        /* [individual_count]; 0xFFFFFFFF for a parent no child references */
    float *fitness;                /* [individual_count] */
    uint32_t *evaluation_counts;   /* [individual_count] */
    uint8_t *has_fitness;          /* [individual_count] */
    size_t child_count;
    uint32_t *parent_pairs;        /* [child_count][2] (SlabParentPair) */
    size_t live_count;
    uint32_t *live_organisms;      /* [live_count] organism (individual) index of each genome record */
    uint8_t *live_genomes;         /* [live_count][slab_layout.slot_stride_bytes] genome images */
} nwg_checkpoint;

/* TryCreatePrebreedingCheckpointOnDevice (slab_runtime.hpp:151-157): nwg_prepare_generation, then the boundary
 * downloaded into *checkpoint (slab_runtime.cu:1260-1372). The runtime stays prepared: nwg_assemble_prepared
 * continues it exactly as nwg_advance would have. catalog_letters (catalog_count rows of 5 letter indices) may be
 * NULL; when given it enters the training-data identity hash, like the reference's host catalog. When an
 * injection is pending the checkpoint describes the widened slab, as the reference's does: the layout at the new
 * action count, each parent's genome zero-padded to the new stride. */
int nwg_checkpoint_capture(nwg_runtime *runtime, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                           const nwg_generation_assembly_config *config, const nwg_pending_injection *pending,
                           nwg_post_fitness_fn post_fitness, void *post_fitness_user,
                           nwg_shard_release_fn shard_release, void *shard_release_user,
                           const nwg_shard_release_history *history, const uint8_t *catalog_letters,
                           size_t catalog_count, nwg_checkpoint *checkpoint);

/* TryRestorePrebreedingCheckpointToDevice (slab_runtime.hpp:159): a new runtime holding the checkpoint's
 * generation (fitness kept), genomes and parent plan, prepared for assembly. NWG_INVALID_CHECKPOINT when a check
 * of the reference's fails (versions, resume phase, checksum, layout, records, plan). The new runtime evaluates in
 * the plain form and has no per-cell word lists until they are set again. */
int nwg_checkpoint_restore(const nwg_checkpoint *checkpoint, nwg_runtime **runtime_out);

/* TryResumeGenerationFromCheckpointOnDevice (slab_runtime.hpp:161-162): assemble the restored boundary. */
int nwg_checkpoint_resume(nwg_runtime *runtime);

/* TryWriteRuntimeCheckpointAtomically / TryReadRuntimeCheckpoint (slab_runtime.hpp:164-167): the reference's file
 * format byte for byte (little-endian, records at their LP64 sizes), written to path.tmp and renamed. write
 * refuses a checkpoint whose checksum field is stale; read rejects a bad magic, version or checksum. */
int nwg_checkpoint_write(const nwg_checkpoint *checkpoint, const char *path);
int nwg_checkpoint_read(const char *path, nwg_checkpoint *checkpoint);
void nwg_checkpoint_free(nwg_checkpoint *checkpoint);

/* ComputeRuntimeCheckpointChecksum (slab_runtime.cu:1205-1248): FNV-1a 64 over the fields in file order. */
uint64_t nwg_checkpoint_checksum(const nwg_checkpoint *checkpoint);

/* The training-data identity hash of TryDownloadBoundaryCheckpointPayload (slab_runtime.cu:1283-1297): FNV-1a 64
 * over the word counts, the release history (may be NULL) and the catalog (may be NULL). */
uint64_t nwg_checkpoint_identity_hash(const nwg_runtime_word_counts *counts, const nwg_shard_release_history *history,
                                      const uint8_t *catalog_letters, size_t catalog_count);

/* WinnerArtifactMetadata (model_artifact/winner_artifact.hpp:12-21) without its path member, which the artefact
 * calls take as a string. */
typedef struct {
    float best_fitness;
    size_t generation_index;
    size_t best_index;
    uint32_t best_slot_index;
    size_t action_count;
    size_t genome_byte_count;
    uint32_t seed;
} nwg_winner_metadata;

/* TryWriteWinnerArtifactToPaths (model_artifact/winner_artifact.hpp:33-36): genome_byte_count bytes of the genome
 * image to binary_path and the reference's JSON metadata (format_version 2, the first action_count catalog words)
 * to metadata_path, each through path.tmp and a rename. timestamp_local NULL = now, local time. */
int nwg_winner_artifact_write(const char *binary_path, const char *metadata_path, const uint8_t *genome_bytes,
                              const nwg_winner_metadata *metadata, const uint8_t *catalog_letters,
                              size_t catalog_count, const char *action_space_path, const char *timestamp_local);

/* TryPersistWinningGenome (cli/run_genetic_algorithm.cu:1519-1532): the last evaluation's best individual (its
 * summary and slot image) written as a winner artefact. */
int nwg_winner_artifact_persist(const nwg_runtime *runtime, uint32_t seed, const uint8_t *catalog_letters,
                                size_t catalog_count, const char *action_space_path, const char *binary_path,
                                const char *metadata_path, const char *timestamp_local);

/* TryReadWinnerArtifact (model_artifact/winner_artifact_reader.hpp:20-21). Any output but metadata may be NULL;
 * catalog_letters holds up to NWG_CATALOG_CAPACITY rows of 5 letter indices. */
int nwg_winner_artifact_read(const char *binary_path, const char *metadata_path, nwg_winner_metadata *metadata,
                             uint8_t *genome_bytes, size_t genome_capacity, uint8_t *catalog_letters,
                             size_t *catalog_count, char *action_space_path, size_t path_capacity,
                             char *timestamp_local, size_t timestamp_capacity);

/* GenerationFitnessTelemetryRow (cli/run_genetic_algorithm.cu:594-610). */
typedef struct {
    size_t generation;
    size_t population_size;
    size_t training_word_count;
    float fitness_min;
    float fitness_mean;
    float fitness_median;
    float fitness_p90;
    float fitness_p99;
    float fitness_max;
    float fitness_stddev;
    size_t distinct_fitness_count;
    bool has_breeding_metrics;
    size_t parent_childless_count;
    size_t parent_one_child_count;
    size_t parent_multiple_children_count;
} nwg_fitness_telemetry;

/* GeneticConvergenceTelemetryRow (cli/run_genetic_algorithm.cu:612-624); elapsed_ms is device time here. */
typedef struct {
    size_t generation;
    size_t sample_organisms;
    size_t sample_weights;
    size_t pair_count;
    float centroid_distance_mean;
    float centroid_distance_min;
    float centroid_distance_max;
    float pairwise_distance_mean;
    float pairwise_distance_min;
    float pairwise_distance_max;
    float elapsed_ms;
} nwg_convergence_telemetry;

/* The adaptive release thresholds of the reference CLI (run_genetic_algorithm.cu:94-101); its defaults
 * (training_folder/training_data.hpp:17-20) are 3, 10, 6.0 and 0.20. */
typedef struct {
    size_t min_gap_generations;
    size_t first_new_release_generation;
    float centroid_distance_threshold;
    float fitness_p99_threshold;
} nwg_shard_release_policy;

/* TryCollectGenerationFitnessTelemetry (cli/run_genetic_algorithm.cu:1080-1186) on the GPU: the current
 * generation's fitness min, mean, median, p90 and p99 (nearest rank), max, population standard deviation and
 * distinct-value count, bit-identical to the reference's host sort and sequential double sums; with
 * with_breeding, the last plan's childless / one-child / several-children parent counts. counts may be NULL
 * (training_word_count 0). Populations up to 32,768 (NWG_UNSUPPORTED beyond); NWG_POPULATION_NOT_EVALUATED when an
 * individual has no fitness. */
int nwg_fitness_telemetry_collect(const nwg_runtime *runtime, const nwg_runtime_word_counts *counts,
                                  bool with_breeding, nwg_fitness_telemetry *row);

/* TryCollectGeneticConvergenceTelemetry (cli/run_genetic_algorithm.cu:941-1054) on the GPU: the sample plan
 * (genetic_convergence.hpp:86-119: 256 organisms, 8,192 trainable scalars, 512 pairs, seeded by run seed and
 * generation) gathered from the slab and reduced to centroid and pairwise distances, bit-identical to the
 * reference's TryComputeMetrics. */
int nwg_convergence_telemetry_collect(const nwg_runtime *runtime, uint32_t run_seed, nwg_convergence_telemetry *row);

/* MakeSamplePlan (genetic_convergence.hpp:86-119): organisms[<=256], weights[<=8192], pairs[512][2]. */
int nwg_convergence_sample_plan(size_t organism_count, size_t trainable_count, uint32_t run_seed, size_t generation,
                                uint32_t *organisms, size_t *organism_count_out, uint32_t *weights,
                                size_t *weight_count_out, uint32_t *pairs, size_t *pair_count_out);

/* TryMaybeReleaseTrainingDataShard (cli/run_genetic_algorithm.cu:1199-1282): after the foundation release and the
 * gap rules, releases the next word_count_step catalog words when the centroid distance mean is at most its
 * threshold and the fitness p99 exceeds its threshold: records the release in history and fills pending (for
 * nwg_advance) and next_word_count. Meant for the shard-release callback. The telemetry rows it computed are
 * returned when the pointers are not NULL (left zero when a gap rule decided). */
int nwg_maybe_release_training_shard(const nwg_runtime *runtime, const nwg_runtime_word_counts *counts,
                                     const nwg_shard_release_policy *policy, size_t catalog_word_count,
                                     uint32_t run_seed, nwg_shard_release_history *history,
                                     nwg_pending_injection *pending, size_t *next_word_count,
                                     nwg_fitness_telemetry *fitness_row, nwg_convergence_telemetry *convergence_row);

/* Single-model inference (inference/single_model_device_runtime.hpp:22-47): one genome and its own action-space
 * catalog on the device. */
typedef struct nwg_single_model nwg_single_model;

/* SelectedAction (model/output_embedding/output_embedding.hpp:35-39). */
typedef struct {
    uint8_t word[5];      /* letter indices */
    float score;
    size_t action_index;
} nwg_selected_action;

/* TryCreateSingleModelDeviceRuntime (single_model_device_runtime.hpp:38-40): genome_byte_count must be the
 * stride of catalog_count actions (NWG_INVALID_RUNTIME_CONFIG otherwise). */
int nwg_single_model_create(const uint8_t *genome_bytes, size_t genome_byte_count, const uint8_t *catalog_letters,
                            size_t catalog_count, nwg_single_model **model_out);
void nwg_single_model_destroy(nwg_single_model *model);
int nwg_single_model_set_stream(nwg_single_model *model, void *cuda_stream);

/* TrySelectNextGuessWithSingleModelDeviceRuntime (single_model_device_runtime.hpp:44-47) for grid_count grids in
 * one call: grid g has turn_counts[g] turns, turn u's guess at guess_letters[(g*6+u)*5 ..] (letter indices) and
 * its tiles at feedback[(g*6+u)*5 ..] (0 green, 1 yellow, 2 grey). Each selection is the reference's: FP32 scores
 * over the whole catalog, words already guessed masked, ties to the lowest index. A grid with more than five
 * turns, a won turn or an invalid letter or tile gives NWG_POLICY_FORWARD_FAILED (the reference's
 * kPolicyForwardFailed) and no selection; a grid whose every action is guessed gives NWG_ACTION_SELECTION_FAILED
 * (its action zeroed, the others filled). */
int nwg_single_model_select(nwg_single_model *model, const uint8_t *guess_letters, const uint8_t *feedback,
                            const uint8_t *turn_counts, size_t grid_count, nwg_selected_action *actions);

/* The learned surrogate's network (no reference counterpart): an MLP 8,192 -> 512 -> 128 -> 1 with GELU, BF16
 * weights in the products, FP32 masters, FP32 accumulation, Adam (lr given, beta 0.9 / 0.999, eps 1e-8). Inputs are
 * device buffers of BF16 descriptors, [rows][8192], rows a multiple of 128 (NWG_UNSUPPORTED otherwise) and at most
 * the capacity given at creation. Parameters are one flat FP32 vector: W1 [512][8192], b1, W2 [128][512], b2,
 * w3 [128], b3. */
typedef struct nwg_mlp nwg_mlp;
int nwg_mlp_create(size_t capacity_rows, uint32_t seed, float learning_rate, nwg_mlp **out);
void nwg_mlp_destroy(nwg_mlp *mlp);
int nwg_mlp_set_stream(nwg_mlp *mlp, void *cuda_stream);
size_t nwg_mlp_parameter_count(void);
/* Copies the parameters out to host_out and/or in from host_in (either may be NULL). */
int nwg_mlp_parameters(nwg_mlp *mlp, float *host_out, const float *host_in);
/* y (device, rows floats) = the network's outputs. */
int nwg_mlp_forward(nwg_mlp *mlp, const uint16_t *x, size_t rows, float *y);
/* Gradients of mean((y - t)^2) (t: device targets) into grads_out (host, parameter_count floats; may be NULL) and
 * the loss; no update. */
int nwg_mlp_gradients(nwg_mlp *mlp, const uint16_t *x, const float *targets, size_t rows, float *grads_out,
                      float *loss_out);
/* One Adam step on mean((y - t)^2). */
int nwg_mlp_train_step(nwg_mlp *mlp, const uint16_t *x, const float *targets, size_t rows);

/* Behavioural descriptors (no reference counterpart): for each of count genomes (device slab, slot indices on the
 * device), its FP32 policy vectors on the 128 probe states, times scale, rounded to BF16, into out[count][8192]
 * (device). Probe p has probe_turns[p] <= 4 turns, guess and tiles of turn u at probe_letters / probe_feedback
 * [(p * 4 + u) * 5 ..] (host arrays). Synchronises the stream. */
int nwg_descriptors(const void *slab, size_t pitch, const uint32_t *slots, size_t count, const uint8_t *probe_letters,
                    const uint8_t *probe_feedback, const uint8_t *probe_turns, float scale, uint16_t *out,
                    void *cuda_stream);

/* Test hook: the 16-bit score table (column maxima, K-major tiles, per-tile column moments) that the last evaluation
 * in a tensor-core form built for one individual of the evaluated generation; bytes_out gets its size (host_out
 * NULL: size only). NWG_POPULATION_NOT_EVALUATED when no such evaluation ran. */
int nwg_read_score_table(const nwg_runtime *runtime, size_t individual, void *host_out, size_t capacity,
                         size_t *bytes_out);

/* Test hook: C[m][n] FP32 = A[m][k] . B[n][k]^T on tcgen05 (BF16 device operands, K contiguous); m % 128, n % 256,
 * k % 64, lda % 8, ldb % 8 and ldc % 4 zero, bases 16-byte aligned (NWG_UNSUPPORTED otherwise). */
int nwg_bf16_gemm_nt(const void *a, size_t lda, const void *b, size_t ldb, float *c, size_t ldc, size_t m, size_t n,
                     size_t k, void *cuda_stream);

/* Surrogate-screened generation step (no reference counterpart): each cell breeds candidates_per_cell children, the
 * network (nwg_mlp) scores their behavioural descriptors (policy vectors on 128 fixed probe states of 0..4 turns),
 * and only the best-scored child of each cell plus an audit sample is played; every child is played instead while
 * the network is untrained, while the replay ring holds fewer than warmup_pairs pairs, or when the last audit's
 * Spearman rank correlation fell below spearman_floor. Played (descriptor, fitness) pairs train the network online
 * (train_steps Adam steps of batch_rows rows from a replay ring of replay_capacity pairs, targets standardised per
 * minibatch). The population must have per-cell word lists (nwg_set_cell_words) and keeps its size. */
typedef struct {
    size_t candidates_per_cell;   /* 4 */
    float audit_fraction;         /* 0.05 of the candidates */
    float spearman_floor;         /* 0.6 */
    size_t replay_capacity;       /* 65,536 */
    size_t warmup_pairs;          /* pairs in the ring before screening may start */
    size_t train_steps;           /* per generation */
    size_t batch_rows;            /* a multiple of 128 */
    float learning_rate;          /* Adam; 1e-4 */
    uint32_t seed;                /* probes, network initialisation, audit and minibatch draws */
    int evaluation_form;          /* NWG_FORM_* used to play the children (NWG_FORM_TC_TRUNK_FP16) */
    float margin_tau;             /* its margin guard (trunk forms) */
} nwg_surrogate_config;

typedef struct {
    size_t generation;            /* index of the generation installed */
    size_t candidates;            /* children bred */
    size_t evaluated;             /* children played */
    bool screened;                /* false: every child was played */
    float spearman;               /* audit rank correlation of score and fitness (NaN while untrained) */
    float train_loss;             /* standardised MSE on the last minibatch */
    size_t train_steps;
    size_t replay_size;
    double mean_fitness;          /* of the new generation */
    double mean_solve_rate;
    /* on a step that played every child (NaN otherwise; the model's pick also NaN while untrained): the mean
     * fitness of the model's best-scored child per cell, of candidate 0 (the plain step's child) and of the truly
     * best child per cell, all from the same brood */
    double mean_fitness_model_pick;
    double mean_fitness_first_candidate;
    double mean_fitness_best_candidate;
    uint64_t game_steps;          /* decisions played this step */
    float ms_select_breed, ms_descriptors, ms_inference, ms_evaluation, ms_training, ms_install, ms_total;
} nwg_surrogate_stats;

typedef struct nwg_surrogate nwg_surrogate;

/* runtime: the population (evaluated or not, per-cell word lists set); catalog_letters: the uploaded catalog's rows
 * (probe words); secret_pool: catalog indices the probes' secrets come from (NULL: the selectable words). */
int nwg_surrogate_create(nwg_runtime *runtime, const nwg_surrogate_config *config, const uint8_t *catalog_letters,
                         size_t catalog_count, const uint32_t *secret_pool, size_t pool_count,
                         nwg_surrogate **surrogate_out);
void nwg_surrogate_destroy(nwg_surrogate *surrogate);
/* One surrogate-screened step of the population (config: selection radius and exponent, breeding, mutation). */
int nwg_surrogate_advance(nwg_surrogate *surrogate, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                          const nwg_generation_assembly_config *config, nwg_surrogate_stats *stats);

/* SwapDeviceSlabGenerationBuffers (slab_runtime.hpp:181). */
int nwg_swap_generations(nwg_runtime *runtime);

/* TryReadDeviceSlabGARuntimeStatus (slab_runtime.hpp:183-184). */
int nwg_read_status(const nwg_runtime *runtime, int *status);

/* TryDownloadCurrentGenerationFromDevice (slab_runtime.hpp:131-132). Arrays hold `capacity` entries. */
int nwg_download_current_generation(const nwg_runtime *runtime, uint32_t *slot_indices, float *fitness,
                                    uint32_t *evaluation_counts, uint8_t *has_fitness, size_t capacity,
                                    size_t *count_out, size_t *generation_index_out);

/* TryDownloadNextGenerationFromDevice (slab_runtime.hpp:134-135): the other generation buffer (after an advance,
 * the parents). */
int nwg_download_next_generation(const nwg_runtime *runtime, uint32_t *slot_indices, float *fitness,
                                 uint32_t *evaluation_counts, uint8_t *has_fitness, size_t capacity,
                                 size_t *count_out, size_t *generation_index_out);

/* TryDownloadSlabSlotBytesFromDevice (slab_runtime.hpp:128-129): the slot's genome image,
 * slot_stride_bytes long, byte-identical to the reference layout. */
int nwg_download_slot(const nwg_runtime *runtime, uint32_t slot_index, uint8_t *bytes, size_t capacity,
                      size_t *byte_count_out);

/* TryUploadSlabToDevice / TryUploadCurrentGenerationToDevice (genotype_slab/device_runtime.hpp:89-93):
 * place a genome image in a slot, and set the current generation's slot list. */
int nwg_upload_slot(nwg_runtime *runtime, uint32_t slot_index, const uint8_t *bytes, size_t byte_count);
int nwg_upload_current_generation(nwg_runtime *runtime, const uint32_t *slot_indices, size_t count,
                                  size_t generation_index);

/* The assembly plan of the last advance: count (first, second) parent indices (SlabParentPair,
 * genotype_slab/assembly.hpp:12-15). */
int nwg_download_assembly_plan(const nwg_runtime *runtime, uint32_t *pairs, size_t capacity, size_t *count_out);

/* Test and benchmark hooks (no reference counterpart). */
int nwg_device_slab(const nwg_runtime *runtime, void **slab_out, size_t *pitch_out);

/* Evaluation with per-episode trace of the first trace_episodes episodes of every individual
 * (device buffers, each may be NULL): choices[ind][e][6], turns[ind][e], scores[ind][e],
 * policy[ind][e][6][64]. */
int nwg_evaluate_traced(nwg_runtime *runtime, const nwg_runtime_word_counts *counts,
                        const nwg_shard_release_history *history, size_t trace_episodes, void *choices,
                        void *turns, void *scores, void *policy);

/* Parent selection and child assembly as separate device steps over caller buffers (device pointers),
 * for differential tests: select writes child_count pairs; breed writes child i to child_slab slot i. */
int nwg_select_parents_device(const float *fitness, const uint8_t *has_fitness, size_t population,
                              size_t columns, size_t child_count, size_t generation_index,
                              const nwg_parent_selection_config *config, uint32_t planning_seed, uint32_t *pairs,
                              void *cuda_stream);
int nwg_breed_device(const void *parent_slab, size_t parent_pitch, const uint32_t *parent_slots,
                     void *child_slab, size_t child_pitch, const uint32_t *pairs, size_t child_count,
                     size_t action_count, uint32_t generation_seed, size_t generation_index,
                     const nwg_breeding_config *breeding, const nwg_mutation_config *mutation, void *cuda_stream);
int nwg_bootstrap_device(void *slab, size_t pitch, size_t population, size_t generation_index, uint32_t seed,
                         size_t action_count, void *cuda_stream);

/* FP32 fused multiply-add throughput of the current device in TFLOP/s, measured by a short kernel of independent
 * FMA chains on every SM (no counterpart in the reference): the roofline denominator of the FP32 evaluation forms.
 * Allocates a few bytes, synchronises the stream. */
int nwg_measure_fp32_peak(double *tflops_out, void *cuda_stream);

/* ---- Row bands: one population split by grid rows across ranks (no counterpart in the reference, which runs on
 * one GPU). The split follows the path's own dependencies: evaluation is per individual; selection reads the
 * fitness of the Moore neighbourhood (selection_ops.cuh:218-263, spatial/grid.hpp:181-218), so a band selects over
 * the whole grid's fitness, gathered by the caller; breeding reads the two parents' genomes
 * (genome_ops.cuh:386-407), which for children on a band's edge lie up to `radius` rows into the neighbouring
 * band, so each band holds `halo_rows` rows above and below it, copied in by the caller. Children keep their
 * whole-grid indices in every Philox stream, so the bands together produce exactly the children of a single
 * runtime holding the whole grid.
 *
 * nwg_set_band: this runtime holds rows [band_row_first, band_row_first + rows) of a grid of global_rows rows
 * (rows = population_size_ceiling / grid_column_count); the top 2 * halo_rows * columns slots of its slab hold the
 * halo (create it with room for two band generations plus those slots). global_rows = 0 returns to a whole
 * population. The whole-grid paths (nwg_prepare_generation, nwg_advance, nwg_advance_graphed) return
 * NWG_UNSUPPORTED in band mode; nwg_bootstrap of a band (its full size) draws its rows' organisms of the whole
 * grid's generation. Per generation:
 *   nwg_evaluate (the band's own cells, set by nwg_set_cell_words in band order);
 *   nwg_device_generation -> the band's fitness and has-fitness device arrays, gathered by the caller into the
 *     whole grid's arrays (band k at offset k * band cells);
 *   nwg_band_prepare: selection for the band's children over the whole grid (radius <= halo_rows, <= 2);
 *   nwg_band_copy_rows: band rows [band_row, band_row + rows) into a device buffer (the halo a neighbour needs);
 *   nwg_band_install_halo: the rows above (global rows first - halo .. first - 1) and below (first + rows ..),
 *     halo_rows * columns genomes each at src_pitch, from device buffers;
 *   nwg_assemble_prepared: breed the band's children and make them the current generation. */
int nwg_set_band(nwg_runtime *runtime, size_t global_rows, size_t band_row_first, size_t halo_rows);
int nwg_device_generation(const nwg_runtime *runtime, void **fitness, void **has_fitness, size_t *count);
int nwg_band_prepare(nwg_runtime *runtime, uint32_t generation_seed, const nwg_generation_assembly_config *config,
                     const float *fitness_all, const uint8_t *has_fitness_all);
int nwg_band_copy_rows(nwg_runtime *runtime, size_t band_row, size_t rows, void *dst, size_t dst_pitch);
int nwg_band_install_halo(nwg_runtime *runtime, const void *above, const void *below, size_t src_pitch);

/* Fitness evaluation that allocates no device memory. No counterpart in the reference.
 * For callers that cannot call cudaMalloc: embedders whose device memory belongs to another allocator or
 * pool, and processes that keep a fixed device-memory footprint after start-up (a late allocation can fail
 * or stall the device). Every pointer is a device pointer the caller
 * owns: the slab (individual i's genome image at slab + slot_indices[i] * slot_pitch), the catalog as
 * rows of 5 letter indices, the per-cell word lists in CSR form (catalog indices), and the outputs
 * fitness[population] and, when not NULL, counters[3] (game steps, encoded turns, episodes). The
 * selectable actions are catalog words [0, action_count). Everything else lives in one fixed array of
 * 4,789,760 bytes inside the library, which every GPU that loads the library holds until the process
 * exits; it limits population to 4,096 and the catalog to 4,739 words (NWG_UNSUPPORTED beyond). All
 * calls share that array and it keeps the last call's contents, so calls that overlap on the GPU (other
 * streams or host threads) race and must be serialised by the caller. The first call on each device
 * resolves the array's device address (cudaGetSymbolAddress with that device current). A cell whose
 * offsets decrease, or whose list is empty or longer than 2^20 words, gives NWG_INVALID_TRAINING_SHARD
 * without a read of its words. population 0 gives NWG_INVALID_RUNTIME_CONFIG. The call synchronises its
 * stream and returns the evaluation status. */
int nwg_evaluate_noalloc(const void *slab, size_t slot_pitch, const uint32_t *slot_indices, size_t population,
                         size_t grid_column_count, size_t action_count, const uint8_t *catalog_letters,
                         size_t catalog_count, const uint32_t *cell_offsets, const uint32_t *cell_words,
                         float *fitness, uint64_t *counters, void *cuda_stream);

#ifdef __cplusplus
}
#endif

#endif /* NWG_CAPI_H */
