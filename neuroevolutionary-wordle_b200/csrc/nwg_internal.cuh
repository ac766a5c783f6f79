// Internal kernel interfaces of the runtime (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_layout.cuh"

namespace nwg {

// Status codes: the reference's DeviceSlabGARuntimeStatusCode values
// (genetic_algorithm/device/slab_runtime.hpp:21-39) followed by this runtime's additions.
enum Status : int {
    kOk = 0,
    kCudaFailure = 1,
    kInvalidRuntimeConfig = 2,
    kInvalidSlab = 3,
    kInvalidGeneration = 4,
    kInvalidTrainingShard = 5,
    kGuessAppendFailed = 6,
    kPolicyForwardFailed = 7,
    kActionSelectionFailed = 8,
    kPopulationNotEvaluated = 9,
    kInvalidAssemblyConfig = 10,
    kParentSelectionFailed = 11,
    kInvalidAssemblyPlan = 12,
    kInvalidParentIndex = 13,
    kSlabFull = 14,
    kOutputEmbeddingInjectionFailed = 15,
    kSlabRepackFailed = 16,
    kTimeout = 17,
    kUnsupported = 18,
    kInvalidCheckpoint = 19,
};

__device__ inline void SetStatus(int *status, int code) { atomicCAS(status, 0, code); }

// Where each cell's local training words come from: the reference shard set
// (training_data.hpp:251-316) or an explicit per-cell list (CSR).
struct WordSource {
    int mode;  // 0: CSR lists, 1: shard records
    const std::uint32_t *cell_offsets;
    const std::uint32_t *cell_words;
    const ShardRecord *shards;
    std::uint32_t shard_count;
    std::uint32_t rows;
    std::uint32_t cols;
};

// ---- fitness evaluation (plain FP32 form) ----
constexpr int kEvalThreads = 256;
constexpr int kChunkGames = 128;
// Longest word list a cell may have (2^20 words: three chunk counts per cell stay far from 32-bit overflow).
constexpr std::uint32_t kMaxCellWords = 1u << 20;

struct EvalParams {
    const std::uint8_t *slab;
    std::size_t pitch;
    const std::uint32_t *slot_of_individual;
    std::uint32_t population;
    std::uint32_t action_count;       // selectable actions
    std::uint32_t catalog_count;
    const std::uint32_t *codes;       // packed catalog words
    const float *fixed_t;             // [26][action_pad] fixed word features
    std::uint32_t action_pad;
    WordSource source;
    const std::uint32_t *chunk_start; // [population + 1]; chunk_start[population] = total chunks
    const std::uint32_t *local_words; // [population]
    float *scratch;                   // per CTA: kChunkGames x 256 layer-1 accumulators
    std::uint32_t *score_sum;         // [population]
    std::uint32_t *won_sum;           // [population] games won (may be null)
    unsigned long long *steps;        // [0] policy decisions, [1] turns encoded, [2] episodes
    int *status;
    // optional trace (null when unused)
    std::int32_t *trace_choices;      // [population * trace_episodes * 6]
    std::int32_t *trace_turns;        // [population * trace_episodes]
    float *trace_scores;              // [population * trace_episodes]
    float *trace_policy;              // [population * trace_episodes * 6 * 64]
    std::uint32_t trace_episodes;
    // the per-individual exact trunk tables (LaunchBuildExactTrunkTables), or null: the FP32 forms then stage the
    // weights from the genome itself
    const std::uint8_t *xt;
    std::size_t xt_pitch;
};

std::size_t EvalScratchFloatsPerCta();
int EvalCtaCount(std::uint32_t total_chunks);
cudaError_t LaunchEvalPrepare(const WordSource &source, std::uint32_t population, std::uint32_t catalog_count,
                              std::uint32_t *local_words, std::uint32_t *chunk_start, std::uint32_t *score_sum,
                              int *status, cudaStream_t stream);
cudaError_t LaunchEvalFp32(const EvalParams &params, int cta_count, cudaStream_t stream);
cudaError_t LaunchFinalizeFitness(const std::uint32_t *score_sum, const std::uint32_t *local_words,
                                  std::uint32_t population, float *fitness, std::uint32_t *evaluation_counts,
                                  std::uint8_t *has_fitness, int *status, cudaStream_t stream);

// Per-individual exact trunk tables (trunk_table.cu): the encoder and trunk weights as FP32 [input][output] blocks for
// the FP32 forms' streamed policy path.
std::size_t ExactTrunkTablePitch();
cudaError_t LaunchBuildExactTrunkTables(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                        std::uint32_t population, std::uint8_t *tables, cudaStream_t stream);

// ---- fitness evaluation, tensor-core scoring form ----
std::size_t TcTablePitch(std::uint32_t action_count);
cudaError_t LaunchBuildTcTables(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                std::uint32_t population, const float *fixed_t, std::uint32_t action_pad,
                                std::uint32_t action_count, std::uint8_t *tables, bool fp16, bool with_moments,
                                cudaStream_t stream);
// Polls of a bounded mbarrier wait in the tensor-core evaluation kernels before it gives up with NWG_TIMEOUT.
constexpr std::uint32_t kDefaultWaitLimit = 1u << 26;
cudaError_t LaunchEvalTc(const EvalParams &params, const std::uint8_t *tables, std::size_t table_pitch, float kappa,
                         bool fp16, unsigned long long *tc_counters, int cta_count, cudaStream_t stream,
                         std::uint32_t wait_limit = kDefaultWaitLimit);

// ---- fitness evaluation, tensor-core trunk form ----
std::size_t TrunkTablePitch();
cudaError_t LaunchBuildTrunkTables(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                   std::uint32_t population, std::uint8_t *tables, bool fp16, cudaStream_t stream);
cudaError_t LaunchEvalTct(const EvalParams &params, const std::uint8_t *embed_tables, std::size_t embed_pitch,
                          const std::uint8_t *trunk_tables, float tau, bool fp16, unsigned long long *counters,
                          int cta_count, cudaStream_t stream, std::uint32_t wait_limit = kDefaultWaitLimit);

struct SummaryDevice {
    float best_fitness;
    float average_fitness;
    std::uint64_t best_index;
    std::uint32_t best_slot_index;
    std::uint32_t pad;
    double mean_fp64;
    double variance_fp64;
};

cudaError_t LaunchSummarize(const float *fitness, const std::uint8_t *has_fitness, const std::uint32_t *slots,
                            std::uint32_t population, SummaryDevice *out, int *status, cudaStream_t stream);

// ---- selection ----
struct SelectParams {
    const float *fitness;
    const std::uint8_t *has_fitness;
    std::uint32_t rows;
    std::uint32_t cols;
    std::uint32_t child_count;
    std::uint64_t generation_index;
    std::uint64_t radius;
    float rank_exponent;
    std::uint32_t planning_seed;
    std::uint32_t *pairs;  // [child_count * 2]
    int *status;
    std::uint32_t child_first;  // global index of child 0 (a band of a larger grid; 0 for a whole population)
};
cudaError_t LaunchSelect(const SelectParams &params, cudaStream_t stream);

// ---- breeding ----
struct BreedParams {
    const std::uint8_t *parent_slab;
    std::size_t parent_pitch;
    const std::uint32_t *parent_slots;  // slot of each current individual
    std::uint8_t *child_slab;
    std::size_t child_pitch;
    const std::uint32_t *child_slots;   // slot of each child (null: child i at slot i)
    const std::uint32_t *pairs;
    std::uint32_t child_count;
    std::uint32_t action_count;
    std::uint32_t generation_seed;
    std::uint64_t generation_index;
    float crossover_l1, crossover_l2, crossover_l3;
    float mutation_probability, mutation_sigma, row_scale_probability;
    int *status;
    std::uint32_t child_first;  // global index of child 0: its Philox subsequence (0 for a whole population)
};
cudaError_t LaunchBreed(const BreedParams &params, cudaStream_t stream, int warps_per_cta = 4);

// ---- output-embedding injection (action-space growth) ----
cudaError_t LaunchInject(std::uint8_t *slab, std::size_t pitch, const std::uint32_t *child_slots,
                         std::uint32_t child_count, std::uint32_t parent_action_count, std::uint32_t injection_count,
                         const std::uint32_t *guess_codes, const std::uint16_t *tiles, const int4 *chunks,
                         const std::uint32_t *order, int chunk_count, float *scratch, float *sums, int cta_count,
                         int *status, cudaStream_t stream);

// ---- bootstrap ----
// Organism i is organism organism_first + i of a population of stream_population (0: population) in the
// random-stream map.
cudaError_t LaunchBootstrap(std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                            std::uint32_t population, std::uint64_t generation_index, std::uint32_t seed,
                            std::uint32_t action_count, cudaStream_t stream, std::uint32_t organism_first = 0,
                            std::uint32_t stream_population = 0);

// ---- the pre-breeding boundary, for checkpoints (checkpoint.cu) ----

// What a prepared runtime holds between nwg_prepare_generation and nwg_assemble_prepared, in the reference's
// terms: slab_bytes is GenotypeSlabLayout::slab_bytes (slot_count x stride at creation, kept across widening).
struct BoundaryState {
    std::uint32_t seed;
    nwg_generation_assembly_config config;
    nwg_pending_injection injection;
    std::size_t action_count, next_action_count, stride, slot_count, slab_bytes;
    std::size_t generation_byte_budget, host_spill_budget, max_generation_size, grid_column_count, epicenter_rows;
    std::size_t generation_index, generation_size, planned_children;
};

// kInvalidAssemblyPlan when the runtime is not prepared.
int ReadBoundary(const nwg_runtime *rt, BoundaryState *out);

// Device buffers of the current generation, for read-only consumers (telemetry.cu). Pointers are the runtime's.
struct GenerationView {
    cudaStream_t stream;
    const std::uint8_t *slab;
    std::size_t pitch, action_count;
    const std::uint32_t *slots;
    const float *fitness;
    const std::uint8_t *has_fitness;
    const std::uint32_t *pairs;  // the last plan's (first, second) parent indices
    std::size_t generation_index, generation_size, planned_children;
    std::size_t grid_column_count, stride, slot_count;
    const std::uint32_t *cell_offsets, *cell_words;  // per-cell word lists (CSR), when set
    std::size_t cell_count;
    bool evaluated;  // the current generation's fitness is from an evaluation of this generation
    int *status;
};
int ReadGenerationView(const nwg_runtime *rt, GenerationView *out);

// Makes `count` genomes held elsewhere (src_slab at src_pitch, host slot list) the runtime's next generation with
// their known fitness (one evaluation each), copied into slots the current generation does not use, and swaps
// it in; the population size and pitch must be the runtime's.
int InstallGeneration(nwg_runtime *rt, const std::uint8_t *src_slab, std::size_t src_pitch,
                      const std::vector<std::uint32_t> &src_slots, const std::vector<float> &fitness,
                      std::size_t generation_index);

// Device catalog tables: packed words [pad] and fixed word features [26][pad], pad = word count rounded up to 128.
int BuildCatalogTables(const std::uint8_t *letters, std::size_t word_count, std::uint32_t **codes_out,
                       float **fixed_out, std::size_t *pad_out, std::vector<std::uint32_t> *host_codes);

// Single-model inference (eval_fp32.cu): grids grouped in chunks of up to 128 with one turn count each.
struct SingleModelParams {
    const std::uint8_t *genome;      // one genome image
    std::uint32_t action_count;
    const std::uint32_t *codes;      // the model's catalog
    const float *fixed_t;
    std::uint32_t action_pad;
    const std::uint32_t *guess_codes;  // [grid][5 turns]
    const std::uint16_t *tiles;        // [grid][5 turns]
    const int4 *chunks;                // {turns, first entry of order, grids, 0}
    const std::uint32_t *order;        // grid indices, grouped by turn count
    int chunk_count;
    float *scratch;                    // per CTA: layer-1 accumulators
    std::int32_t *best_index;          // [grid]; -1 when every action is masked
    float *best_score;                 // [grid]
};
cudaError_t LaunchSingleModelSelect(const SingleModelParams &params, int cta_count, cudaStream_t stream);

// Behavioural descriptors (eval_fp32.cu): each genome's FP32 policy vectors on 128 fixed probe states of 0..4
// turns, scaled and rounded to BF16, row g of the output = [probe][64] of genome g.
constexpr int kProbeStates = 128;
constexpr int kProbeMaxTurns = 4;
constexpr int kDescriptorWidth = kProbeStates * 64;  // 8,192
struct DescriptorParams {
    const std::uint8_t *slab;
    std::size_t pitch;
    const std::uint32_t *slots;        // genome g at slab + slots[g] * pitch
    std::uint32_t count;
    const std::uint32_t *probe_codes;  // [probe][4] packed guesses
    const std::uint16_t *probe_tiles;  // [probe][4] packed feedback
    const std::uint8_t *probe_turns;   // [probe]
    float scale;                       // applied before the BF16 rounding
    float *scratch;                    // per CTA: layer-1 accumulators
    std::uint16_t *out;                // [count][8192] BF16 bits, row stride out_ld elements
    std::size_t out_ld;
};
cudaError_t LaunchDescriptors(const DescriptorParams &params, int cta_count, cudaStream_t stream);

// C[M][N] FP32 = A[M][K] . B[N][K]^T on tcgen05, A and B BF16 with K contiguous (surrogate_mlp.cu). M % 128,
// N % 256, K % 64, lda % 8, ldb % 8 and ldc % 4 must be zero and the bases 16-byte aligned (cudaErrorInvalidValue
// otherwise); *error is set to 1 when a bounded wait gave up.
cudaError_t LaunchGemmNt(const void *a, std::size_t lda, const void *b, std::size_t ldb, float *c, std::size_t ldc,
                         std::size_t m, std::size_t n, std::size_t k, int *error, cudaStream_t stream);

// A runtime with explicit sizes (a restored checkpoint's, slab_runtime.cu:1746-1765).
struct RuntimeShape {
    std::size_t action_count, slot_count, slab_bytes, max_generation_size, grid_column_count;
    std::size_t generation_byte_budget, host_spill_budget, epicenter_rows;
};
int CreateShapedRuntime(const RuntimeShape &shape, nwg_runtime **out);

// Installs a restored boundary: the current generation (slots may be 0xFFFFFFFF for released parents, which no
// child references; evaluation is refused until the next swap), its fitness, the parent plan and the assembly
// inputs; the runtime is left prepared.
int InstallBoundary(nwg_runtime *rt, const std::uint32_t *slots, const float *fitness, const std::uint32_t *eval,
                    const std::uint8_t *has, std::size_t count, std::size_t generation_index,
                    const std::uint32_t *pairs, std::size_t child_count, std::uint32_t seed,
                    const nwg_generation_assembly_config &config, const nwg_pending_injection &injection,
                    std::size_t next_action_count);

// Raises a kernel's dynamic shared memory limit on the current device. The limit belongs to each device's
// context, so `devices_done` keeps one bit per device ordinal and the attribute is set once per device.
template <typename Kernel>
inline cudaError_t RaiseSharedLimit(Kernel kernel, int bytes, std::atomic<unsigned long long> &devices_done) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        return e;
    }
    const unsigned long long bit = 1ull << (device & 63);
    if ((devices_done.load(std::memory_order_acquire) & bit) != 0) {
        return cudaSuccess;
    }
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) {
        devices_done.fetch_or(bit, std::memory_order_acq_rel);
    }
    return e;
}

}  // namespace nwg
