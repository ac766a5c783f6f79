// Host runtime behind the C ABI (include/nwg_capi.h).
//
// Mirrors the reference's device GA runtime (genetic_algorithm/device/slab_runtime.cu) at its public
// entry points, with B200-first internals:
//   - the slab is a planned slot array (no device free list, no spin lock, no host spill): the
//     current generation's slots are fixed, and before assembly one kernel marks the parents the plan
//     references and hands the remaining slots to the children in ascending order;
//   - the whole generation (evaluate -> finalize -> summary -> select -> plan slots -> breed) is issued
//     on the runtime's stream with no intermediate host synchronisation; the call synchronises once at
//     the end and reads the sticky device status, which keeps the reference's "bool + status" contract.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

using namespace nwg;

namespace {

constexpr std::size_t kMaxSizeT = std::numeric_limits<std::size_t>::max();

struct Catalog {
    std::uint32_t *codes = nullptr;  // device
    float *fixed_t = nullptr;        // device [26][pad]
    std::size_t count = 0;
    std::size_t pad = 0;
    int device = -1;
    std::vector<std::uint32_t> host_codes;  // packed words, for the hint grids of injected words
};

Catalog g_catalog;
std::mutex g_catalog_mutex;

}  // namespace

struct nwg_runtime {
    cudaStream_t stream = nullptr;
    std::size_t action_count = 0;
    std::size_t stride = 0;
    std::size_t pitch = 0;
    std::size_t slot_count = 0;
    std::size_t max_generation_size = 0;
    std::size_t grid_column_count = 0;
    std::size_t generation_byte_budget = 0;
    std::size_t slab_byte_budget = 0;
    std::size_t host_spill_budget = 0;
    std::size_t epicenter_rows = 0;

    std::uint8_t *slab = nullptr;
    std::uint32_t *cur_slots = nullptr, *next_slots = nullptr;
    float *cur_fitness = nullptr, *next_fitness = nullptr;
    std::uint32_t *cur_eval = nullptr, *next_eval = nullptr;
    std::uint8_t *cur_has = nullptr, *next_has = nullptr;
    std::uint32_t *pairs = nullptr;
    std::uint8_t *slot_used = nullptr;
    std::size_t cur_gen_index = 0, cur_gen_size = 0, next_gen_index = 0, next_gen_size = 0, planned_children = 0;

    int *status = nullptr;
    SummaryDevice *summary = nullptr;
    ShardRecord *shards = nullptr;
    std::size_t shard_count = 0;
    std::uint32_t *cell_offsets = nullptr, *cell_words = nullptr;
    std::size_t cell_count = 0, cell_word_capacity = 0;
    std::uint32_t *local_words = nullptr, *chunk_start = nullptr, *score_sum = nullptr, *won_sum = nullptr;
    unsigned long long *steps = nullptr;
    float *scratch = nullptr;
    int scratch_ctas = 0;
    int form = NWG_FORM_FP32;
    std::uint8_t *tc_tables = nullptr;
    std::size_t tc_tables_bytes = 0;
    std::size_t last_table_pitch = 0;  // of the tables the last tensor-core evaluation built (0: none)
    std::uint8_t *trunk_tables = nullptr;
    std::uint8_t *xt_tables = nullptr;  // exact trunk tables of the FP32 forms (ExactTrunkTablePitch per individual)
    float margin_tau = 1.0e-3f;
    std::uint32_t wait_limit = kDefaultWaitLimit;  // bounded mbarrier waits of the tensor-core kernels
    // a generation prepared for assembly (evaluated and planned; nwg_prepare_generation / checkpoint restore)
    bool prepared = false;
    std::uint32_t prepared_seed = 0;
    nwg_generation_assembly_config prepared_config{};
    nwg_pending_injection prepared_injection{};
    std::size_t prepared_next_action_count = 0;
    // the current generation holds released parents (slot 0xFFFFFFFF), as a restored boundary does; it can only
    // be assembled, not evaluated
    bool released_parents = false;
    // the win counters describe the current generation (false after a generation is installed with known fitness)
    bool rates_valid = false;

    // pinned host staging
    ShardRecord *host_shards = nullptr;
    int *host_status = nullptr;
    SummaryDevice *host_summary = nullptr;
    // [9]: decisions, encoded turns, episodes, re-scored chunks, full rows (scoring forms), then candidate
    // chunks, fallback steps, exact chunks, exact rows (trunk forms)
    unsigned long long *host_steps = nullptr;
    cudaEvent_t eval_begin = nullptr;
    cudaEvent_t eval_end = nullptr;
    std::uint64_t last_episodes = 0;
    // launch shapes: CTAs of the persistent evaluation kernels (0: scratch_ctas) and children per breeding CTA
    int eval_ctas = 0;
    int breed_warps = 4;
    cudaEvent_t breed_begin = nullptr;
    cudaEvent_t breed_end = nullptr;
    // graphed generations (nwg_advance_graphed) and the online launch-shape tuning per (width, form)
    cudaStream_t own_stream = nullptr;  // capture stream when the caller's stream is the legacy default stream
    cudaGraphExec_t graph_exec = nullptr;
    nwg_graph_info graph{};
    bool autotune = true;
    std::map<std::uint64_t, nwg_launch_tuning> tuning;
    std::map<int, bool> single_cta_lost;  // per form: one evaluation CTA per SM lost by more than 20% at some width
    std::size_t last_eval_population = 0;
    std::size_t last_action_count = 0;
    std::size_t last_eval_generation = 0;
    // row band of a population split across ranks (nwg_set_band): this runtime holds rows
    // [band_row_first, band_row_first + band rows) of a grid of band_global_rows rows; the halo rows above and below
    // live in the top band_reserved_slots slots, which children never take
    bool band = false;
    std::size_t band_global_rows = 0, band_row_first = 0, band_halo_rows = 0, band_reserved_slots = 0;
    std::uint32_t *band_parent_table = nullptr;  // [global population]: parent index -> slot (0xFFFFFFFF: absent)
    bool band_halo_ready = false;                // the halo of the current generation is installed
};

namespace {

constexpr int kStepCounters = 9;

#define NWG_TRY(expr)                                \
    do {                                             \
        if ((expr) != cudaSuccess) {                 \
            return kCudaFailure;                     \
        }                                            \
    } while (0)

// ---- byte budgets (genetic_algorithm/genome/dynamic_layout.hpp:38-54, spatial/grid.hpp:61-67) ----
std::size_t SlotsForBudget(std::size_t budget, std::size_t action_count, std::size_t ceiling = 0) {
    const std::size_t stride = GenomeStrideBytes(action_count);
    if (stride == 0 || budget < stride) {
        return 0;
    }
    const std::size_t n = budget / stride;
    return (ceiling == 0 || n < ceiling) ? n : ceiling;
}

std::size_t FloorRows(std::size_t n, std::size_t cols) { return cols == 0 ? 0 : (n / cols) * cols; }

// slab_runtime.hpp:50-60
bool ValidConfig(const nwg_runtime_config &c) {
    return c.genotype_slab_byte_budget_bytes >= c.generation_byte_budget_bytes && c.action_count > 0 &&
           c.grid_column_count > 0 && (c.population_size_ceiling == 0 || c.population_size_ceiling % c.grid_column_count == 0) &&
           SlotsForBudget(c.genotype_slab_byte_budget_bytes, c.action_count) > 0 &&
           SlotsForBudget(c.generation_byte_budget_bytes, c.action_count, c.population_size_ceiling) / c.grid_column_count > 0;
}

// ---- training-data shard set (training_folder/training_data.hpp:73-117, :150-206, :251-316) ----
bool ValidSchedule(const nwg_word_count_schedule &s) {
    return s.initial_word_count > 0 && s.word_count_step_period_generations > 0;
}

std::size_t ShardCountForIntroduced(const nwg_word_count_schedule &s, std::size_t introduced) {
    if (!ValidSchedule(s) || introduced == 0) {
        return 0;
    }
    const std::size_t foundation = std::min(s.initial_word_count, introduced);
    if (introduced == foundation) {
        return 1;
    }
    if (s.word_count_step == 0) {
        return 0;
    }
    return 1 + (introduced - foundation + s.word_count_step - 1) / s.word_count_step;
}

bool ValidHistoryFor(const nwg_word_count_schedule &s, std::size_t introduced, const nwg_shard_release_history &h) {
    const std::size_t required = ShardCountForIntroduced(s, introduced);
    if (required == 0 || h.release_count == 0 || h.release_count > NWG_CATALOG_CAPACITY) {
        return false;
    }
    for (std::size_t i = 1; i < h.release_count; ++i) {
        if (h.release_generations[i] <= h.release_generations[i - 1]) {
            return false;
        }
    }
    return h.release_count >= required;
}

std::size_t RadiusAtGeneration(std::size_t intro, std::size_t current, std::size_t initial, std::size_t period) {
    if (period == 0 || current < intro) {
        return 0;
    }
    const std::size_t steps = (current - intro) / period;
    if (steps > kMaxSizeT - initial) {
        return kMaxSizeT;
    }
    return initial + steps;
}

bool BuildShardSet(const nwg_runtime_word_counts &wc, std::size_t generation_index, std::size_t rows,
                   std::size_t cols, std::size_t epicenter_rows, const nwg_shard_release_history *history,
                   std::vector<ShardRecord> &out) {
    out.clear();
    const std::size_t introduced = wc.training_word_count;
    const nwg_word_count_schedule &s = wc.training_word_schedule;
    if (!ValidSchedule(s) || introduced == 0 || introduced > NWG_CATALOG_CAPACITY || rows == 0 || cols == 0 ||
        epicenter_rows == 0 || wc.shard_radius_growth_period_generations == 0) {
        return false;
    }
    if (history != nullptr && !ValidHistoryFor(s, introduced, *history)) {
        return false;
    }
    const std::size_t foundation = std::min(s.initial_word_count, introduced);
    out.push_back(ShardRecord{0, foundation, 0, 0, 0, 1});
    if (s.word_count_step == 0 || foundation == introduced) {
        return true;
    }
    std::size_t next = foundation;
    std::size_t local = 0;
    const std::size_t epicenter_cells = epicenter_rows * cols;
    while (next < introduced) {
        const std::size_t count = std::min(introduced - next, s.word_count_step);
        const std::size_t history_index = out.size();
        const std::size_t intro = history == nullptr ? (local + 1) * s.word_count_step_period_generations
                                                     : history->release_generations[history_index];
        // DeterministicTrainingShardCenterCoordinate: golden-ratio stride over the epicentre grid
        const std::size_t cell =
            static_cast<std::size_t>((static_cast<std::uint64_t>(local + 1) * 11400714819323198485ull) % epicenter_cells);
        const std::size_t row = cell / cols;
        const std::size_t col = cell % cols;
        out.push_back(ShardRecord{next, count, std::min(row, rows - 1), col,
                                  RadiusAtGeneration(intro, generation_index, wc.shard_initial_radius,
                                                     wc.shard_radius_growth_period_generations),
                                  0});
        next += count;
        ++local;
    }
    return true;
}

int Sync(nwg_runtime *rt) {
    if (cudaMemcpyAsync(rt->host_status, rt->status, sizeof(int), cudaMemcpyDeviceToHost, rt->stream) != cudaSuccess ||
        cudaStreamSynchronize(rt->stream) != cudaSuccess) {
        return kCudaFailure;
    }
    return *rt->host_status;
}

int SetHostStatus(nwg_runtime *rt, int code) {
    *rt->host_status = code;
    cudaMemcpyAsync(rt->status, rt->host_status, sizeof(int), cudaMemcpyHostToDevice, rt->stream);
    cudaStreamSynchronize(rt->stream);
    return code;
}

// ---- hint grids of a newly released word (wordle/hint_grid.hpp:76-162) ----
constexpr std::uint32_t kAllYellow = 0x155u;  // every position's 2-bit tile is 1 (yellow)

std::uint32_t RotateCode(std::uint32_t code, int rotation) {  // hint_grid.hpp:19-27 (rotate left)
    std::uint8_t letters[kWordLength];
    for (int p = 0; p < kWordLength; ++p) {
        letters[p] = static_cast<std::uint8_t>(WordLetter(code, (p + rotation) % kWordLength));
    }
    return PackWord(letters);
}

int CountTiles(std::uint32_t feedback, std::uint32_t tile) {
    int n = 0;
    for (int p = 0; p < kWordLength; ++p) {
        n += ((feedback >> (2 * p)) & 3u) == tile;
    }
    return n;
}

struct HintGroup {
    int turns[3] = {0, 0, 0};
    std::uint32_t guess[3][4] = {};
    std::uint16_t tiles[3][4] = {};
};

// The cyclic grid (the word's distinct left rotations whose feedback is all yellow), then the first two
// distinct letter swaps whose feedback is three green and two yellow; false when the word has no such group.
bool BuildHintGroup(std::uint32_t word, HintGroup &g) {
    g = HintGroup{};
    for (int rotation = 1; rotation < kWordLength; ++rotation) {
        const std::uint32_t guess = RotateCode(word, rotation);
        bool seen = guess == word;
        for (int t = 0; t < g.turns[0]; ++t) {
            seen |= g.guess[0][t] == guess;
        }
        const std::uint32_t fb = FeedbackPacked(guess, word);
        if (seen || fb != kAllYellow) {
            continue;
        }
        g.guess[0][g.turns[0]] = guess;
        g.tiles[0][g.turns[0]] = static_cast<std::uint16_t>(fb);
        ++g.turns[0];
    }
    int selected = 0;
    for (int i = 0; i < kWordLength && selected < 2; ++i) {
        for (int j = i + 1; j < kWordLength && selected < 2; ++j) {
            if (WordLetter(word, i) == WordLetter(word, j)) {
                continue;
            }
            std::uint8_t letters[kWordLength];
            for (int p = 0; p < kWordLength; ++p) {
                letters[p] = static_cast<std::uint8_t>(WordLetter(word, p));
            }
            std::swap(letters[i], letters[j]);
            const std::uint32_t guess = PackWord(letters);
            const std::uint32_t fb = FeedbackPacked(guess, word);
            if (CountTiles(fb, kGreen) != 3 || CountTiles(fb, kYellow) != 2 ||
                (selected == 1 && g.guess[1][0] == guess)) {
                continue;
            }
            g.turns[1 + selected] = 1;
            g.guess[1 + selected][0] = guess;
            g.tiles[1 + selected][0] = static_cast<std::uint16_t>(fb);
            ++selected;
        }
    }
    return selected == 2;
}

__global__ void PlanChildSlotsKernel(const std::uint32_t *pairs, std::uint32_t child_count,
                                     const std::uint32_t *parent_slots, std::uint32_t parent_count,
                                     std::uint8_t *used, std::uint32_t slot_count, std::uint32_t *child_slots,
                                     int *status, std::uint32_t parent_slot_limit) {
    __shared__ std::uint32_t partial[1024];
    __shared__ std::uint32_t base;
    const std::uint32_t t = threadIdx.x;
    for (std::uint32_t s = t; s < slot_count; s += blockDim.x) {
        used[s] = 0;
    }
    __syncthreads();
    for (std::uint32_t c = t; c < child_count; c += blockDim.x) {
        const std::uint32_t a = pairs[2 * c];
        const std::uint32_t b = pairs[2 * c + 1];
        // parents held in slots at or above slot_count (a band's halo rows) are valid up to parent_slot_limit and
        // are never candidates for a child's slot
        if (a >= parent_count || b >= parent_count || parent_slots[a] >= parent_slot_limit ||
            parent_slots[b] >= parent_slot_limit) {
            SetStatus(status, kInvalidParentIndex);
            continue;
        }
        if (parent_slots[a] < slot_count) {
            used[parent_slots[a]] = 1;
        }
        if (parent_slots[b] < slot_count) {
            used[parent_slots[b]] = 1;
        }
    }
    if (t == 0) {
        base = 0;
    }
    __syncthreads();
    for (std::uint32_t start = 0; start < slot_count; start += blockDim.x) {
        const std::uint32_t s = start + t;
        const std::uint32_t is_free = (s < slot_count && used[s] == 0) ? 1u : 0u;
        partial[t] = is_free;
        __syncthreads();
        for (std::uint32_t off = 1; off < blockDim.x; off <<= 1) {
            const std::uint32_t v = t >= off ? partial[t - off] : 0;
            __syncthreads();
            partial[t] += v;
            __syncthreads();
        }
        const std::uint32_t index = base + partial[t] - is_free;
        if (is_free && index < child_count) {
            child_slots[index] = s;
        }
        __syncthreads();
        if (t == blockDim.x - 1) {
            base += partial[t];
        }
        __syncthreads();
    }
    if (t == 0 && base < child_count) {
        SetStatus(status, kSlabFull);
    }
}

// Copies whole slots (pitch bytes, 16-byte vectors) from one slab to another: slot src_slots[i] to dst_slots[i].
__global__ void CopySlotsKernel(const std::uint8_t *src, std::size_t src_pitch, const std::uint32_t *src_slots,
                                std::uint8_t *dst, std::size_t dst_pitch, const std::uint32_t *dst_slots,
                                std::uint32_t n) {
    const std::size_t vectors = dst_pitch / 16;
    for (std::uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint4 *s = reinterpret_cast<const uint4 *>(src + static_cast<std::size_t>(src_slots[i]) * src_pitch);
        uint4 *d = reinterpret_cast<uint4 *>(dst + static_cast<std::size_t>(dst_slots[i]) * dst_pitch);
        for (std::size_t v = threadIdx.x; v < vectors; v += blockDim.x) {
            d[v] = s[v];
        }
    }
}

// Copies `n` genomes (`bytes` per genome, a multiple of 16) from slots src_slots[i] to dst + i * dst_pitch.
__global__ void GatherSlotsKernel(const std::uint8_t *src, std::size_t src_pitch, const std::uint32_t *src_slots,
                                  std::uint8_t *dst, std::size_t dst_pitch, std::size_t bytes, std::uint32_t n) {
    const std::size_t vectors = bytes / 16;
    for (std::uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint4 *s = reinterpret_cast<const uint4 *>(src + static_cast<std::size_t>(src_slots[i]) * src_pitch);
        uint4 *d = reinterpret_cast<uint4 *>(dst + static_cast<std::size_t>(i) * dst_pitch);
        for (std::size_t v = threadIdx.x; v < vectors; v += blockDim.x) {
            d[v] = s[v];
        }
    }
}

// The band's parent table over the whole grid: its own rows at their slots, the halo rows above (global rows
// first - halo .. first - 1, toroidal) and below (first + band .. first + band + halo - 1) at the reserved slots
// from reserved_base on, every other cell absent.
__global__ void BandParentTableKernel(std::uint32_t *table, std::uint32_t global_rows, std::uint32_t cols,
                                      std::uint32_t first_row, std::uint32_t band_rows, std::uint32_t halo_rows,
                                      const std::uint32_t *band_slots, std::uint32_t reserved_base) {
    const std::uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= global_rows * cols) {
        return;
    }
    const std::uint32_t row = g / cols;
    const std::uint32_t col = g - row * cols;
    const std::uint32_t offset = (row + global_rows - first_row) % global_rows;  // rows after the band's first row
    std::uint32_t slot = 0xFFFFFFFFu;
    if (offset < band_rows) {
        slot = band_slots[offset * cols + col];
    } else if (offset < band_rows + halo_rows) {  // below the band
        slot = reserved_base + (halo_rows + offset - band_rows) * cols + col;
    } else if (offset >= global_rows - halo_rows) {  // above the band
        slot = reserved_base + (offset - (global_rows - halo_rows)) * cols + col;
    }
    table[g] = slot;
}

void FreeRuntime(nwg_runtime *rt) {
    if (rt == nullptr) {
        return;
    }
    void *device_ptrs[] = {rt->slab,       rt->cur_slots,    rt->next_slots,  rt->cur_fitness, rt->next_fitness,
                           rt->cur_eval,   rt->next_eval,    rt->cur_has,     rt->next_has,    rt->pairs,
                           rt->slot_used,  rt->status,       rt->summary,     rt->shards,      rt->cell_offsets,
                           rt->cell_words, rt->local_words,  rt->chunk_start, rt->score_sum,   rt->steps,
                           rt->won_sum,
                           rt->scratch,    rt->tc_tables,    rt->trunk_tables, rt->band_parent_table,
                           rt->xt_tables};
    for (void *p : device_ptrs) {
        if (p != nullptr) {
            cudaFree(p);
        }
    }
    void *host_ptrs[] = {rt->host_shards, rt->host_status, rt->host_summary, rt->host_steps};
    for (void *p : host_ptrs) {
        if (p != nullptr) {
            cudaFreeHost(p);
        }
    }
    if (rt->eval_begin != nullptr) {
        cudaEventDestroy(rt->eval_begin);
    }
    if (rt->eval_end != nullptr) {
        cudaEventDestroy(rt->eval_end);
    }
    if (rt->breed_begin != nullptr) {
        cudaEventDestroy(rt->breed_begin);
    }
    if (rt->breed_end != nullptr) {
        cudaEventDestroy(rt->breed_end);
    }
    if (rt->graph_exec != nullptr) {
        cudaGraphExecDestroy(rt->graph_exec);
    }
    if (rt->own_stream != nullptr) {
        cudaStreamDestroy(rt->own_stream);
    }
    delete rt;
}

// A timing event: a plain record, or an event node of the graph while the stream is being captured.
cudaError_t RecordEvent(cudaEvent_t event, cudaStream_t stream) {
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (stream != nullptr && cudaStreamIsCapturing(stream, &capture) == cudaSuccess &&
        capture == cudaStreamCaptureStatusActive) {
        return cudaEventRecordWithFlags(event, stream, cudaEventRecordExternal);
    }
    return cudaEventRecord(event, stream);
}

// CTAs of the persistent evaluation kernels: the tuned count, never more than the scratch holds.
// The FP32 forms' exact trunk tables, allocated on first use. Never while the runtime's stream is being captured
// (an allocation would break the capture): that evaluation then stages the weights from the genome, with the same
// results; so does one whose allocation fails.
void EnsureExactTrunkTables(nwg_runtime *rt) {
    if (rt->xt_tables != nullptr) {
        return;
    }
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    if (rt->stream != nullptr && cudaStreamIsCapturing(rt->stream, &capture) == cudaSuccess &&
        capture != cudaStreamCaptureStatusNone) {
        return;
    }
    if (cudaMalloc(&rt->xt_tables, rt->max_generation_size * ExactTrunkTablePitch()) != cudaSuccess) {
        rt->xt_tables = nullptr;
        (void)cudaGetLastError();
    }
}

int EvalGrid(const nwg_runtime *rt) {
    return rt->eval_ctas > 0 && rt->eval_ctas < rt->scratch_ctas ? rt->eval_ctas : rt->scratch_ctas;
}

bool ValidWordCounts(const nwg_runtime_word_counts &wc, std::size_t catalog_count) {
    // evaluation_ops.cuh:77-85
    return wc.training_word_count <= catalog_count && wc.action_space_word_count <= catalog_count &&
           wc.training_word_count <= wc.action_space_word_count && ValidSchedule(wc.training_word_schedule) &&
           wc.shard_radius_growth_period_generations > 0;
}

int EvaluateImpl(nwg_runtime *rt, const nwg_runtime_word_counts *counts, const nwg_shard_release_history *history,
                 std::size_t trace_episodes, void *choices, void *turns, void *scores, void *policy) {
    if (rt == nullptr || counts == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (rt->max_generation_size == 0 || rt->cur_gen_size == 0 || rt->cur_gen_size > rt->max_generation_size ||
        rt->cur_gen_size % rt->grid_column_count != 0 || rt->released_parents) {
        return kInvalidGeneration;
    }
    NWG_TRY(cudaMemsetAsync(rt->status, 0, sizeof(int), rt->stream));
    const std::size_t rows = rt->cur_gen_size / rt->grid_column_count;
    const std::size_t cols = rt->grid_column_count;
    const std::size_t selectable = std::min(rt->action_count, counts->action_space_word_count);
    if (g_catalog.codes == nullptr || !ValidWordCounts(*counts, g_catalog.count) || selectable == 0) {
        return SetHostStatus(rt, kInvalidTrainingShard);
    }
    WordSource src{};
    src.rows = static_cast<std::uint32_t>(rows);
    src.cols = static_cast<std::uint32_t>(cols);
    if (rt->cell_count > 0) {
        if (rt->cell_count != rt->cur_gen_size) {
            return SetHostStatus(rt, kInvalidTrainingShard);
        }
        src.mode = 0;
        src.cell_offsets = rt->cell_offsets;
        src.cell_words = rt->cell_words;
    } else {
        std::vector<ShardRecord> set;
        if (!BuildShardSet(*counts, rt->cur_gen_index, rows, cols, rt->epicenter_rows, history, set) ||
            set.size() > NWG_CATALOG_CAPACITY) {
            return SetHostStatus(rt, kInvalidTrainingShard);
        }
        std::memcpy(rt->host_shards, set.data(), set.size() * sizeof(ShardRecord));
        NWG_TRY(cudaMemcpyAsync(rt->shards, rt->host_shards, set.size() * sizeof(ShardRecord), cudaMemcpyHostToDevice,
                                rt->stream));
        rt->shard_count = set.size();
        src.mode = 1;
        src.shards = rt->shards;
        src.shard_count = static_cast<std::uint32_t>(set.size());
    }
    const std::uint32_t population = static_cast<std::uint32_t>(rt->cur_gen_size);
    NWG_TRY(cudaMemsetAsync(rt->cur_fitness, 0, rt->max_generation_size * sizeof(float), rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->cur_eval, 0, rt->max_generation_size * sizeof(std::uint32_t), rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->cur_has, 0, rt->max_generation_size, rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->steps, 0, kStepCounters * sizeof(unsigned long long), rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->won_sum, 0, population * sizeof(std::uint32_t), rt->stream));
    NWG_TRY(LaunchEvalPrepare(src, population, static_cast<std::uint32_t>(g_catalog.count), rt->local_words,
                              rt->chunk_start, rt->score_sum, rt->status, rt->stream));
    EvalParams p{};
    p.slab = rt->slab;
    p.pitch = rt->pitch;
    p.slot_of_individual = rt->cur_slots;
    p.population = population;
    p.action_count = static_cast<std::uint32_t>(selectable);
    p.catalog_count = static_cast<std::uint32_t>(g_catalog.count);
    p.codes = g_catalog.codes;
    p.fixed_t = g_catalog.fixed_t;
    p.action_pad = static_cast<std::uint32_t>(g_catalog.pad);
    p.source = src;
    p.chunk_start = rt->chunk_start;
    p.local_words = rt->local_words;
    p.scratch = rt->scratch;
    p.score_sum = rt->score_sum;
    p.won_sum = rt->won_sum;
    p.steps = rt->steps;
    p.status = rt->status;
    p.trace_episodes = static_cast<std::uint32_t>(trace_episodes);
    p.trace_choices = static_cast<std::int32_t *>(choices);
    p.trace_turns = static_cast<std::int32_t *>(turns);
    p.trace_scores = static_cast<float *>(scores);
    p.trace_policy = static_cast<float *>(policy);
    // the FP32 chains of the plain and exact forms stream their weights from the exact trunk tables
    const bool fp32_trunk = rt->form == NWG_FORM_FP32 || rt->form == NWG_FORM_TC_BF16 ||
                            rt->form == NWG_FORM_TC_FP16 || selectable <= 128;
    if (fp32_trunk) {
        EnsureExactTrunkTables(rt);
        if (rt->xt_tables != nullptr) {
            NWG_TRY(LaunchBuildExactTrunkTables(rt->slab, rt->pitch, rt->cur_slots, population, rt->xt_tables,
                                                rt->stream));
            p.xt = rt->xt_tables;
            p.xt_pitch = ExactTrunkTablePitch();
        }
    }
    // at <= 128 selectable actions every form scores on the reference's tensor-tile path, in the plain kernel
    if (rt->form == NWG_FORM_FP32 || selectable <= 128) {
        NWG_TRY(RecordEvent(rt->eval_begin, rt->stream));
        NWG_TRY(LaunchEvalFp32(p, EvalGrid(rt), rt->stream));
        NWG_TRY(RecordEvent(rt->eval_end, rt->stream));
    } else if (rt->form == NWG_FORM_TC_TRUNK_BF16 || rt->form == NWG_FORM_TC_TRUNK_FP16) {
        const bool fp16 = rt->form == NWG_FORM_TC_TRUNK_FP16;
        rt->last_table_pitch = TcTablePitch(static_cast<std::uint32_t>(selectable));
        NWG_TRY(LaunchBuildTcTables(rt->slab, rt->pitch, rt->cur_slots, population, g_catalog.fixed_t,
                                    static_cast<std::uint32_t>(g_catalog.pad), static_cast<std::uint32_t>(selectable),
                                    rt->tc_tables, fp16, true, rt->stream));
        NWG_TRY(LaunchBuildTrunkTables(rt->slab, rt->pitch, rt->cur_slots, population, rt->trunk_tables, fp16,
                                       rt->stream));
        NWG_TRY(RecordEvent(rt->eval_begin, rt->stream));
        NWG_TRY(LaunchEvalTct(p, rt->tc_tables, TcTablePitch(static_cast<std::uint32_t>(selectable)), rt->trunk_tables,
                              rt->margin_tau, fp16, rt->steps + 5, EvalGrid(rt), rt->stream, rt->wait_limit));
        NWG_TRY(RecordEvent(rt->eval_end, rt->stream));
    } else {
        const bool fp16 = rt->form == NWG_FORM_TC_FP16;
        // |16-bit product - FP32 product| <= (2u + u^2)|p||e| with u = 2^-8 (BF16: p and e rounded) or 2^-11 (FP16:
        // p rounded, e exact), plus 64-term FP32 accumulation on both sides; with a safety margin.
        const float kappa = fp16 ? 6.5e-4f : 1.0e-2f;
        rt->last_table_pitch = TcTablePitch(static_cast<std::uint32_t>(selectable));
        NWG_TRY(LaunchBuildTcTables(rt->slab, rt->pitch, rt->cur_slots, population, g_catalog.fixed_t,
                                    static_cast<std::uint32_t>(g_catalog.pad), static_cast<std::uint32_t>(selectable),
                                    rt->tc_tables, fp16, false, rt->stream));
        NWG_TRY(RecordEvent(rt->eval_begin, rt->stream));
        NWG_TRY(LaunchEvalTc(p, rt->tc_tables, TcTablePitch(static_cast<std::uint32_t>(selectable)), kappa, fp16,
                             rt->steps + 3, EvalGrid(rt), rt->stream, rt->wait_limit));
        NWG_TRY(RecordEvent(rt->eval_end, rt->stream));
    }
    NWG_TRY(LaunchFinalizeFitness(rt->score_sum, rt->local_words, population, rt->cur_fitness, rt->cur_eval,
                                  rt->cur_has, rt->status, rt->stream));
    NWG_TRY(LaunchSummarize(rt->cur_fitness, rt->cur_has, rt->cur_slots, population, rt->summary, rt->status,
                            rt->stream));
    NWG_TRY(cudaMemcpyAsync(rt->host_summary, rt->summary, sizeof(SummaryDevice), cudaMemcpyDeviceToHost, rt->stream));
    NWG_TRY(cudaMemcpyAsync(rt->host_steps, rt->steps, kStepCounters * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            rt->stream));
    rt->last_eval_population = population;
    rt->last_action_count = rt->action_count;
    rt->last_eval_generation = rt->cur_gen_index;
    rt->rates_valid = true;
    return kOk;
}

// Action-space growth (slab_runtime.cu:1464-1482, genotype_slab/device_runtime.cu:1338-1432, :518-617).
// Instead of compacting and re-laying the referenced parents in place at the wider stride (the reference's
// single-CTA PrepareSlabForExpandedActionCountKernel), the children are bred straight from the parents'
// slots into a fresh slab laid out at the new width (the breeding kernel reads and writes different pitches),
// which is the same byte movement the assembly does anyway; the old slab is then released. The new rows of
// every child are then injected on the device (inject.cu).
int AdvanceWithInjection(nwg_runtime *rt, std::uint32_t generation_seed, const nwg_generation_assembly_config &cfg,
                         const nwg_pending_injection &injection, const std::vector<HintGroup> &hints,
                         std::size_t next_action_count, std::size_t next_size) {
    const std::size_t n = injection.injection_count;
    const std::size_t parent_action_count = injection.first_catalog_word_index;
    const std::size_t new_pitch = SlotPitchBytes(next_action_count);
    const std::size_t new_slots = SlotsForBudget(rt->slab_byte_budget, next_action_count);
    if (new_slots < next_size || new_slots >= 0xFFFFFFFFull) {
        return SetHostStatus(rt, kSlabRepackFailed);
    }
    // per injected word and grid: up to four turns (packed guess, packed feedback); grids sorted by turn count
    std::vector<std::uint32_t> codes(n * 12, 0);
    std::vector<std::uint16_t> tiles(n * 12, 0);
    std::vector<std::uint32_t> order(3 * n);
    std::vector<int4> chunks;
    for (std::size_t i = 0; i < n; ++i) {
        for (int g = 0; g < 3; ++g) {
            for (int t = 0; t < hints[i].turns[g]; ++t) {
                codes[(i * 3 + g) * 4 + t] = hints[i].guess[g][t];
                tiles[(i * 3 + g) * 4 + t] = hints[i].tiles[g][t];
            }
        }
    }
    for (int g = 0; g < 3; ++g) {
        std::uint32_t *ord = order.data() + g * n;
        for (std::size_t i = 0; i < n; ++i) {
            ord[i] = static_cast<std::uint32_t>(i);
        }
        std::stable_sort(ord, ord + n, [&](std::uint32_t a, std::uint32_t b) {
            return hints[a].turns[g] < hints[b].turns[g];
        });
        std::size_t k = 0;
        while (k < n) {
            const int turns = hints[ord[k]].turns[g];
            std::size_t e = k;
            while (e < n && e - k < static_cast<std::size_t>(kChunkGames) && hints[ord[e]].turns[g] == turns) {
                ++e;
            }
            chunks.push_back(make_int4(g, turns, static_cast<int>(g * n + k), static_cast<int>(e - k)));
            k = e;
        }
    }
    std::vector<std::uint32_t> identity(next_size);
    for (std::size_t c = 0; c < next_size; ++c) {
        identity[c] = static_cast<std::uint32_t>(c);
    }
    std::uint8_t *new_slab = nullptr;
    std::uint8_t *new_used = nullptr;
    std::uint32_t *d_codes = nullptr, *d_order = nullptr;
    std::uint16_t *d_tiles = nullptr;
    int4 *d_chunks = nullptr;
    float *d_sums = nullptr;
    auto release = [&]() {
        void *ptrs[] = {d_codes, d_order, d_tiles, d_chunks, d_sums};
        for (void *p : ptrs) {
            if (p != nullptr) {
                cudaFree(p);
            }
        }
    };
    bool ok = cudaMalloc(&new_slab, new_slots * new_pitch) == cudaSuccess &&
              cudaMalloc(&new_used, new_slots) == cudaSuccess &&
              cudaMalloc(&d_codes, codes.size() * sizeof(std::uint32_t)) == cudaSuccess &&
              cudaMalloc(&d_tiles, tiles.size() * sizeof(std::uint16_t)) == cudaSuccess &&
              cudaMalloc(&d_order, order.size() * sizeof(std::uint32_t)) == cudaSuccess &&
              cudaMalloc(&d_chunks, chunks.size() * sizeof(int4)) == cudaSuccess &&
              cudaMalloc(&d_sums, static_cast<std::size_t>(rt->scratch_ctas) * n * kTailDim * sizeof(float)) ==
                  cudaSuccess;
    ok = ok && cudaMemsetAsync(new_slab, 0, new_slots * new_pitch, rt->stream) == cudaSuccess &&
         cudaMemsetAsync(new_used, 0, new_slots, rt->stream) == cudaSuccess &&
         cudaMemcpyAsync(d_codes, codes.data(), codes.size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice,
                         rt->stream) == cudaSuccess &&
         cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * sizeof(std::uint16_t), cudaMemcpyHostToDevice,
                         rt->stream) == cudaSuccess &&
         cudaMemcpyAsync(d_order, order.data(), order.size() * sizeof(std::uint32_t), cudaMemcpyHostToDevice,
                         rt->stream) == cudaSuccess &&
         cudaMemcpyAsync(d_chunks, chunks.data(), chunks.size() * sizeof(int4), cudaMemcpyHostToDevice,
                         rt->stream) == cudaSuccess &&
         cudaMemcpyAsync(rt->next_slots, identity.data(), next_size * sizeof(std::uint32_t), cudaMemcpyHostToDevice,
                         rt->stream) == cudaSuccess;
    BreedParams bp{};
    bp.parent_slab = rt->slab;
    bp.parent_pitch = rt->pitch;
    bp.parent_slots = rt->cur_slots;
    bp.child_slab = new_slab;
    bp.child_pitch = new_pitch;
    bp.child_slots = rt->next_slots;
    bp.pairs = rt->pairs;
    bp.child_count = static_cast<std::uint32_t>(next_size);
    bp.action_count = static_cast<std::uint32_t>(parent_action_count);  // the parents' rows
    bp.generation_seed = generation_seed;
    bp.generation_index = rt->cur_gen_index;
    bp.crossover_l1 = cfg.breeding.crossover_temperature_level1;
    bp.crossover_l2 = cfg.breeding.crossover_temperature_level2;
    bp.crossover_l3 = cfg.breeding.crossover_temperature_level3;
    bp.mutation_probability = cfg.mutation.mutation_probability;
    bp.mutation_sigma = cfg.mutation.mutation_sigma;
    bp.row_scale_probability = cfg.mutation.output_tail_row_scale_mutation_probability;
    bp.status = rt->status;
    ok = ok && LaunchBreed(bp, rt->stream) == cudaSuccess;
    ok = ok && LaunchInject(new_slab, new_pitch, rt->next_slots, static_cast<std::uint32_t>(next_size),
                            static_cast<std::uint32_t>(parent_action_count), static_cast<std::uint32_t>(n), d_codes,
                            d_tiles, d_chunks, d_order, static_cast<int>(chunks.size()), rt->scratch, d_sums,
                            rt->scratch_ctas, rt->status, rt->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(rt->next_fitness, 0, rt->max_generation_size * sizeof(float), rt->stream) == cudaSuccess &&
         cudaMemsetAsync(rt->next_eval, 0, rt->max_generation_size * sizeof(std::uint32_t), rt->stream) ==
             cudaSuccess &&
         cudaMemsetAsync(rt->next_has, 0, rt->max_generation_size, rt->stream) == cudaSuccess;
    const int st = ok ? Sync(rt) : kCudaFailure;
    release();
    if (st != kOk) {
        cudaFree(new_slab);
        cudaFree(new_used);
        return st;
    }
    // the children now own the widened slab
    cudaFree(rt->slab);
    cudaFree(rt->slot_used);
    rt->slab = new_slab;
    rt->slot_used = new_used;
    rt->action_count = next_action_count;
    rt->stride = GenomeStrideBytes(next_action_count);
    rt->pitch = new_pitch;
    rt->slot_count = new_slots;
    if (rt->tc_tables != nullptr) {
        // the 16-bit embedding tables are sized by the action count
        cudaFree(rt->tc_tables);
        rt->tc_tables = nullptr;
        const std::size_t bytes = rt->max_generation_size * TcTablePitch(static_cast<std::uint32_t>(next_action_count));
        if (cudaMalloc(&rt->tc_tables, bytes) != cudaSuccess) {
            rt->tc_tables = nullptr;
            rt->form = NWG_FORM_FP32;
            return SetHostStatus(rt, kCudaFailure);
        }
        rt->tc_tables_bytes = bytes;
    }
    rt->next_gen_index = rt->cur_gen_index + 1;
    rt->next_gen_size = next_size;
    return nwg_swap_generations(rt);
}

}  // namespace

namespace nwg {

int CreateShapedRuntime(const RuntimeShape &shape, nwg_runtime **out) {
    *out = nullptr;
    const std::size_t max_gen = shape.max_generation_size;
    const std::size_t slot_count = shape.slot_count;
    if (shape.action_count == 0 || shape.grid_column_count == 0 || max_gen == 0 || slot_count == 0 ||
        slot_count >= 0xFFFFFFFFull || shape.epicenter_rows == 0) {
        return kInvalidRuntimeConfig;
    }
    nwg_runtime *rt = new (std::nothrow) nwg_runtime();
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    rt->action_count = shape.action_count;
    rt->stride = GenomeStrideBytes(shape.action_count);
    rt->pitch = SlotPitchBytes(shape.action_count);
    rt->slot_count = slot_count;
    rt->max_generation_size = max_gen;
    rt->grid_column_count = shape.grid_column_count;
    rt->generation_byte_budget = shape.generation_byte_budget;
    rt->slab_byte_budget = shape.slab_bytes;
    rt->host_spill_budget = shape.host_spill_budget;
    rt->epicenter_rows = shape.epicenter_rows;
    rt->scratch_ctas = EvalCtaCount(0xFFFFFFFFu);
    bool ok = true;
    auto alloc = [&](auto **ptr, std::size_t bytes) {
        ok = ok && cudaMalloc(reinterpret_cast<void **>(ptr), bytes) == cudaSuccess;
        if (ok) {
            ok = cudaMemset(*ptr, 0, bytes) == cudaSuccess;
        }
    };
    alloc(&rt->slab, slot_count * rt->pitch);
    alloc(&rt->cur_slots, max_gen * sizeof(std::uint32_t));
    alloc(&rt->next_slots, max_gen * sizeof(std::uint32_t));
    alloc(&rt->cur_fitness, max_gen * sizeof(float));
    alloc(&rt->next_fitness, max_gen * sizeof(float));
    alloc(&rt->cur_eval, max_gen * sizeof(std::uint32_t));
    alloc(&rt->next_eval, max_gen * sizeof(std::uint32_t));
    alloc(&rt->cur_has, max_gen);
    alloc(&rt->next_has, max_gen);
    alloc(&rt->pairs, max_gen * 2 * sizeof(std::uint32_t));
    alloc(&rt->slot_used, slot_count);
    alloc(&rt->status, sizeof(int));
    alloc(&rt->summary, sizeof(SummaryDevice));
    alloc(&rt->shards, NWG_CATALOG_CAPACITY * sizeof(ShardRecord));
    alloc(&rt->local_words, max_gen * sizeof(std::uint32_t));
    alloc(&rt->chunk_start, (max_gen + 1) * sizeof(std::uint32_t));
    alloc(&rt->score_sum, max_gen * sizeof(std::uint32_t));
    alloc(&rt->won_sum, max_gen * sizeof(std::uint32_t));
    alloc(&rt->steps, kStepCounters * sizeof(unsigned long long));
    alloc(&rt->scratch, static_cast<std::size_t>(rt->scratch_ctas) * EvalScratchFloatsPerCta() * sizeof(float));
    ok = ok && cudaMallocHost(&rt->host_shards, NWG_CATALOG_CAPACITY * sizeof(ShardRecord)) == cudaSuccess;
    ok = ok && cudaMallocHost(&rt->host_status, sizeof(int)) == cudaSuccess;
    ok = ok && cudaMallocHost(&rt->host_summary, sizeof(SummaryDevice)) == cudaSuccess;
    ok = ok && cudaMallocHost(&rt->host_steps, kStepCounters * sizeof(unsigned long long)) == cudaSuccess;
    ok = ok && cudaEventCreate(&rt->eval_begin) == cudaSuccess && cudaEventCreate(&rt->eval_end) == cudaSuccess;
    if (!ok) {
        FreeRuntime(rt);
        return kCudaFailure;
    }
    std::memset(rt->host_summary, 0, sizeof(SummaryDevice));
    std::memset(rt->host_steps, 0, kStepCounters * sizeof(unsigned long long));
    *out = rt;
    return kOk;
}

int ReadBoundary(const nwg_runtime *rt, BoundaryState *out) {
    if (rt == nullptr || out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (!rt->prepared) {
        return kInvalidAssemblyPlan;
    }
    out->seed = rt->prepared_seed;
    out->config = rt->prepared_config;
    out->injection = rt->prepared_injection;
    out->action_count = rt->action_count;
    out->next_action_count = rt->prepared_next_action_count;
    out->stride = rt->stride;
    out->slot_count = rt->slot_count;
    out->slab_bytes = rt->slab_byte_budget;
    out->generation_byte_budget = rt->generation_byte_budget;
    out->host_spill_budget = rt->host_spill_budget;
    out->max_generation_size = rt->max_generation_size;
    out->grid_column_count = rt->grid_column_count;
    out->epicenter_rows = rt->epicenter_rows;
    out->generation_index = rt->cur_gen_index;
    out->generation_size = rt->cur_gen_size;
    out->planned_children = rt->planned_children;
    return kOk;
}

int BuildCatalogTables(const std::uint8_t *letters, std::size_t word_count, std::uint32_t **codes_out,
                       float **fixed_out, std::size_t *pad_out, std::vector<std::uint32_t> *host_codes) {
    *codes_out = nullptr;
    *fixed_out = nullptr;
    const std::size_t pad = ((word_count + 127) / 128) * 128;
    std::vector<std::uint32_t> codes(pad, 0);
    std::vector<float> fixed(static_cast<std::size_t>(kFixedDim) * pad, 0.0f);
    for (std::size_t w = 0; w < word_count; ++w) {
        codes[w] = PackWord(letters + kWordLength * w);
        int counts[kAlphabet] = {0};
        for (int p = 0; p < kWordLength; ++p) {
            ++counts[letters[kWordLength * w + p]];
        }
        // output_embedding.hpp:59-73: letter count, or -1 when the letter is absent
        for (int l = 0; l < kFixedDim; ++l) {
            fixed[static_cast<std::size_t>(l) * pad + w] = counts[l] == 0 ? -1.0f : static_cast<float>(counts[l]);
        }
    }
    if (cudaMalloc(codes_out, pad * sizeof(std::uint32_t)) != cudaSuccess ||
        cudaMalloc(fixed_out, fixed.size() * sizeof(float)) != cudaSuccess ||
        cudaMemcpy(*codes_out, codes.data(), pad * sizeof(std::uint32_t), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(*fixed_out, fixed.data(), fixed.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(*codes_out);
        cudaFree(*fixed_out);
        *codes_out = nullptr;
        *fixed_out = nullptr;
        return kCudaFailure;
    }
    *pad_out = pad;
    if (host_codes != nullptr) {
        host_codes->assign(codes.begin(), codes.begin() + static_cast<std::ptrdiff_t>(word_count));
    }
    return kOk;
}

int ReadGenerationView(const nwg_runtime *rt, GenerationView *out) {
    if (rt == nullptr || out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    out->stream = rt->stream;
    out->slab = rt->slab;
    out->pitch = rt->pitch;
    out->action_count = rt->action_count;
    out->slots = rt->cur_slots;
    out->fitness = rt->cur_fitness;
    out->has_fitness = rt->cur_has;
    out->pairs = rt->pairs;
    out->generation_index = rt->cur_gen_index;
    out->generation_size = rt->cur_gen_size;
    out->planned_children = rt->planned_children;
    out->grid_column_count = rt->grid_column_count;
    out->stride = rt->stride;
    out->slot_count = rt->slot_count;
    out->cell_offsets = rt->cell_offsets;
    out->cell_words = rt->cell_words;
    out->cell_count = rt->cell_count;
    out->evaluated = rt->last_eval_population == rt->cur_gen_size && rt->last_eval_generation == rt->cur_gen_index &&
                     rt->cur_gen_size > 0 && !rt->released_parents;
    out->status = rt->status;
    return kOk;
}

int InstallGeneration(nwg_runtime *rt, const std::uint8_t *src_slab, std::size_t src_pitch,
                      const std::vector<std::uint32_t> &src_slots, const std::vector<float> &fitness,
                      std::size_t generation_index) {
    const std::size_t n = src_slots.size();
    if (n == 0 || n != fitness.size() || n > rt->max_generation_size || src_pitch != rt->pitch ||
        n % rt->grid_column_count != 0) {
        return kInvalidGeneration;
    }
    std::vector<std::uint32_t> current(rt->cur_gen_size);
    if (cudaStreamSynchronize(rt->stream) != cudaSuccess ||
        (rt->cur_gen_size > 0 &&
         cudaMemcpy(current.data(), rt->cur_slots, current.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)) {
        return kCudaFailure;
    }
    std::vector<std::uint8_t> used(rt->slot_count, 0);
    for (const std::uint32_t s : current) {
        if (s < rt->slot_count) {
            used[s] = 1;
        }
    }
    std::vector<std::uint32_t> target;
    target.reserve(n);
    for (std::uint32_t s = 0; s < rt->slot_count && target.size() < n; ++s) {
        if (!used[s]) {
            target.push_back(s);
        }
    }
    if (target.size() < n) {
        return SetHostStatus(rt, kSlabFull);
    }
    std::uint32_t *d_src = nullptr;
    std::vector<std::uint32_t> ones(n, 1u);
    std::vector<std::uint8_t> has(n, 1u);
    bool ok = cudaMalloc(&d_src, n * 4) == cudaSuccess &&
              cudaMemcpyAsync(d_src, src_slots.data(), n * 4, cudaMemcpyHostToDevice, rt->stream) == cudaSuccess &&
              cudaMemcpyAsync(rt->next_slots, target.data(), n * 4, cudaMemcpyHostToDevice, rt->stream) ==
                  cudaSuccess &&
              cudaMemcpyAsync(rt->next_fitness, fitness.data(), n * 4, cudaMemcpyHostToDevice, rt->stream) ==
                  cudaSuccess &&
              cudaMemcpyAsync(rt->next_eval, ones.data(), n * 4, cudaMemcpyHostToDevice, rt->stream) == cudaSuccess &&
              cudaMemcpyAsync(rt->next_has, has.data(), n, cudaMemcpyHostToDevice, rt->stream) == cudaSuccess;
    if (ok) {
        CopySlotsKernel<<<256, 256, 0, rt->stream>>>(src_slab, src_pitch, d_src, rt->slab, rt->pitch, rt->next_slots,
                                                     static_cast<std::uint32_t>(n));
        ok = cudaGetLastError() == cudaSuccess;
    }
    ok = ok && cudaStreamSynchronize(rt->stream) == cudaSuccess;
    cudaFree(d_src);
    if (!ok) {
        return kCudaFailure;
    }
    rt->prepared = false;
    rt->next_gen_index = generation_index;
    rt->next_gen_size = n;
    nwg_swap_generations(rt);
    NWG_TRY(LaunchSummarize(rt->cur_fitness, rt->cur_has, rt->cur_slots, static_cast<std::uint32_t>(n), rt->summary,
                            rt->status, rt->stream));
    NWG_TRY(cudaMemcpyAsync(rt->host_summary, rt->summary, sizeof(SummaryDevice), cudaMemcpyDeviceToHost, rt->stream));
    rt->last_eval_population = n;
    rt->last_action_count = rt->action_count;
    rt->last_eval_generation = generation_index;
    rt->rates_valid = false;
    return Sync(rt);
}

int InstallBoundary(nwg_runtime *rt, const std::uint32_t *slots, const float *fitness, const std::uint32_t *eval,
                    const std::uint8_t *has, std::size_t count, std::size_t generation_index,
                    const std::uint32_t *pairs, std::size_t child_count, std::uint32_t seed,
                    const nwg_generation_assembly_config &config, const nwg_pending_injection &injection,
                    std::size_t next_action_count) {
    if (count == 0 || count > rt->max_generation_size || child_count == 0 || child_count > rt->max_generation_size) {
        return kInvalidCheckpoint;
    }
    bool released = false;
    for (std::size_t i = 0; i < count; ++i) {
        if (slots[i] == 0xFFFFFFFFu) {
            released = true;
        } else if (slots[i] >= rt->slot_count) {
            return kInvalidCheckpoint;
        }
    }
    for (std::size_t c = 0; c < 2 * child_count; ++c) {
        if (pairs[c] >= count || slots[pairs[c]] == 0xFFFFFFFFu) {
            return kInvalidCheckpoint;
        }
    }
    NWG_TRY(cudaStreamSynchronize(rt->stream));
    NWG_TRY(cudaMemcpy(rt->cur_slots, slots, count * sizeof(std::uint32_t), cudaMemcpyHostToDevice));
    NWG_TRY(cudaMemcpy(rt->cur_fitness, fitness, count * sizeof(float), cudaMemcpyHostToDevice));
    NWG_TRY(cudaMemcpy(rt->cur_eval, eval, count * sizeof(std::uint32_t), cudaMemcpyHostToDevice));
    NWG_TRY(cudaMemcpy(rt->cur_has, has, count, cudaMemcpyHostToDevice));
    NWG_TRY(cudaMemcpy(rt->pairs, pairs, child_count * 2 * sizeof(std::uint32_t), cudaMemcpyHostToDevice));
    NWG_TRY(cudaMemset(rt->status, 0, sizeof(int)));
    rt->cur_gen_index = generation_index;
    rt->cur_gen_size = count;
    rt->next_gen_index = 0;
    rt->next_gen_size = 0;
    rt->planned_children = child_count;
    rt->released_parents = released;
    rt->prepared = true;
    rt->prepared_seed = seed;
    rt->prepared_config = config;
    rt->prepared_injection = injection;
    rt->prepared_next_action_count = next_action_count;
    return kOk;
}

}  // namespace nwg

extern "C" {

int nwg_abi_version(void) { return NWG_ABI_VERSION; }

const char *nwg_status_string(int status) {
    switch (status) {
    case NWG_OK: return "ok";
    case NWG_CUDA_FAILURE: return "cuda failure";
    case NWG_INVALID_RUNTIME_CONFIG: return "invalid slab ga runtime config";
    case NWG_INVALID_SLAB: return "invalid slab state";
    case NWG_INVALID_GENERATION: return "invalid generation state";
    case NWG_INVALID_TRAINING_SHARD: return "invalid training-data shard";
    case NWG_GUESS_APPEND_FAILED: return "could not append a model-selected guess to the Wordle grid";
    case NWG_POLICY_FORWARD_FAILED: return "policy model forward pass failed";
    case NWG_ACTION_SELECTION_FAILED: return "output-embedding action selection failed";
    case NWG_POPULATION_NOT_EVALUATED:
        return "population fitness summary requested before the population was fully evaluated";
    case NWG_INVALID_ASSEMBLY_CONFIG: return "invalid next-generation assembly config";
    case NWG_PARENT_SELECTION_FAILED: return "device parent selection failed";
    case NWG_INVALID_ASSEMBLY_PLAN: return "invalid slab assembly plan";
    case NWG_INVALID_PARENT_INDEX: return "invalid parent index in slab assembly plan";
    case NWG_SLAB_FULL: return "slab is genuinely full";
    case NWG_OUTPUT_EMBEDDING_INJECTION_FAILED: return "device output-embedding injection failed";
    case NWG_SLAB_REPACK_FAILED: return "slab compaction/repacking failed";
    case NWG_TIMEOUT: return "a bounded device wait gave up";
    case NWG_UNSUPPORTED: return "request not supported by this runtime";
    case NWG_INVALID_CHECKPOINT: return "invalid runtime checkpoint";
    default: return "unknown slab ga runtime status";
    }
}

int nwg_upload_catalog(const uint8_t *letters, size_t word_count) {
    if (letters == nullptr || word_count == 0 || word_count > NWG_CATALOG_CAPACITY) {
        return kInvalidTrainingShard;
    }
    for (std::size_t i = 0; i < word_count * kWordLength; ++i) {
        if (letters[i] >= kAlphabet) {
            return kInvalidTrainingShard;
        }
    }
    std::lock_guard<std::mutex> lock(g_catalog_mutex);
    if (g_catalog.codes != nullptr) {
        cudaFree(g_catalog.codes);
        cudaFree(g_catalog.fixed_t);
        g_catalog = Catalog{};
    }
    std::vector<std::uint32_t> host_codes;
    const int st = BuildCatalogTables(letters, word_count, &g_catalog.codes, &g_catalog.fixed_t, &g_catalog.pad,
                                      &host_codes);
    if (st != kOk) {
        g_catalog = Catalog{};
        return st;
    }
    g_catalog.count = word_count;
    g_catalog.host_codes = std::move(host_codes);
    cudaGetDevice(&g_catalog.device);
    return kOk;
}

// TryCreateDeviceSlabGARuntimeBuffers (slab_runtime.cu:943-1003): slot count from the slab budget, generation
// capacity from the generation budget (floored to whole grid rows); the slab's byte size is slot_count x stride
// (genotype_slab/device_runtime.cu:1047-1050), which action-space growth re-divides at the wider stride.
int nwg_create(const nwg_runtime_config *config, nwg_runtime **runtime_out) {
    if (runtime_out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    *runtime_out = nullptr;
    if (config == nullptr || !ValidConfig(*config)) {
        return kInvalidRuntimeConfig;
    }
    const std::size_t slot_count = SlotsForBudget(config->genotype_slab_byte_budget_bytes, config->action_count);
    const std::size_t max_gen = FloorRows(
        SlotsForBudget(config->generation_byte_budget_bytes, config->action_count, config->population_size_ceiling),
        config->grid_column_count);
    if (slot_count < max_gen || max_gen == 0 || slot_count >= 0xFFFFFFFFull) {
        return kInvalidRuntimeConfig;
    }
    const std::size_t stride = GenomeStrideBytes(config->action_count);
    RuntimeShape shape{};
    shape.action_count = config->action_count;
    shape.slot_count = slot_count;
    shape.slab_bytes = slot_count * stride;
    shape.max_generation_size = max_gen;
    shape.grid_column_count = config->grid_column_count;
    shape.generation_byte_budget = max_gen * stride;
    shape.host_spill_budget = config->host_spillover_byte_budget_bytes;
    shape.epicenter_rows = max_gen / config->grid_column_count;
    return CreateShapedRuntime(shape, runtime_out);
}

void nwg_destroy(nwg_runtime *runtime) {
    if (runtime != nullptr) {
        cudaStreamSynchronize(runtime->stream);
    }
    FreeRuntime(runtime);
}

int nwg_set_stream(nwg_runtime *runtime, void *cuda_stream) {
    if (runtime == nullptr) {
        return kInvalidRuntimeConfig;
    }
    runtime->stream = static_cast<cudaStream_t>(cuda_stream);
    return kOk;
}

int nwg_get_info(const nwg_runtime *rt, nwg_runtime_info *info) {
    if (rt == nullptr || info == nullptr) {
        return kInvalidRuntimeConfig;
    }
    info->action_count = rt->action_count;
    info->slot_stride_bytes = rt->stride;
    info->slot_pitch_bytes = rt->pitch;
    info->slot_count = rt->slot_count;
    info->max_generation_size = rt->max_generation_size;
    info->grid_column_count = rt->grid_column_count;
    info->current_generation_index = rt->cur_gen_index;
    info->current_generation_size = rt->cur_gen_size;
    info->next_generation_index = rt->next_gen_index;
    info->next_generation_size = rt->next_gen_size;
    info->planned_child_count = rt->planned_children;
    info->slab_bytes = rt->slab_byte_budget;
    info->generation_byte_budget_bytes = rt->generation_byte_budget;
    info->host_spillover_byte_budget_bytes = rt->host_spill_budget;
    info->epicenter_row_count = rt->epicenter_rows;
    info->prepared = rt->prepared ? 1u : 0u;
    return kOk;
}

int nwg_set_evaluation_form(nwg_runtime *rt, int form) {
    if (rt == nullptr || form < NWG_FORM_FP32 || form > NWG_FORM_TC_TRUNK_FP16) {
        return kInvalidRuntimeConfig;
    }
    if ((form == NWG_FORM_TC_TRUNK_BF16 || form == NWG_FORM_TC_TRUNK_FP16) && rt->trunk_tables == nullptr) {
        if (cudaMalloc(&rt->trunk_tables, rt->max_generation_size * TrunkTablePitch()) != cudaSuccess) {
            rt->trunk_tables = nullptr;
            return kCudaFailure;
        }
    }
    if (form != NWG_FORM_FP32 && rt->tc_tables == nullptr) {
        const std::size_t bytes = rt->max_generation_size * TcTablePitch(static_cast<std::uint32_t>(rt->action_count));
        if (cudaMalloc(&rt->tc_tables, bytes) != cudaSuccess) {
            rt->tc_tables = nullptr;
            return kCudaFailure;
        }
        rt->tc_tables_bytes = bytes;
    }
    rt->form = form;
    return kOk;
}

int nwg_set_wait_limit(nwg_runtime *rt, uint32_t polls) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    rt->wait_limit = polls;
    return kOk;
}

int nwg_set_margin_guard(nwg_runtime *rt, float tau) {
    if (rt == nullptr || !(tau >= 0.0f) || !(tau <= 3.0e38f)) {
        return kInvalidRuntimeConfig;
    }
    rt->margin_tau = tau;
    return kOk;
}

int nwg_bootstrap(nwg_runtime *rt, size_t generation_size, uint32_t generation_seed, size_t generation_index) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    rt->prepared = false;
    if (generation_size == 0 || generation_size > rt->max_generation_size ||
        generation_size % rt->grid_column_count != 0) {
        return kInvalidGeneration;
    }
    // a band bootstraps its own rows of the whole grid's generation 0 (their organisms' random streams)
    if (rt->band && generation_size != rt->max_generation_size) {
        return kInvalidGeneration;
    }
    const std::uint32_t organism_first =
        rt->band ? static_cast<std::uint32_t>(rt->band_row_first * rt->grid_column_count) : 0u;
    const std::uint32_t stream_population =
        rt->band ? static_cast<std::uint32_t>(rt->band_global_rows * rt->grid_column_count) : 0u;
    std::vector<std::uint32_t> slots(generation_size);
    for (std::size_t i = 0; i < generation_size; ++i) {
        slots[i] = static_cast<std::uint32_t>(i);
    }
    NWG_TRY(cudaMemcpyAsync(rt->cur_slots, slots.data(), generation_size * sizeof(std::uint32_t),
                            cudaMemcpyHostToDevice, rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->cur_fitness, 0, rt->max_generation_size * sizeof(float), rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->cur_eval, 0, rt->max_generation_size * sizeof(std::uint32_t), rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->cur_has, 0, rt->max_generation_size, rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->status, 0, sizeof(int), rt->stream));
    NWG_TRY(cudaMemsetAsync(rt->summary, 0, sizeof(SummaryDevice), rt->stream));
    NWG_TRY(LaunchBootstrap(rt->slab, rt->pitch, rt->cur_slots, static_cast<std::uint32_t>(generation_size),
                            generation_index, generation_seed, static_cast<std::uint32_t>(rt->action_count),
                            rt->stream, organism_first, stream_population));
    const int st = Sync(rt);
    if (st != kOk) {
        rt->cur_gen_size = 0;
        return st;
    }
    rt->cur_gen_index = generation_index;
    rt->cur_gen_size = generation_size;
    rt->band_halo_ready = false;
    rt->released_parents = false;
    rt->next_gen_index = 0;
    rt->next_gen_size = 0;
    rt->planned_children = 0;
    return kOk;
}

int nwg_set_cell_words(nwg_runtime *rt, const uint32_t *offsets, const uint32_t *words, size_t cell_count) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (cell_count == 0) {
        rt->cell_count = 0;
        return kOk;
    }
    if (offsets == nullptr || words == nullptr || cell_count > rt->max_generation_size || offsets[0] != 0) {
        return kInvalidTrainingShard;
    }
    for (std::size_t c = 0; c < cell_count; ++c) {
        if (offsets[c + 1] < offsets[c] || offsets[c + 1] == offsets[c]) {
            return kInvalidTrainingShard;
        }
    }
    const std::size_t total = offsets[cell_count];
    if (rt->cell_offsets == nullptr || rt->cell_word_capacity < total) {
        if (rt->cell_words != nullptr) {
            cudaFree(rt->cell_words);
            rt->cell_words = nullptr;
        }
        if (rt->cell_offsets == nullptr) {
            NWG_TRY(cudaMalloc(&rt->cell_offsets, (rt->max_generation_size + 1) * sizeof(std::uint32_t)));
        }
        NWG_TRY(cudaMalloc(&rt->cell_words, total * sizeof(std::uint32_t)));
        rt->cell_word_capacity = total;
    }
    NWG_TRY(cudaMemcpyAsync(rt->cell_offsets, offsets, (cell_count + 1) * sizeof(std::uint32_t),
                            cudaMemcpyHostToDevice, rt->stream));
    NWG_TRY(cudaMemcpyAsync(rt->cell_words, words, total * sizeof(std::uint32_t), cudaMemcpyHostToDevice, rt->stream));
    NWG_TRY(cudaStreamSynchronize(rt->stream));
    rt->cell_count = cell_count;
    return kOk;
}

int nwg_evaluate(nwg_runtime *rt, const nwg_runtime_word_counts *counts, const nwg_shard_release_history *history) {
    const int st = EvaluateImpl(rt, counts, history, 0, nullptr, nullptr, nullptr, nullptr);
    if (st != kOk) {
        return st;
    }
    return Sync(rt);
}

int nwg_evaluate_traced(nwg_runtime *rt, const nwg_runtime_word_counts *counts,
                        const nwg_shard_release_history *history, size_t trace_episodes, void *choices, void *turns,
                        void *scores, void *policy) {
    const int st = EvaluateImpl(rt, counts, history, trace_episodes, choices, turns, scores, policy);
    if (st != kOk) {
        return st;
    }
    return Sync(rt);
}

int nwg_read_summary(const nwg_runtime *rt, nwg_fitness_summary *summary) {
    if (rt == nullptr || summary == nullptr) {
        return kInvalidRuntimeConfig;
    }
    summary->best_fitness = rt->host_summary->best_fitness;
    summary->average_fitness = rt->host_summary->average_fitness;
    summary->best_index = rt->host_summary->best_index;
    summary->best_slot_index = rt->host_summary->best_slot_index;
    summary->generation_index = rt->last_eval_generation;
    summary->action_count = rt->last_action_count;
    summary->population_size = rt->last_eval_population;
    return kOk;
}

int nwg_read_evaluation_stats(const nwg_runtime *rt, nwg_evaluation_stats *stats) {
    if (rt == nullptr || stats == nullptr) {
        return kInvalidRuntimeConfig;
    }
    stats->game_steps = rt->host_steps[0];
    stats->encoded_turns = rt->host_steps[1];
    stats->episodes = rt->host_steps[2];
    stats->rescored_chunks = rt->host_steps[3] + rt->host_steps[7];
    stats->full_rescores = rt->host_steps[4] + rt->host_steps[8];
    stats->candidate_chunks = rt->host_steps[5];
    stats->fallback_steps = rt->host_steps[6];
    stats->fitness_mean_fp64 = rt->host_summary->mean_fp64;
    stats->fitness_variance_fp64 = rt->host_summary->variance_fp64;
    float ms = 0.0f;
    stats->eval_kernel_ms = cudaEventElapsedTime(&ms, rt->eval_begin, rt->eval_end) == cudaSuccess ? ms : -1.0;
    return kOk;
}

int nwg_read_score_table(const nwg_runtime *rt, size_t individual, void *host_out, size_t capacity,
                         size_t *bytes_out) {
    if (rt == nullptr || rt->tc_tables == nullptr || rt->last_table_pitch == 0 ||
        individual >= rt->last_eval_population) {
        return kPopulationNotEvaluated;
    }
    if (bytes_out != nullptr) {
        *bytes_out = rt->last_table_pitch;
    }
    if (host_out == nullptr) {
        return kOk;
    }
    if (capacity < rt->last_table_pitch) {
        return kInvalidGeneration;
    }
    if (cudaStreamSynchronize(rt->stream) != cudaSuccess ||
        cudaMemcpy(host_out, rt->tc_tables + individual * rt->last_table_pitch, rt->last_table_pitch,
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
        return kCudaFailure;
    }
    return kOk;
}

int nwg_read_solve_rates(const nwg_runtime *rt, float *rates, size_t capacity, size_t *count_out,
                         double *mean_out) {
    if (rt == nullptr || rt->last_eval_population == 0 || rt->last_eval_population != rt->cur_gen_size ||
        !rt->rates_valid || rt->last_eval_generation != rt->cur_gen_index) {
        return kPopulationNotEvaluated;
    }
    const std::size_t n = rt->cur_gen_size;
    if (rates != nullptr && capacity < n) {
        return kInvalidGeneration;
    }
    std::vector<std::uint32_t> won(n), words(n);
    if (cudaStreamSynchronize(rt->stream) != cudaSuccess ||
        cudaMemcpy(won.data(), rt->won_sum, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(words.data(), rt->local_words, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        return kCudaFailure;
    }
    double total = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        const double games = 3.0 * static_cast<double>(words[i]);  // three episodes per local word
        const double rate = games > 0.0 ? static_cast<double>(won[i]) / games : 0.0;
        if (rates != nullptr) {
            rates[i] = static_cast<float>(rate);
        }
        total += rate;
    }
    if (count_out != nullptr) {
        *count_out = n;
    }
    if (mean_out != nullptr) {
        *mean_out = total / static_cast<double>(n);
    }
    return kOk;
}

int nwg_prepare_generation(nwg_runtime *rt, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                           const nwg_generation_assembly_config *config, const nwg_pending_injection *pending,
                           nwg_post_fitness_fn post_fitness, void *post_fitness_user,
                           nwg_shard_release_fn shard_release, void *shard_release_user,
                           const nwg_shard_release_history *history) {
    if (rt == nullptr || counts == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (rt->band) {
        return kUnsupported;  // a band selects over the whole grid's fitness: nwg_band_prepare
    }
    rt->prepared = false;
    nwg_generation_assembly_config cfg{};
    cfg.parent_selection.cellular_breeding_radius = 2;  // selection.hpp:13-18, spatial/grid.hpp:11
    cfg.parent_selection.rank_exponent = 0.5f;
    cfg.breeding = {0.02f, 0.01f, 0.005f};              // breeding.hpp:6-14
    cfg.mutation = {0.0001f, 0.02f, 0.0f};              // mutation.hpp:7-15
    if (config != nullptr) {
        cfg = *config;
    }
    nwg_pending_injection injection{};
    if (pending != nullptr) {
        injection = *pending;
    }
    // generation_assembly.hpp:15-19
    const auto in01 = [](float v) { return v >= 0.0f && v <= 1.0f; };
    const bool valid = cfg.parent_selection.cellular_breeding_radius > 0 && cfg.parent_selection.rank_exponent >= 0.0f &&
                       cfg.parent_selection.rank_exponent <= 4.0f && in01(cfg.breeding.crossover_temperature_level1) &&
                       in01(cfg.breeding.crossover_temperature_level2) &&
                       in01(cfg.breeding.crossover_temperature_level3) && in01(cfg.mutation.mutation_probability) &&
                       cfg.mutation.mutation_sigma >= 0.0f &&
                       in01(cfg.mutation.output_tail_row_scale_mutation_probability);
    if (!valid) {
        return SetHostStatus(rt, kInvalidAssemblyConfig);
    }
    int st = EvaluateImpl(rt, counts, history, 0, nullptr, nullptr, nullptr, nullptr);
    if (st != kOk) {
        return st;
    }
    if (shard_release != nullptr || post_fitness != nullptr) {
        st = Sync(rt);
        if (st != kOk) {
            return st;
        }
    }
    if (shard_release != nullptr && !shard_release(rt, counts, &injection, shard_release_user)) {
        return SetHostStatus(rt, kInvalidAssemblyConfig);
    }
    // slab_runtime.cu:678-683, :919-939: the next width, then the next population from the generation byte
    // budget at that width
    std::size_t next_action_count = rt->action_count;
    std::vector<HintGroup> hints;
    if (injection.enabled) {
        if (injection.injection_count == 0 || injection.first_catalog_word_index != rt->action_count) {
            return SetHostStatus(rt, kInvalidAssemblyConfig);
        }
        next_action_count = rt->action_count + injection.injection_count;
        // injection_ops.cuh:31-37 and output_embedding_injection.hpp:123-131: the new words must exist in the
        // catalog and each must have a hint-grid group
        if (next_action_count > g_catalog.count) {
            return SetHostStatus(rt, kOutputEmbeddingInjectionFailed);
        }
        hints.resize(injection.injection_count);
        for (std::size_t i = 0; i < injection.injection_count; ++i) {
            if (!BuildHintGroup(g_catalog.host_codes[rt->action_count + i], hints[i])) {
                return SetHostStatus(rt, kOutputEmbeddingInjectionFailed);
            }
        }
    }
    std::size_t next_size = FloorRows(SlotsForBudget(rt->generation_byte_budget, next_action_count,
                                                     rt->max_generation_size),
                                      rt->grid_column_count);
    next_size = std::min(next_size, rt->cur_gen_size);
    if (next_size == 0) {
        return SetHostStatus(rt, kInvalidAssemblyConfig);
    }
    SelectParams sp{};
    sp.fitness = rt->cur_fitness;
    sp.has_fitness = rt->cur_has;
    sp.rows = static_cast<std::uint32_t>(rt->cur_gen_size / rt->grid_column_count);
    sp.cols = static_cast<std::uint32_t>(rt->grid_column_count);
    sp.child_count = static_cast<std::uint32_t>(next_size);
    sp.generation_index = rt->cur_gen_index;
    sp.radius = cfg.parent_selection.cellular_breeding_radius;
    sp.rank_exponent = cfg.parent_selection.rank_exponent;
    sp.planning_seed = generation_seed ^ 0xA341316Cu;  // slab_runtime.cu:1443
    sp.pairs = rt->pairs;
    sp.status = rt->status;
    NWG_TRY(LaunchSelect(sp, rt->stream));
    rt->planned_children = next_size;
    if (post_fitness != nullptr) {
        st = Sync(rt);
        if (st != kOk) {
            return st;
        }
        if (!post_fitness(rt, counts, post_fitness_user)) {
            return SetHostStatus(rt, kInvalidAssemblyConfig);
        }
    }
    rt->prepared = true;
    rt->prepared_seed = generation_seed;
    rt->prepared_config = cfg;
    rt->prepared_injection = injection;
    rt->prepared_next_action_count = next_action_count;
    return kOk;
}

namespace {

// The device work of assembling planned children without injection: slot plan, breeding, cleared next arrays.
// In band mode the parents are named by their index in the whole grid and found through the band's parent table
// (the band's own slots and its halo slots), the children's streams are their whole-grid indices, and the halo
// slots are never given to a child.
cudaError_t AssembleLaunch(nwg_runtime *rt, std::uint32_t generation_seed, const nwg_generation_assembly_config &cfg,
                           std::size_t next_size) {
    const std::uint32_t *parent_slots = rt->band ? rt->band_parent_table : rt->cur_slots;
    const std::size_t parent_count =
        rt->band ? rt->band_global_rows * rt->grid_column_count : rt->cur_gen_size;
    const std::size_t assignable = rt->slot_count - rt->band_reserved_slots;
    PlanChildSlotsKernel<<<1, 1024, 0, rt->stream>>>(rt->pairs, static_cast<std::uint32_t>(next_size), parent_slots,
                                                     static_cast<std::uint32_t>(parent_count), rt->slot_used,
                                                     static_cast<std::uint32_t>(assignable), rt->next_slots,
                                                     rt->status, static_cast<std::uint32_t>(rt->slot_count));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return e;
    }
    BreedParams bp{};
    bp.parent_slab = rt->slab;
    bp.parent_pitch = rt->pitch;
    bp.parent_slots = parent_slots;
    bp.child_slab = rt->slab;
    bp.child_pitch = rt->pitch;
    bp.child_slots = rt->next_slots;
    bp.child_first = rt->band ? static_cast<std::uint32_t>(rt->band_row_first * rt->grid_column_count) : 0u;
    bp.pairs = rt->pairs;
    bp.child_count = static_cast<std::uint32_t>(next_size);
    bp.action_count = static_cast<std::uint32_t>(rt->action_count);
    bp.generation_seed = generation_seed;
    bp.generation_index = rt->cur_gen_index;
    bp.crossover_l1 = cfg.breeding.crossover_temperature_level1;
    bp.crossover_l2 = cfg.breeding.crossover_temperature_level2;
    bp.crossover_l3 = cfg.breeding.crossover_temperature_level3;
    bp.mutation_probability = cfg.mutation.mutation_probability;
    bp.mutation_sigma = cfg.mutation.mutation_sigma;
    bp.row_scale_probability = cfg.mutation.output_tail_row_scale_mutation_probability;
    bp.status = rt->status;
    if (rt->breed_begin != nullptr &&
        (e = RecordEvent(rt->breed_begin, rt->stream)) != cudaSuccess) {
        return e;
    }
    if ((e = LaunchBreed(bp, rt->stream, rt->breed_warps)) != cudaSuccess) {
        return e;
    }
    if (rt->breed_end != nullptr &&
        (e = RecordEvent(rt->breed_end, rt->stream)) != cudaSuccess) {
        return e;
    }
    if ((e = cudaMemsetAsync(rt->next_fitness, 0, rt->max_generation_size * sizeof(float), rt->stream)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(rt->next_eval, 0, rt->max_generation_size * sizeof(std::uint32_t), rt->stream)) !=
            cudaSuccess) {
        return e;
    }
    return cudaMemsetAsync(rt->next_has, 0, rt->max_generation_size, rt->stream);
}

// Waits for the assembly, then makes the children the current generation.
int AssembleFinish(nwg_runtime *rt, std::size_t next_size) {
    const int st = Sync(rt);
    if (st != kOk) {
        return st;
    }
    rt->next_gen_index = rt->cur_gen_index + 1;
    rt->next_gen_size = next_size;
    return nwg_swap_generations(rt);
}

}  // namespace

// TryAssemblePreparedGenerationOnDevice (slab_runtime.cu:1511-1680): breed (and inject) the planned children,
// then swap generations.
int nwg_assemble_prepared(nwg_runtime *rt) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (!rt->prepared) {
        return SetHostStatus(rt, kInvalidAssemblyPlan);
    }
    if (rt->band && !rt->band_halo_ready) {
        return SetHostStatus(rt, kInvalidAssemblyPlan);  // the halo rows of this generation are not installed
    }
    rt->prepared = false;
    const std::uint32_t generation_seed = rt->prepared_seed;
    const nwg_generation_assembly_config cfg = rt->prepared_config;
    const nwg_pending_injection injection = rt->prepared_injection;
    const std::size_t next_size = rt->planned_children;
    if (injection.enabled) {
        std::vector<HintGroup> hints(injection.injection_count);
        for (std::size_t i = 0; i < injection.injection_count; ++i) {
            if (injection.first_catalog_word_index + i >= g_catalog.host_codes.size() ||
                !BuildHintGroup(g_catalog.host_codes[injection.first_catalog_word_index + i], hints[i])) {
                return SetHostStatus(rt, kOutputEmbeddingInjectionFailed);
            }
        }
        return AdvanceWithInjection(rt, generation_seed, cfg, injection, hints, rt->prepared_next_action_count,
                                    next_size);
    }
    NWG_TRY(AssembleLaunch(rt, generation_seed, cfg, next_size));
    return AssembleFinish(rt, next_size);
}

int nwg_advance(nwg_runtime *rt, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                const nwg_generation_assembly_config *config, const nwg_pending_injection *pending,
                nwg_post_fitness_fn post_fitness, void *post_fitness_user, nwg_shard_release_fn shard_release,
                void *shard_release_user, const nwg_shard_release_history *history) {
    const int st = nwg_prepare_generation(rt, generation_seed, counts, config, pending, post_fitness, post_fitness_user,
                                          shard_release, shard_release_user, history);
    return st != kOk ? st : nwg_assemble_prepared(rt);
}

namespace {

constexpr int kBreedWarpChoices[3] = {4, 8, 16};

std::uint64_t TuningKey(std::size_t width, int form) { return (static_cast<std::uint64_t>(width) << 8) | (form & 0xFF); }

}  // namespace

int nwg_advance_graphed(nwg_runtime *rt, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                        const nwg_generation_assembly_config *config, const nwg_pending_injection *pending) {
    if (rt == nullptr || counts == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (pending != nullptr && pending->enabled) {
        return nwg_advance(rt, generation_seed, counts, config, pending, nullptr, nullptr, nullptr, nullptr, nullptr);
    }
    if (rt->band) {
        return kUnsupported;
    }
    if (rt->breed_begin == nullptr) {
        NWG_TRY(cudaEventCreate(&rt->breed_begin));
        NWG_TRY(cudaEventCreate(&rt->breed_end));
    }
    // stream capture needs a stream other than the legacy default stream
    const cudaStream_t caller = rt->stream;
    if (caller == nullptr) {
        if (rt->own_stream == nullptr) {
            NWG_TRY(cudaStreamCreateWithFlags(&rt->own_stream, cudaStreamNonBlocking));
        }
        NWG_TRY(cudaStreamSynchronize(nullptr));
        rt->stream = rt->own_stream;
    }
    // launch shapes of this generation
    nwg_launch_tuning &tune = rt->tuning[TuningKey(rt->action_count, rt->form)];
    const bool trial = rt->autotune && !tune.decided;
    const bool try_single = !rt->single_cta_lost[rt->form];
    if (trial) {
        rt->eval_ctas = tune.trials % 2 == 1 && try_single ? std::max(1, rt->scratch_ctas / 2) : rt->scratch_ctas;
        rt->breed_warps = kBreedWarpChoices[tune.trials % 3];
    } else if (rt->autotune) {
        rt->eval_ctas = tune.eval_ctas;
        rt->breed_warps = tune.breed_warps;
    } else {
        rt->eval_ctas = 0;
        rt->breed_warps = 4;
    }
    auto restore = [&](int status) {
        rt->stream = caller;
        rt->eval_ctas = 0;
        rt->breed_warps = 4;
        return status;
    };
    // capture: prepare (no callbacks, so it never waits on the device) and the assembly's device work; the FP32
    // forms' exact trunk tables are allocated first, since nothing is allocated while capturing
    if (rt->form == NWG_FORM_FP32 || rt->form == NWG_FORM_TC_BF16 || rt->form == NWG_FORM_TC_FP16 ||
        rt->action_count <= 128) {
        EnsureExactTrunkTables(rt);
    }
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(rt->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        return restore(kCudaFailure);
    }
    int st = nwg_prepare_generation(rt, generation_seed, counts, config, nullptr, nullptr, nullptr, nullptr, nullptr,
                                    nullptr);
    const std::uint32_t seed = rt->prepared_seed;
    const nwg_generation_assembly_config cfg = rt->prepared_config;
    const std::size_t next_size = rt->planned_children;
    if (st == kOk) {
        rt->prepared = false;
        if (AssembleLaunch(rt, seed, cfg, next_size) != cudaSuccess) {
            st = kCudaFailure;
        }
    }
    const cudaError_t end = cudaStreamEndCapture(rt->stream, &graph);
    if (st != kOk || end != cudaSuccess || graph == nullptr) {
        if (graph != nullptr) {
            cudaGraphDestroy(graph);
        }
        cudaGetLastError();
        rt->prepared = false;
        // a rejected call leaves the same status behind as nwg_advance does
        return restore(st != kOk ? SetHostStatus(rt, st) : kCudaFailure);
    }
    cudaGraphExecUpdateResultInfo info{};
    if (rt->graph_exec != nullptr && cudaGraphExecUpdate(rt->graph_exec, graph, &info) == cudaSuccess) {
        ++rt->graph.updates;
    } else {
        cudaGetLastError();  // a failed update is not an error of the run: instantiate afresh
        if (rt->graph_exec != nullptr) {
            cudaGraphExecDestroy(rt->graph_exec);
            rt->graph_exec = nullptr;
        }
        if (cudaGraphInstantiate(&rt->graph_exec, graph, 0) != cudaSuccess) {
            cudaGraphDestroy(graph);
            rt->graph_exec = nullptr;
            return restore(kCudaFailure);
        }
        ++rt->graph.instantiations;
    }
    cudaGraphDestroy(graph);
    if (cudaGraphLaunch(rt->graph_exec, rt->stream) != cudaSuccess) {
        return restore(kCudaFailure);
    }
    ++rt->graph.launches;
    st = AssembleFinish(rt, next_size);
    if (st == kOk && trial) {
        float eval_ms = 0.0f, breed_ms = 0.0f;
        if (cudaEventElapsedTime(&eval_ms, rt->eval_begin, rt->eval_end) == cudaSuccess &&
            cudaEventElapsedTime(&breed_ms, rt->breed_begin, rt->breed_end) == cudaSuccess) {
            // running mean per evaluation shape (two CTAs per SM on trials 0 and 2, and on trial 1 too once one CTA
            // per SM has lost by a wide margin)
            const int e = tune.trials % 2 == 1 && try_single ? 1 : 0;
            const int n_before = e == 1 ? 0 : (try_single ? tune.trials / 2 : tune.trials);
            tune.eval_ms[e] += (eval_ms - tune.eval_ms[e]) / static_cast<float>(n_before + 1);
            tune.breed_ms[tune.trials % 3] = breed_ms;
            ++tune.trials;
            if (tune.trials == 3) {
                tune.decided = 1;
                const bool single = tune.eval_ms[1] > 0.0f && tune.eval_ms[1] < tune.eval_ms[0];
                tune.eval_ctas = single ? std::max(1, rt->scratch_ctas / 2) : rt->scratch_ctas;
                if (tune.eval_ms[1] > 1.2f * tune.eval_ms[0]) {
                    rt->single_cta_lost[rt->form] = true;
                }
                int best = 0;
                for (int b = 1; b < 3; ++b) {
                    best = tune.breed_ms[b] < tune.breed_ms[best] ? b : best;
                }
                tune.breed_warps = kBreedWarpChoices[best];
            }
        }
        cudaGetLastError();
    }
    return restore(st);
}

int nwg_hint_groups_available(const uint8_t *letters, size_t count, uint8_t *available) {
    if (count > 0 && (letters == nullptr || available == nullptr)) {
        return kInvalidRuntimeConfig;
    }
    for (std::size_t i = 0; i < count; ++i) {
        for (int k = 0; k < kWordLength; ++k) {
            if (letters[i * kWordLength + k] >= kAlphabet) {
                return kInvalidRuntimeConfig;
            }
        }
        HintGroup g;
        available[i] = BuildHintGroup(PackWord(letters + i * kWordLength), g) ? 1 : 0;
    }
    return kOk;
}

int nwg_read_graph_info(const nwg_runtime *rt, nwg_graph_info *info) {
    if (rt == nullptr || info == nullptr) {
        return kInvalidRuntimeConfig;
    }
    *info = rt->graph;
    return kOk;
}

int nwg_read_launch_tuning(const nwg_runtime *rt, size_t action_width, int form, nwg_launch_tuning *out) {
    if (rt == nullptr || out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    const auto it = rt->tuning.find(TuningKey(action_width, form));
    *out = it == rt->tuning.end() ? nwg_launch_tuning{} : it->second;
    return kOk;
}

int nwg_set_launch_tuning(nwg_runtime *rt, int enabled) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    rt->autotune = enabled != 0;
    return kOk;
}

int nwg_swap_generations(nwg_runtime *rt) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    std::swap(rt->cur_slots, rt->next_slots);
    std::swap(rt->cur_fitness, rt->next_fitness);
    std::swap(rt->cur_eval, rt->next_eval);
    std::swap(rt->cur_has, rt->next_has);
    std::swap(rt->cur_gen_index, rt->next_gen_index);
    std::swap(rt->cur_gen_size, rt->next_gen_size);
    rt->prepared = false;
    rt->released_parents = false;
    rt->band_halo_ready = false;
    return kOk;
}

int nwg_read_status(const nwg_runtime *rt, int *status) {
    if (rt == nullptr || status == nullptr) {
        return kInvalidRuntimeConfig;
    }
    int value = 0;
    if (cudaMemcpy(&value, rt->status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
        return kCudaFailure;
    }
    *status = value;
    return kOk;
}

namespace {

int DownloadGeneration(const nwg_runtime *rt, bool current, uint32_t *slot_indices, float *fitness,
                       uint32_t *evaluation_counts, uint8_t *has_fitness, size_t capacity, size_t *count_out,
                       size_t *generation_index_out) {
    const std::size_t n = current ? rt->cur_gen_size : rt->next_gen_size;
    if (n == 0 || capacity < n) {
        return kInvalidGeneration;
    }
    const std::uint32_t *slots = current ? rt->cur_slots : rt->next_slots;
    const float *fit = current ? rt->cur_fitness : rt->next_fitness;
    const std::uint32_t *evals = current ? rt->cur_eval : rt->next_eval;
    const std::uint8_t *has = current ? rt->cur_has : rt->next_has;
    cudaStreamSynchronize(rt->stream);
    if ((slot_indices && cudaMemcpy(slot_indices, slots, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (fitness && cudaMemcpy(fitness, fit, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (evaluation_counts && cudaMemcpy(evaluation_counts, evals, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (has_fitness && cudaMemcpy(has_fitness, has, n, cudaMemcpyDeviceToHost) != cudaSuccess)) {
        return kCudaFailure;
    }
    if (count_out) {
        *count_out = n;
    }
    if (generation_index_out) {
        *generation_index_out = current ? rt->cur_gen_index : rt->next_gen_index;
    }
    return kOk;
}

}  // namespace

int nwg_download_current_generation(const nwg_runtime *rt, uint32_t *slot_indices, float *fitness,
                                    uint32_t *evaluation_counts, uint8_t *has_fitness, size_t capacity,
                                    size_t *count_out, size_t *generation_index_out) {
    if (rt == nullptr) {
        return kInvalidGeneration;
    }
    return DownloadGeneration(rt, true, slot_indices, fitness, evaluation_counts, has_fitness, capacity, count_out,
                              generation_index_out);
}

int nwg_download_next_generation(const nwg_runtime *rt, uint32_t *slot_indices, float *fitness,
                                 uint32_t *evaluation_counts, uint8_t *has_fitness, size_t capacity,
                                 size_t *count_out, size_t *generation_index_out) {
    if (rt == nullptr) {
        return kInvalidGeneration;
    }
    return DownloadGeneration(rt, false, slot_indices, fitness, evaluation_counts, has_fitness, capacity, count_out,
                              generation_index_out);
}

int nwg_download_slot(const nwg_runtime *rt, uint32_t slot_index, uint8_t *bytes, size_t capacity,
                      size_t *byte_count_out) {
    if (rt == nullptr || bytes == nullptr || slot_index >= rt->slot_count || capacity < rt->stride) {
        return kInvalidSlab;
    }
    cudaStreamSynchronize(rt->stream);
    if (cudaMemcpy(bytes, rt->slab + static_cast<std::size_t>(slot_index) * rt->pitch, rt->stride,
                   cudaMemcpyDeviceToHost) != cudaSuccess) {
        return kCudaFailure;
    }
    if (byte_count_out) {
        *byte_count_out = rt->stride;
    }
    return kOk;
}

int nwg_upload_slot(nwg_runtime *rt, uint32_t slot_index, const uint8_t *bytes, size_t byte_count) {
    if (rt == nullptr || bytes == nullptr || slot_index >= rt->slot_count || byte_count != rt->stride) {
        return kInvalidSlab;
    }
    cudaStreamSynchronize(rt->stream);
    if (cudaMemcpy(rt->slab + static_cast<std::size_t>(slot_index) * rt->pitch, bytes, byte_count,
                   cudaMemcpyHostToDevice) != cudaSuccess) {
        return kCudaFailure;
    }
    return kOk;
}

int nwg_upload_current_generation(nwg_runtime *rt, const uint32_t *slot_indices, size_t count,
                                  size_t generation_index) {
    if (rt == nullptr || slot_indices == nullptr || count == 0 || count > rt->max_generation_size ||
        count % rt->grid_column_count != 0) {
        return kInvalidGeneration;
    }
    for (std::size_t i = 0; i < count; ++i) {
        if (slot_indices[i] >= rt->slot_count) {
            return kInvalidGeneration;
        }
    }
    cudaStreamSynchronize(rt->stream);
    if (cudaMemcpy(rt->cur_slots, slot_indices, count * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(rt->cur_fitness, 0, rt->max_generation_size * 4) != cudaSuccess ||
        cudaMemset(rt->cur_eval, 0, rt->max_generation_size * 4) != cudaSuccess ||
        cudaMemset(rt->cur_has, 0, rt->max_generation_size) != cudaSuccess) {
        return kCudaFailure;
    }
    rt->cur_gen_size = count;
    rt->cur_gen_index = generation_index;
    rt->prepared = false;
    rt->released_parents = false;
    rt->band_halo_ready = false;
    return kOk;
}

int nwg_download_assembly_plan(const nwg_runtime *rt, uint32_t *pairs, size_t capacity, size_t *count_out) {
    if (rt == nullptr || pairs == nullptr || capacity < rt->planned_children) {
        return kInvalidAssemblyPlan;
    }
    cudaStreamSynchronize(rt->stream);
    if (cudaMemcpy(pairs, rt->pairs, rt->planned_children * 2 * sizeof(std::uint32_t), cudaMemcpyDeviceToHost) !=
        cudaSuccess) {
        return kCudaFailure;
    }
    if (count_out) {
        *count_out = rt->planned_children;
    }
    return kOk;
}

int nwg_device_slab(const nwg_runtime *rt, void **slab_out, size_t *pitch_out) {
    if (rt == nullptr || slab_out == nullptr || pitch_out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    *slab_out = rt->slab;
    *pitch_out = rt->pitch;
    return kOk;
}

int nwg_set_band(nwg_runtime *rt, size_t global_rows, size_t band_row_first, size_t halo_rows) {
    if (rt == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (global_rows == 0) {  // back to a whole population
        rt->band = false;
        rt->band_global_rows = rt->band_row_first = rt->band_halo_rows = rt->band_reserved_slots = 0;
        rt->band_halo_ready = false;
        return kOk;
    }
    const std::size_t cols = rt->grid_column_count;
    const std::size_t band_rows = rt->max_generation_size / cols;
    const std::size_t reserved = 2 * halo_rows * cols;
    // the halo rows must be other rows than the band's (and than each other's), and the slab must hold the band's
    // parents, its children and the halo
    if (band_rows == 0 || halo_rows == 0 || band_row_first >= global_rows || global_rows < band_rows + 2 * halo_rows ||
        global_rows * cols > 0xFFFFFFFFull || rt->slot_count < 2 * rt->max_generation_size + reserved) {
        return kInvalidRuntimeConfig;
    }
    if (rt->band_parent_table == nullptr || rt->band_global_rows * cols < global_rows * cols) {
        if (rt->band_parent_table != nullptr) {
            cudaFree(rt->band_parent_table);
            rt->band_parent_table = nullptr;
        }
        NWG_TRY(cudaMalloc(&rt->band_parent_table, global_rows * cols * sizeof(std::uint32_t)));
    }
    rt->band = true;
    rt->band_global_rows = global_rows;
    rt->band_row_first = band_row_first;
    rt->band_halo_rows = halo_rows;
    rt->band_reserved_slots = reserved;
    rt->band_halo_ready = false;
    rt->prepared = false;
    return kOk;
}

int nwg_device_generation(const nwg_runtime *rt, void **fitness, void **has_fitness, size_t *count) {
    if (rt == nullptr || fitness == nullptr || has_fitness == nullptr || count == nullptr) {
        return kInvalidRuntimeConfig;
    }
    *fitness = rt->cur_fitness;
    *has_fitness = rt->cur_has;
    *count = rt->cur_gen_size;
    return kOk;
}

int nwg_band_copy_rows(nwg_runtime *rt, size_t band_row, size_t rows, void *dst, size_t dst_pitch) {
    if (rt == nullptr || dst == nullptr || rt->released_parents) {
        return kInvalidRuntimeConfig;
    }
    const std::size_t cols = rt->grid_column_count;
    const std::size_t bytes = (rt->stride + 15) / 16 * 16;
    if (rows == 0 || (band_row + rows) * cols > rt->cur_gen_size || dst_pitch < bytes || dst_pitch % 16 != 0 ||
        reinterpret_cast<std::uintptr_t>(dst) % 16 != 0) {
        return kInvalidRuntimeConfig;
    }
    const std::uint32_t n = static_cast<std::uint32_t>(rows * cols);
    GatherSlotsKernel<<<n < 1024 ? n : 1024, 256, 0, rt->stream>>>(rt->slab, rt->pitch, rt->cur_slots + band_row * cols,
                                                                   static_cast<std::uint8_t *>(dst), dst_pitch, bytes,
                                                                   n);
    NWG_TRY(cudaGetLastError());
    return Sync(rt);
}

int nwg_band_install_halo(nwg_runtime *rt, const void *above, const void *below, size_t src_pitch) {
    if (rt == nullptr || !rt->band || above == nullptr || below == nullptr || src_pitch < rt->stride ||
        rt->released_parents) {
        return kInvalidRuntimeConfig;
    }
    const std::size_t cols = rt->grid_column_count;
    const std::size_t band_rows = rt->cur_gen_size / cols;
    const std::size_t halo_cells = rt->band_halo_rows * cols;
    const std::size_t reserved_base = rt->slot_count - rt->band_reserved_slots;
    if (band_rows * cols != rt->cur_gen_size || band_rows + 2 * rt->band_halo_rows > rt->band_global_rows) {
        return kInvalidGeneration;
    }
    std::uint8_t *base = rt->slab + reserved_base * rt->pitch;
    NWG_TRY(cudaMemcpy2DAsync(base, rt->pitch, above, src_pitch, rt->stride, halo_cells, cudaMemcpyDeviceToDevice,
                              rt->stream));
    NWG_TRY(cudaMemcpy2DAsync(base + halo_cells * rt->pitch, rt->pitch, below, src_pitch, rt->stride, halo_cells,
                              cudaMemcpyDeviceToDevice, rt->stream));
    const std::uint32_t cells = static_cast<std::uint32_t>(rt->band_global_rows * cols);
    BandParentTableKernel<<<(cells + 255) / 256, 256, 0, rt->stream>>>(
        rt->band_parent_table, static_cast<std::uint32_t>(rt->band_global_rows), static_cast<std::uint32_t>(cols),
        static_cast<std::uint32_t>(rt->band_row_first), static_cast<std::uint32_t>(band_rows),
        static_cast<std::uint32_t>(rt->band_halo_rows), rt->cur_slots, static_cast<std::uint32_t>(reserved_base));
    NWG_TRY(cudaGetLastError());
    const int st = Sync(rt);
    rt->band_halo_ready = st == kOk;
    return st;
}

int nwg_band_prepare(nwg_runtime *rt, uint32_t generation_seed, const nwg_generation_assembly_config *config,
                     const float *fitness_all, const uint8_t *has_fitness_all) {
    if (rt == nullptr || !rt->band || fitness_all == nullptr || has_fitness_all == nullptr) {
        return kInvalidRuntimeConfig;
    }
    rt->prepared = false;
    nwg_generation_assembly_config cfg{};
    cfg.parent_selection.cellular_breeding_radius = 2;  // selection.hpp:13-18, spatial/grid.hpp:11
    cfg.parent_selection.rank_exponent = 0.5f;
    cfg.breeding = {0.02f, 0.01f, 0.005f};
    cfg.mutation = {0.0001f, 0.02f, 0.0f};
    if (config != nullptr) {
        cfg = *config;
    }
    const auto in01 = [](float v) { return v >= 0.0f && v <= 1.0f; };
    // the band's children reach rows up to the radius away: the halo must cover them (radius <= 2 keeps the
    // Moore-list selection, which the halo bounds; the whole-grid scan above that is not split)
    const bool valid = cfg.parent_selection.cellular_breeding_radius > 0 &&
                       cfg.parent_selection.cellular_breeding_radius <= rt->band_halo_rows &&
                       cfg.parent_selection.cellular_breeding_radius <= 2 &&
                       cfg.parent_selection.rank_exponent >= 0.0f && cfg.parent_selection.rank_exponent <= 4.0f &&
                       in01(cfg.breeding.crossover_temperature_level1) &&
                       in01(cfg.breeding.crossover_temperature_level2) &&
                       in01(cfg.breeding.crossover_temperature_level3) && in01(cfg.mutation.mutation_probability) &&
                       cfg.mutation.mutation_sigma >= 0.0f &&
                       in01(cfg.mutation.output_tail_row_scale_mutation_probability);
    if (!valid) {
        return SetHostStatus(rt, kInvalidAssemblyConfig);
    }
    if (rt->cur_gen_size == 0 || rt->cur_gen_size % rt->grid_column_count != 0 || rt->released_parents) {
        return SetHostStatus(rt, kInvalidGeneration);
    }
    SelectParams sp{};
    sp.fitness = fitness_all;
    sp.has_fitness = has_fitness_all;
    sp.rows = static_cast<std::uint32_t>(rt->band_global_rows);
    sp.cols = static_cast<std::uint32_t>(rt->grid_column_count);
    sp.child_count = static_cast<std::uint32_t>(rt->cur_gen_size);
    sp.child_first = static_cast<std::uint32_t>(rt->band_row_first * rt->grid_column_count);
    sp.generation_index = rt->cur_gen_index;
    sp.radius = cfg.parent_selection.cellular_breeding_radius;
    sp.rank_exponent = cfg.parent_selection.rank_exponent;
    sp.planning_seed = generation_seed ^ 0xA341316Cu;  // slab_runtime.cu:1443
    sp.pairs = rt->pairs;
    sp.status = rt->status;
    NWG_TRY(LaunchSelect(sp, rt->stream));
    const int st = Sync(rt);
    if (st != kOk) {
        return st;
    }
    rt->planned_children = rt->cur_gen_size;
    rt->prepared = true;
    rt->prepared_seed = generation_seed;
    rt->prepared_config = cfg;
    rt->prepared_injection = nwg_pending_injection{};
    rt->prepared_next_action_count = rt->action_count;
    return kOk;
}

int nwg_select_parents_device(const float *fitness, const uint8_t *has_fitness, size_t population, size_t columns,
                              size_t child_count, size_t generation_index, const nwg_parent_selection_config *config,
                              uint32_t planning_seed, uint32_t *pairs, void *cuda_stream) {
    if (fitness == nullptr || has_fitness == nullptr || pairs == nullptr || config == nullptr || columns == 0 ||
        population % columns != 0 || child_count % columns != 0 || child_count > population ||
        config->cellular_breeding_radius == 0) {
        return kInvalidAssemblyConfig;
    }
    int *status = nullptr;
    if (cudaMalloc(&status, sizeof(int)) != cudaSuccess) {
        return kCudaFailure;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    cudaMemsetAsync(status, 0, sizeof(int), stream);
    SelectParams sp{};
    sp.fitness = fitness;
    sp.has_fitness = has_fitness;
    sp.rows = static_cast<std::uint32_t>(population / columns);
    sp.cols = static_cast<std::uint32_t>(columns);
    sp.child_count = static_cast<std::uint32_t>(child_count);
    sp.generation_index = generation_index;
    sp.radius = config->cellular_breeding_radius;
    sp.rank_exponent = config->rank_exponent;
    sp.planning_seed = planning_seed;
    sp.pairs = pairs;
    sp.status = status;
    int host_status = kCudaFailure;
    if (LaunchSelect(sp, stream) == cudaSuccess &&
        cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, stream) == cudaSuccess) {
        cudaStreamSynchronize(stream);
    }
    cudaFree(status);
    return host_status;
}

int nwg_breed_device(const void *parent_slab, size_t parent_pitch, const uint32_t *parent_slots, void *child_slab,
                     size_t child_pitch, const uint32_t *pairs, size_t child_count, size_t action_count,
                     uint32_t generation_seed, size_t generation_index, const nwg_breeding_config *breeding,
                     const nwg_mutation_config *mutation, void *cuda_stream) {
    if (parent_slab == nullptr || child_slab == nullptr || parent_slots == nullptr || pairs == nullptr ||
        breeding == nullptr || mutation == nullptr || parent_pitch % 16 != 0 || child_pitch % 16 != 0 ||
        parent_pitch < GenomeStrideBytes(action_count) || child_pitch < GenomeStrideBytes(action_count)) {
        return kInvalidAssemblyConfig;
    }
    BreedParams bp{};
    bp.parent_slab = static_cast<const std::uint8_t *>(parent_slab);
    bp.parent_pitch = parent_pitch;
    bp.parent_slots = parent_slots;
    bp.child_slab = static_cast<std::uint8_t *>(child_slab);
    bp.child_pitch = child_pitch;
    bp.child_slots = nullptr;
    bp.pairs = pairs;
    bp.child_count = static_cast<std::uint32_t>(child_count);
    bp.action_count = static_cast<std::uint32_t>(action_count);
    bp.generation_seed = generation_seed;
    bp.generation_index = generation_index;
    bp.crossover_l1 = breeding->crossover_temperature_level1;
    bp.crossover_l2 = breeding->crossover_temperature_level2;
    bp.crossover_l3 = breeding->crossover_temperature_level3;
    bp.mutation_probability = mutation->mutation_probability;
    bp.mutation_sigma = mutation->mutation_sigma;
    bp.row_scale_probability = mutation->output_tail_row_scale_mutation_probability;
    bp.status = nullptr;
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    if (LaunchBreed(bp, stream) != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess) {
        return kCudaFailure;
    }
    return kOk;
}

int nwg_bootstrap_device(void *slab, size_t pitch, size_t population, size_t generation_index, uint32_t seed,
                         size_t action_count, void *cuda_stream) {
    if (slab == nullptr || pitch < GenomeStrideBytes(action_count) || pitch % 2 != 0) {
        return kInvalidRuntimeConfig;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    if (LaunchBootstrap(static_cast<std::uint8_t *>(slab), pitch, nullptr, static_cast<std::uint32_t>(population),
                        generation_index, seed, static_cast<std::uint32_t>(action_count), stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
        return kCudaFailure;
    }
    return kOk;
}

}  // extern "C"
