// Fitness evaluation for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: embedders whose device memory is owned by another allocator or
// pool (a second allocator would fragment it or exceed its accounting), and processes that must keep a
// fixed device-memory footprint after start-up (an allocation in the middle of a run can fail or stall
// the device). They can hand this entry point device buffers they already own; everything else the
// evaluation needs (the per-CTA layer-1 accumulators, the per-cell word counts and chunk offsets, the
// catalog tables, the score sums and the status word) lives in one fixed array of this file,
// g_noalloc_scratch.
//
// The word lists are the caller's device buffers and are not read on the host: a cell whose offsets
// decrease, or whose list is empty or longer than 2^20 words, is refused on the device
// (NWG_INVALID_TRAINING_SHARD) and none of its words is read. The call ends with a read of the status
// word and a synchronisation of the caller's stream.
//
// The array is a file-scope __device__ variable, so every GPU that loads the library holds it until
// the process exits. Host code cannot use the symbol as a device address: on first use on each device
// its address is resolved with cudaGetSymbolAddress while that device is current, and that pointer is
// what the kernels receive.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kNoAllocCtas = 32;
constexpr std::uint32_t kNoAllocMaxPopulation = 4096;
constexpr std::uint32_t kNoAllocMaxCatalog = NWG_CATALOG_CAPACITY;
constexpr std::uint32_t kNoAllocCatalogPad = ((kNoAllocMaxCatalog + 127) / 128) * 128;

// Byte offsets of the regions inside the scratch array (each 256-byte aligned).
constexpr std::size_t Align256(std::size_t n) { return (n + 255) / 256 * 256; }
constexpr std::size_t kLayer1Bytes = static_cast<std::size_t>(kNoAllocCtas) * kChunkGames * kHidden0 * sizeof(float);
constexpr std::size_t kOffLayer1 = 0;
constexpr std::size_t kOffCodes = kOffLayer1 + Align256(kLayer1Bytes);
constexpr std::size_t kOffFixed = kOffCodes + Align256(kNoAllocCatalogPad * sizeof(std::uint32_t));
constexpr std::size_t kOffWords = kOffFixed + Align256(static_cast<std::size_t>(kFixedDim) * kNoAllocCatalogPad * 4);
constexpr std::size_t kOffChunks = kOffWords + Align256(kNoAllocMaxPopulation * sizeof(std::uint32_t));
constexpr std::size_t kOffScores = kOffChunks + Align256((kNoAllocMaxPopulation + 1) * sizeof(std::uint32_t));
constexpr std::size_t kOffEvals = kOffScores + Align256(kNoAllocMaxPopulation * sizeof(std::uint32_t));
constexpr std::size_t kOffHas = kOffEvals + Align256(kNoAllocMaxPopulation * sizeof(std::uint32_t));
constexpr std::size_t kOffStatus = kOffHas + Align256(kNoAllocMaxPopulation);
constexpr std::size_t kNoAllocScratchBytes = kOffStatus + 256;
static_assert(kNoAllocScratchBytes == 4789760, "the documented maximum scratch size");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
unsigned char *g_scratch_address[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Device address of g_noalloc_scratch on the current device (resolved once per device).
int ScratchAddress(unsigned char **out) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= kMaxDevices) {
        return kCudaFailure;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_address[device] == nullptr) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || ptr == nullptr) {
            return kCudaFailure;
        }
        g_scratch_address[device] = static_cast<unsigned char *>(ptr);
    }
    *out = g_scratch_address[device];
    return kOk;
}

// Packed codes and the [26][pad] fixed word-feature table (output_embedding.hpp:59-73) from letter rows.
__global__ void NoAllocCatalogKernel(const std::uint8_t *letters, std::uint32_t count, std::uint32_t *codes,
                                     float *fixed_t, int *status) {
    const std::uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= kNoAllocCatalogPad) {
        return;
    }
    if (w >= count) {
        codes[w] = 0;
        for (int l = 0; l < kFixedDim; ++l) {
            fixed_t[static_cast<std::size_t>(l) * kNoAllocCatalogPad + w] = 0.0f;
        }
        return;
    }
    int counts[kAlphabet] = {0};
    bool valid = true;
    for (int p = 0; p < kWordLength; ++p) {
        const std::uint8_t letter = letters[kWordLength * w + p];
        valid &= letter < kAlphabet;
        counts[letter < kAlphabet ? letter : 0] += 1;
    }
    if (!valid) {
        SetStatus(status, kInvalidTrainingShard);
    }
    codes[w] = PackWord(letters + kWordLength * w);
    for (int l = 0; l < kFixedDim; ++l) {
        fixed_t[static_cast<std::size_t>(l) * kNoAllocCatalogPad + w] =
            counts[l] == 0 ? -1.0f : static_cast<float>(counts[l]);
    }
}

}  // namespace
}  // namespace nwg

using namespace nwg;

extern "C" int nwg_evaluate_noalloc(const void *slab, size_t slot_pitch, const uint32_t *slot_indices,
                                    size_t population, size_t grid_column_count, size_t action_count,
                                    const uint8_t *catalog_letters, size_t catalog_count,
                                    const uint32_t *cell_offsets, const uint32_t *cell_words, float *fitness,
                                    uint64_t *counters, void *cuda_stream) {
    if (slab == nullptr || slot_indices == nullptr || catalog_letters == nullptr || cell_offsets == nullptr ||
        cell_words == nullptr || fitness == nullptr || grid_column_count == 0 || population == 0 ||
        population % grid_column_count != 0 || slot_pitch % 16 != 0 ||
        slot_pitch < GenomeStrideBytes(action_count) || action_count == 0 || action_count > catalog_count) {
        return kInvalidRuntimeConfig;
    }
    if (population > kNoAllocMaxPopulation || catalog_count > kNoAllocMaxCatalog) {
        return kUnsupported;  // beyond the fixed scratch array
    }
    unsigned char *scratch = nullptr;
    const int setup = ScratchAddress(&scratch);
    if (setup != kOk) {
        return setup;
    }
    cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
    auto *codes = reinterpret_cast<std::uint32_t *>(scratch + kOffCodes);
    auto *fixed_t = reinterpret_cast<float *>(scratch + kOffFixed);
    auto *local_words = reinterpret_cast<std::uint32_t *>(scratch + kOffWords);
    auto *chunk_start = reinterpret_cast<std::uint32_t *>(scratch + kOffChunks);
    auto *score_sum = reinterpret_cast<std::uint32_t *>(scratch + kOffScores);
    auto *evaluation_counts = reinterpret_cast<std::uint32_t *>(scratch + kOffEvals);
    auto *has_fitness = reinterpret_cast<std::uint8_t *>(scratch + kOffHas);
    auto *status = reinterpret_cast<int *>(scratch + kOffStatus);
    // The array keeps the previous call's contents: clear what this call accumulates into.
    if (cudaMemsetAsync(status, 0, sizeof(int), stream) != cudaSuccess ||
        cudaMemsetAsync(evaluation_counts, 0, population * sizeof(std::uint32_t), stream) != cudaSuccess ||
        (counters != nullptr && cudaMemsetAsync(counters, 0, 3 * sizeof(std::uint64_t), stream) != cudaSuccess)) {
        return kCudaFailure;
    }
    NoAllocCatalogKernel<<<(kNoAllocCatalogPad + 255) / 256, 256, 0, stream>>>(
        catalog_letters, static_cast<std::uint32_t>(catalog_count), codes, fixed_t, status);
    if (cudaGetLastError() != cudaSuccess) {
        return kCudaFailure;
    }
    WordSource src{};
    src.mode = 0;
    src.cell_offsets = cell_offsets;
    src.cell_words = cell_words;
    src.rows = static_cast<std::uint32_t>(population / grid_column_count);
    src.cols = static_cast<std::uint32_t>(grid_column_count);
    const std::uint32_t p = static_cast<std::uint32_t>(population);
    if (LaunchEvalPrepare(src, p, static_cast<std::uint32_t>(catalog_count), local_words, chunk_start, score_sum,
                          status, stream) != cudaSuccess) {
        return kCudaFailure;
    }
    EvalParams params{};
    params.slab = static_cast<const std::uint8_t *>(slab);
    params.pitch = slot_pitch;
    params.slot_of_individual = slot_indices;
    params.population = p;
    params.action_count = static_cast<std::uint32_t>(action_count);
    params.catalog_count = static_cast<std::uint32_t>(catalog_count);
    params.codes = codes;
    params.fixed_t = fixed_t;
    params.action_pad = kNoAllocCatalogPad;
    params.source = src;
    params.chunk_start = chunk_start;
    params.local_words = local_words;
    params.scratch = reinterpret_cast<float *>(scratch + kOffLayer1);
    params.score_sum = score_sum;
    params.steps = reinterpret_cast<unsigned long long *>(counters);
    params.status = status;
    if (counters == nullptr) {
        // the kernel always counts; without an output buffer the counts go to the scratch status region's tail
        params.steps = reinterpret_cast<unsigned long long *>(scratch + kOffStatus + 64);
        if (cudaMemsetAsync(params.steps, 0, 3 * sizeof(unsigned long long), stream) != cudaSuccess) {
            return kCudaFailure;
        }
    }
    if (LaunchEvalFp32(params, kNoAllocCtas, stream) != cudaSuccess ||
        LaunchFinalizeFitness(score_sum, local_words, p, fitness, evaluation_counts, has_fitness, status, stream) !=
            cudaSuccess) {
        return kCudaFailure;
    }
    int host_status = kCudaFailure;
    if (cudaMemcpyAsync(&host_status, status, sizeof(int), cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess) {
        return kCudaFailure;
    }
    return host_status;
}
