// Single-model inference runtime (inference/single_model_device_runtime.hpp:22-47, .cu:89-183): one genome and its
// own action-space catalog resident on the device, next-guess selection for caller-given grids. The reference
// selects for one grid per call with one warp; here a call takes any number of grids, groups them by turn count
// into chunks of up to 128 and scores each chunk with the plain form's kernels (eval_fp32.cu,
// SingleModelSelectKernel), so one call answers a whole batch of games. The grid checks are the reference's
// (wordle_grid.hpp:37-67, wordle_grid_state.hpp:74-78): valid letters and tiles, at most five turns, not won.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

using namespace nwg;

struct nwg_single_model {
    cudaStream_t stream = nullptr;
    std::uint8_t *genome = nullptr;
    std::size_t genome_bytes = 0;
    std::size_t action_count = 0;
    std::uint32_t *codes = nullptr;
    float *fixed_t = nullptr;
    std::size_t pad = 0;
    std::vector<std::uint8_t> letters;  // host copy, for the selected words
    float *scratch = nullptr;
    int ctas = 0;
};

namespace {

constexpr std::size_t kInferenceTurns = 5;  // trunk input slots (wordle_grid_state.hpp:74-76)
constexpr int kInferenceCtas = 64;

void FreeModel(nwg_single_model *m) {
    if (m == nullptr) {
        return;
    }
    cudaFree(m->genome);
    cudaFree(m->codes);
    cudaFree(m->fixed_t);
    cudaFree(m->scratch);
    delete m;
}

}  // namespace

extern "C" {

int nwg_single_model_create(const uint8_t *genome_bytes, size_t genome_byte_count, const uint8_t *catalog_letters,
                            size_t catalog_count, nwg_single_model **model_out) {
    if (model_out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    *model_out = nullptr;
    // IsValidCreateInputs (single_model_device_runtime.cu:23-29): the genome's width is the catalog's
    if (genome_bytes == nullptr || catalog_letters == nullptr || catalog_count == 0 ||
        catalog_count > NWG_CATALOG_CAPACITY || genome_byte_count != GenomeStrideBytes(catalog_count)) {
        return kInvalidRuntimeConfig;
    }
    for (std::size_t i = 0; i < catalog_count * kWordLength; ++i) {
        if (catalog_letters[i] >= kAlphabet) {
            return kInvalidRuntimeConfig;
        }
    }
    nwg_single_model *m = new (std::nothrow) nwg_single_model();
    if (m == nullptr) {
        return kCudaFailure;
    }
    m->genome_bytes = genome_byte_count;
    m->action_count = catalog_count;
    m->letters.assign(catalog_letters, catalog_letters + catalog_count * kWordLength);
    m->ctas = kInferenceCtas;
    bool ok = BuildCatalogTables(catalog_letters, catalog_count, &m->codes, &m->fixed_t, &m->pad, nullptr) == kOk &&
              cudaMalloc(&m->genome, genome_byte_count) == cudaSuccess &&
              cudaMemcpy(m->genome, genome_bytes, genome_byte_count, cudaMemcpyHostToDevice) == cudaSuccess &&
              cudaMalloc(&m->scratch, static_cast<std::size_t>(m->ctas) * EvalScratchFloatsPerCta() * sizeof(float)) ==
                  cudaSuccess;
    if (!ok) {
        FreeModel(m);
        return kCudaFailure;
    }
    *model_out = m;
    return kOk;
}

void nwg_single_model_destroy(nwg_single_model *model) { FreeModel(model); }

int nwg_single_model_set_stream(nwg_single_model *model, void *cuda_stream) {
    if (model == nullptr) {
        return kInvalidRuntimeConfig;
    }
    model->stream = static_cast<cudaStream_t>(cuda_stream);
    return kOk;
}

int nwg_single_model_select(nwg_single_model *model, const uint8_t *guess_letters, const uint8_t *feedback,
                            const uint8_t *turn_counts, size_t grid_count, nwg_selected_action *actions) {
    if (model == nullptr || actions == nullptr || turn_counts == nullptr ||
        (grid_count > 0 && (guess_letters == nullptr || feedback == nullptr))) {
        return kInvalidRuntimeConfig;
    }
    if (grid_count == 0) {
        return kOk;
    }
    // pack the grids; group them by turn count
    std::vector<std::uint32_t> codes(grid_count * kInferenceTurns, 0);
    std::vector<std::uint16_t> tiles(grid_count * kInferenceTurns, 0);
    std::vector<std::vector<std::uint32_t>> by_turns(kInferenceTurns + 1);
    for (std::size_t g = 0; g < grid_count; ++g) {
        const std::size_t turns = turn_counts[g];
        if (turns > kInferenceTurns) {
            return kPolicyForwardFailed;
        }
        for (std::size_t u = 0; u < turns; ++u) {
            const std::uint8_t *word = guess_letters + (g * 6 + u) * kWordLength;
            const std::uint8_t *tile = feedback + (g * 6 + u) * kWordLength;
            std::uint32_t packed = 0;
            bool won = true;
            for (int k = 0; k < kWordLength; ++k) {
                if (word[k] >= kAlphabet || tile[k] > kGrey) {
                    return kPolicyForwardFailed;
                }
                packed |= static_cast<std::uint32_t>(tile[k]) << (2 * k);
                won = won && tile[k] == kGreen;
            }
            if (won) {
                return kPolicyForwardFailed;  // a finished grid has no next guess
            }
            codes[g * kInferenceTurns + u] = PackWord(word);
            tiles[g * kInferenceTurns + u] = static_cast<std::uint16_t>(packed);
        }
        by_turns[turns].push_back(static_cast<std::uint32_t>(g));
    }
    std::vector<std::uint32_t> order;
    std::vector<int4> chunks;
    for (std::size_t t = 0; t <= kInferenceTurns; ++t) {
        for (std::size_t b = 0; b < by_turns[t].size(); b += kChunkGames) {
            const std::size_t n = std::min<std::size_t>(kChunkGames, by_turns[t].size() - b);
            chunks.push_back(make_int4(static_cast<int>(t), static_cast<int>(order.size()), static_cast<int>(n), 0));
            order.insert(order.end(), by_turns[t].begin() + static_cast<std::ptrdiff_t>(b),
                         by_turns[t].begin() + static_cast<std::ptrdiff_t>(b + n));
        }
    }
    std::uint32_t *d_codes = nullptr, *d_order = nullptr;
    std::uint16_t *d_tiles = nullptr;
    int4 *d_chunks = nullptr;
    std::int32_t *d_index = nullptr;
    float *d_score = nullptr;
    std::vector<std::int32_t> index(grid_count);
    std::vector<float> score(grid_count);
    cudaStream_t s = model->stream;
    bool ok = cudaMalloc(&d_codes, codes.size() * 4) == cudaSuccess &&
              cudaMalloc(&d_tiles, tiles.size() * 2) == cudaSuccess &&
              cudaMalloc(&d_order, order.size() * 4) == cudaSuccess &&
              cudaMalloc(&d_chunks, chunks.size() * sizeof(int4)) == cudaSuccess &&
              cudaMalloc(&d_index, grid_count * 4) == cudaSuccess && cudaMalloc(&d_score, grid_count * 4) == cudaSuccess;
    ok = ok && cudaMemcpyAsync(d_codes, codes.data(), codes.size() * 4, cudaMemcpyHostToDevice, s) == cudaSuccess &&
         cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * 2, cudaMemcpyHostToDevice, s) == cudaSuccess &&
         cudaMemcpyAsync(d_order, order.data(), order.size() * 4, cudaMemcpyHostToDevice, s) == cudaSuccess &&
         cudaMemcpyAsync(d_chunks, chunks.data(), chunks.size() * sizeof(int4), cudaMemcpyHostToDevice, s) ==
             cudaSuccess;
    if (ok) {
        SingleModelParams q{};
        q.genome = model->genome;
        q.action_count = static_cast<std::uint32_t>(model->action_count);
        q.codes = model->codes;
        q.fixed_t = model->fixed_t;
        q.action_pad = static_cast<std::uint32_t>(model->pad);
        q.guess_codes = d_codes;
        q.tiles = d_tiles;
        q.chunks = d_chunks;
        q.order = d_order;
        q.chunk_count = static_cast<int>(chunks.size());
        q.scratch = model->scratch;
        q.best_index = d_index;
        q.best_score = d_score;
        const int ctas = std::min(model->ctas, static_cast<int>(chunks.size()));
        ok = LaunchSingleModelSelect(q, ctas, s) == cudaSuccess &&
             cudaMemcpyAsync(index.data(), d_index, grid_count * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
             cudaMemcpyAsync(score.data(), d_score, grid_count * 4, cudaMemcpyDeviceToHost, s) == cudaSuccess &&
             cudaStreamSynchronize(s) == cudaSuccess;
    }
    cudaFree(d_codes);
    cudaFree(d_tiles);
    cudaFree(d_order);
    cudaFree(d_chunks);
    cudaFree(d_index);
    cudaFree(d_score);
    if (!ok) {
        return kCudaFailure;
    }
    int status = kOk;
    for (std::size_t g = 0; g < grid_count; ++g) {
        nwg_selected_action &a = actions[g];
        std::memset(&a, 0, sizeof(a));
        if (index[g] < 0) {
            status = kActionSelectionFailed;  // every action already guessed
            continue;
        }
        a.action_index = static_cast<std::size_t>(index[g]);
        a.score = score[g];
        std::memcpy(a.word, model->letters.data() + a.action_index * kWordLength, kWordLength);
    }
    return status;
}

}  // extern "C"
