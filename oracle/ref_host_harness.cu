// Host-side harness around the reference's own host-callable code.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_ref/libref_host.so by oracle/build.py
// from the reference's headers where they lie; never copied into this repository).
// It is the "reference" CPU path: the reference's model forward, scoring, masking,
// feedback and grid rules (all NEUROEVOLUTION_HOST_DEVICE) composed into the
// reference's episode loop. The episode set-up in the reference is __device__-only
// (genetic_algorithm/device/evaluation_ops.cuh:171-237), so that glue is restated
// here on the host, line for line in behaviour.
//
// Compiled by nvcc as host code only because inference/dynamic_policy.hpp declares a
// __device__ template next to the host-callable masking helper it exports.
#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "genetic_algorithm/genome/dynamic_layout.hpp"
#include "inference/dynamic_policy.hpp"
#include "model/output_embedding/output_embedding.hpp"
#include "model/policy_model/policy_model.hpp"
#include "wordle/feedback.hpp"
#include "wordle/wordle_grid.hpp"

namespace {

using neuroevolution::genetic_algorithm::genome::GenomePolicyModelParameters;
using neuroevolution::genetic_algorithm::genome::GenomeTailRows;
using neuroevolution::inference::dynamic_policy::HasGridAlreadyGuessedWord;
using neuroevolution::inference::dynamic_policy::ScoreDynamicActionEmbedding;
using neuroevolution::model::policy_model::PolicyVector;
using neuroevolution::model::policy_model::TryForwardPolicyModel;
using neuroevolution::wordle::MakeWordleGrid;
using neuroevolution::wordle::TryAppendGuess;
using neuroevolution::wordle::Word;
using neuroevolution::wordle::WordleGrid;

Word ToWord(const std::uint8_t *letters) {
    Word word{};
    for (std::size_t p = 0; p < 5; ++p) {
        word.letter_indices[p] = letters[p];
    }
    return word;
}

// Restates evaluation_ops.cuh:203-237 over an explicit local word list.
bool InitializeEpisode(const std::uint8_t *catalog, const std::uint32_t *cell_words, std::size_t w,
                       std::size_t episode, WordleGrid &grid) {
    const std::size_t entry = episode / 3;
    const std::size_t variant = episode % 3;
    grid = MakeWordleGrid(ToWord(catalog + 5 * cell_words[entry]));
    if (variant == 0) {
        return true;
    }
    const std::size_t first = (variant == 1) ? entry + 1 : entry + 3;
    return TryAppendGuess(grid, ToWord(catalog + 5 * cell_words[first % w])) &&
           TryAppendGuess(grid, ToWord(catalog + 5 * cell_words[(first + 1) % w]));
}

// One individual's episodes, in the reference's episode loop
// (evaluation_ops.cuh:511-553 with dynamic_policy.hpp:67-151 semantics).
int EvaluateIndividual(const std::uint8_t *genome, std::size_t action_count, const std::uint8_t *catalog,
                       const std::uint32_t *cell_words, std::size_t w, float &raw_out, std::uint64_t &steps_out) {
    const auto &parameters = GenomePolicyModelParameters(genome);
    const auto *tails = GenomeTailRows(genome);
    std::vector<Word> words(action_count);
    for (std::size_t a = 0; a < action_count; ++a) {
        words[a] = ToWord(catalog + 5 * a);
    }
    float raw = 0.0f;
    std::uint64_t steps = 0;
    for (std::size_t e = 0; e < 3 * w; ++e) {
        WordleGrid grid{};
        if (!InitializeEpisode(catalog, cell_words, w, e, grid)) {
            return 2;
        }
        while (!grid.IsFinished()) {
            PolicyVector policy{};
            if (!TryForwardPolicyModel(parameters, grid, policy)) {
                return 3;
            }
            bool found = false;
            float best = 0.0f;
            std::size_t best_index = 0;
            for (std::size_t a = 0; a < action_count; ++a) {
                if (HasGridAlreadyGuessedWord(grid, words[a])) {
                    continue;
                }
                const float score = ScoreDynamicActionEmbedding(policy, words[a], tails[a]);
                if (!found || score > best) {
                    found = true;
                    best = score;
                    best_index = a;
                }
            }
            if (!found) {
                return 4;
            }
            if (!TryAppendGuess(grid, words[best_index])) {
                return 2;
            }
            ++steps;
        }
        raw += grid.IsWon() ? (10.0f + static_cast<float>(6 - grid.turn_count)) : 0.0f;
    }
    raw_out = raw;
    steps_out = steps;
    return 0;
}

} // namespace

extern "C" {

int refhost_feedback(const std::uint8_t *guess, const std::uint8_t *solution, std::uint8_t *feedback) {
    neuroevolution::wordle::Feedback out{};
    if (!neuroevolution::wordle::TryProvideFeedback(ToWord(guess), ToWord(solution), out)) {
        return 0;
    }
    for (std::size_t p = 0; p < 5; ++p) {
        feedback[p] = static_cast<std::uint8_t>(out[p]);
    }
    return 1;
}

// Policy vector of the grid (solution, guesses[0..turn_count)) built with the reference's TryAppendGuess.
int refhost_policy_forward(const std::uint8_t *genome, const std::uint8_t *solution, std::size_t turn_count,
                           const std::uint8_t *guesses, float *out) {
    WordleGrid grid = MakeWordleGrid(ToWord(solution));
    for (std::size_t t = 0; t < turn_count; ++t) {
        if (!TryAppendGuess(grid, ToWord(guesses + 5 * t))) {
            return 0;
        }
    }
    PolicyVector policy{};
    if (!TryForwardPolicyModel(GenomePolicyModelParameters(genome), grid, policy)) {
        return 0;
    }
    std::memcpy(out, policy.values, sizeof(float) * 64);
    return 1;
}

float refhost_score_action(const float *policy, const std::uint8_t *word, const std::uint8_t *tail_row_bytes) {
    PolicyVector p{};
    std::memcpy(p.values, policy, sizeof(float) * 64);
    neuroevolution::genetic_algorithm::genome::TrainableActionEmbeddingTail tail{};
    std::memcpy(tail.values, tail_row_bytes, sizeof(tail.values));
    return ScoreDynamicActionEmbedding(p, ToWord(word), tail);
}

std::size_t refhost_genome_stride_bytes(std::size_t action_count) {
    return neuroevolution::genetic_algorithm::genome::ComputeDynamicGenomeStrideBytes(action_count);
}

// Evaluates `count` individuals (genome i at genomes + i * pitch) with `threads` host threads.
// Cell c's local words are cell_words[cell_offsets[c] .. cell_offsets[c+1]).
int refhost_evaluate_population(const std::uint8_t *genomes, std::size_t pitch, std::size_t count,
                                std::size_t action_count, const std::uint8_t *catalog,
                                const std::uint32_t *cell_offsets, const std::uint32_t *cell_words,
                                const std::uint32_t *cell_of_individual, int threads, float *raw_out,
                                std::uint64_t *steps_out, int *status_out) {
    std::atomic<std::size_t> next{0};
    auto worker = [&]() {
        for (;;) {
            const std::size_t i = next.fetch_add(1);
            if (i >= count) {
                return;
            }
            const std::uint32_t cell = cell_of_individual[i];
            const std::uint32_t begin = cell_offsets[cell];
            const std::uint32_t end = cell_offsets[cell + 1];
            status_out[i] = EvaluateIndividual(genomes + i * pitch, action_count, catalog, cell_words + begin,
                                               end - begin, raw_out[i], steps_out[i]);
        }
    };
    std::vector<std::thread> pool;
    const int n = threads < 1 ? 1 : threads;
    for (int t = 0; t < n; ++t) {
        pool.emplace_back(worker);
    }
    for (auto &thread : pool) {
        thread.join();
    }
    return 0;
}

} // extern "C"
