/*
 * CPU oracle for the fitness-evaluation / generation-step path of
 * sam-bee/neuroevolutionary-wordle.
 *
 * TEST INFRASTRUCTURE ONLY. Nothing in the product links this library: it is
 * the checker that the CUDA path is compared against in tests/, in
 * __graft_entry__.smoke() and in bench.py's cpu_baseline leg.
 *
 * Every function restates one reference function and cites the reference file
 * and line it follows (paths are relative to the reference project root).
 *
 * Parity pins:
 *   - feedback, encoder, policy and argmax golden vectors from the reference's
 *     own tests (tests/wordle/wordle_grid_test.cpp:107-125,
 *     tests/model/input_encoder/shared_encoder_fixture.hpp,
 *     tests/model/policy_model/policy_model_fixture.hpp:85-107,
 *     tests/inference/dynamic_policy_test.cu:144-232) are checked in
 *     tests/test_oracle_golden.py;
 *   - the reference's host-callable code, compiled from its own headers into
 *     oracle/_ref/libref_host.so, is compared with this restatement on random
 *     genomes in tests/test_oracle_vs_reference_host.py;
 *   - the reference's device functions, compiled into oracle/_ref/libref_dev.so,
 *     are compared on the GPU in tests/test_gpu_parity_*.py.
 *
 * Arithmetic mode: the reference's device code is compiled by nvcc with the
 * default --fmad=true, which contracts every `sum += w * x` into one fused
 * multiply-add. The oracle follows that device arithmetic with fmaf() when
 * nwo_set_fma_mode(1) (the default); nwo_set_fma_mode(0) gives the separately
 * rounded multiply-then-add that the reference's host build (g++, ISO C++,
 * no FMA contraction) produces.
 */
#ifndef NWG_ORACLE_H
#define NWG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Genome image sizes (reference genetic_algorithm/genome/dynamic_layout.hpp:26-36). */
#define NWO_POLICY_HALFS 150528u
#define NWO_TAIL_DIM 38u
#define NWO_FIXED_DIM 26u
#define NWO_POLICY_DIM 64u

size_t nwo_genome_stride_bytes(size_t action_count);
void nwo_set_fma_mode(int on);

/* wordle/feedback.hpp:103-136 ; returns 1 on success, 0 for invalid letters. */
int nwo_feedback(const uint8_t guess[5], const uint8_t solution[5], uint8_t feedback[5]);

/* Encoded turn (shared encoder, model/input_encoder/shared_encoder.hpp:94-117). */
void nwo_encode_turn(const uint16_t *genome, const uint8_t guess[5], const uint8_t feedback[5], float out[64]);

/* Policy forward of a grid state (model/policy_model/policy_model.hpp:28-38).
 * guesses/feedbacks hold turn_count rows of 5 bytes. Returns 1 on success,
 * 0 where the reference's TryEncodeWordleGridState rejects the state. */
int nwo_policy_forward(const uint16_t *genome, size_t turn_count, const uint8_t *guesses, const uint8_t *feedbacks,
                       int finished, float out[64]);

/* model/output_embedding/output_embedding.hpp:98-119 */
float nwo_score_action(const float policy[64], const uint8_t word[5], const uint16_t tail[38]);

/* Episode evaluation of one individual (genetic_algorithm/device/evaluation_ops.cuh:203-237,511-589).
 * cell_words: the cell's local training words (catalog indices) in local order.
 * Per episode e (0 <= e < 3*W): score[e], turns[e], guesses[e*6 .. e*6+5]
 * (catalog indices, -1 past the end), policy[(e*6+s)*64 ..] the policy vector of
 * step s (may be NULL). Returns 0 on success or the reference's
 * DeviceGenomeEvaluationStatusCode (evaluation_ops.cuh:47-53) on failure;
 * *steps_out receives the number of policy decisions. */
int nwo_evaluate_individual(const uint16_t *genome, size_t action_count, const uint8_t *catalog_letters,
                            size_t catalog_count, const uint32_t *cell_words, size_t word_count,
                            float *raw_fitness_out, uint64_t *steps_out, float *episode_scores, int32_t *episode_turns,
                            int32_t *episode_guesses, float *policy_trace);

/* genetic_algorithm/device/evaluation_ops.cuh:97-111 */
float nwo_normalize_fitness(float raw_fitness, size_t training_word_count);

/* Shard coverage (training_folder/training_data.hpp:135-143,208-223). */
typedef struct {
    uint64_t first_catalog_word_index;
    uint64_t word_count;
    uint64_t center_row;
    uint64_t center_column;
    uint64_t radius;
    uint8_t global_from_outset;
} nwo_shard;

/* Expands the cell's local word list from a shard set (evaluation_ops.cuh:122-169).
 * Returns the number of words written (capped at capacity); 0 if uncovered. */
size_t nwo_cell_words_from_shards(const nwo_shard *shards, size_t shard_count, size_t rows, size_t cols,
                                  size_t cell_index, uint32_t *out, size_t capacity);

/* Cellular rank-roulette selection (genetic_algorithm/device/selection_ops.cuh:26-263).
 * draws: per child {tie_seed_hi, tie_seed_lo, uniform_bits, tie_seed_hi2, tie_seed_lo2, uniform_bits2}
 * as consumed from the child's Philox stream (the uniforms are passed as the
 * float bit pattern of the value the stream produced). rank_weights[r] is
 * rank^exponent for r = 0..max_rank (index 0 unused). Returns 1 on success. */
int nwo_select_parent_pair(const float *fitness, const uint8_t *has_fitness, size_t rows, size_t cols,
                           size_t next_rows, size_t child_index, size_t radius, const uint32_t draws[6],
                           const float *rank_weights, size_t max_rank, uint32_t *first_parent, uint32_t *second_parent);

/* Random-draw source for breeding and bootstrap: a tape of one Philox stream
 * indexed by raw 32-bit output position. For position j: raw[j] is the j-th
 * 32-bit output, uniform[j] the uniform derived from it, normal_pair[2j],
 * normal_pair[2j+1] the two standard normals derived from outputs j and j+1.
 * The tape is produced on the GPU by calling the toolkit's generator; the
 * oracle only replays it. */
typedef struct {
    const uint32_t *raw;
    const float *uniform;
    const float *normal_pair;
    size_t length;
    /* walk state */
    size_t position;
    int has_cached_normal;
    float cached_normal;
    int overflow;
} nwo_draw_tape;

typedef struct {
    float crossover_l1, crossover_l2, crossover_l3;
    float mutation_probability, mutation_sigma, row_scale_probability;
} nwo_breed_config;

/* genetic_algorithm/device/genome_ops.cuh:386-407 (BreedAndMutateGenome).
 * Parents and child are genome images of action_count tail rows.
 * Returns 1 on success, 0 if the tape ran out. */
int nwo_breed_and_mutate(const uint16_t *first_parent, const uint16_t *second_parent, size_t action_count,
                         uint16_t *child, nwo_draw_tape *tape, const nwo_breed_config *config);

/* Bootstrap of one organism (genome_ops.cuh:100-143, genotype_slab/device_runtime.cu:258-314).
 * normals[t * normals_per_thread + k] is the k-th standard normal of virtual
 * thread t's stream (t = 0..255). */
void nwo_bootstrap_genome(uint16_t *genome, size_t action_count, const float *normals, size_t normals_per_thread);

/* Number of standard normals that virtual thread `tid` of 256 consumes in bootstrap. */
size_t nwo_bootstrap_normals_per_thread(size_t action_count, size_t tid);

/* Population summary (slab_runtime.cu:588-631). */
void nwo_summarize(const float *fitness, size_t count, float *best, float *average, size_t *best_index);

/* Hint-grid group of a word (wordle/hint_grid.hpp:127-162): the cyclic grid and two swap grids; per grid its
 * turn count and turn rows (guess letters, feedback 0 green / 1 yellow / 2 grey). Returns 0 when the word
 * has no such group. */
int nwo_hint_grid_group(const uint8_t solution[5], size_t turn_counts[3], uint8_t guesses[3][4][5],
                        uint8_t feedbacks[3][4][5]);

/* Median norm of the first row_count tail rows (genetic_algorithm/output_embedding_injection.hpp:77-102). */
float nwo_median_tail_norm(const uint16_t *genome, size_t row_count);

/* Output-embedding injection of `count` new catalog words into a genome whose tail already holds
 * `parent_action_count` rows and has room for `count` more (device/injection_ops.cuh:22-64).
 * Returns 0 on success, 1 for an invalid catalog range, 2 when injection fails. */
int nwo_inject_tails(uint16_t *genome, size_t parent_action_count, const uint8_t *catalog_letters,
                     size_t catalog_count, size_t first, size_t count);

#ifdef __cplusplus
}
#endif

#endif
