/*
 * CPU oracle: a restatement of the reference's fitness-evaluation and
 * generation-step path, written from the reference's behaviour.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg are its only users; no product code links it.
 *
 * Citations are "file:line" in sam-bee/neuroevolutionary-wordle.
 */
#include "nwg_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ---- fp16 storage (common/float16.hpp:9-13): IEEE binary16, round to nearest even ---- */
typedef _Float16 nwo_f16;

static inline float h2f(uint16_t bits) {
    nwo_f16 v;
    memcpy(&v, &bits, sizeof v);
    return (float)v;
}

static inline uint16_t f2h(float value) {
    nwo_f16 v = (nwo_f16)value;
    uint16_t bits;
    memcpy(&bits, &v, sizeof bits);
    return bits;
}

/* ---- genome image offsets, in halfs (parameter structs under model/, in declaration order) ---- */
enum {
    ENC_W1 = 0,          /* 128 x 145, row-major by output (shared_encoder.hpp:17-25) */
    ENC_B1 = 18560,      /* 128 */
    ENC_W2 = 18688,      /* 64 x 128 */
    ENC_B2 = 26880,      /* 64 */
    TR_W1 = 26944,       /* 256 x 321 (dense_trunk.hpp:26-40) */
    TR_B1 = 109120,      /* 256 */
    TR_W2 = 109376,      /* 128 x 256 */
    TR_B2 = 142144,      /* 128 */
    TR_W3 = 142272,      /* 64 x 128 */
    TR_B3 = 150464,      /* 64 */
    POLICY_END = 150528, /* tail rows start here (dynamic_layout.hpp:26-28) */
};

static int g_fma_mode = 1;

void nwo_set_fma_mode(int on) { g_fma_mode = on ? 1 : 0; }

/* One step of the reference's `sum += w * x` (shared_encoder.hpp:40-48, dense_trunk.hpp:46-54). */
static inline float mac(float w, float x, float sum) {
    if (g_fma_mode) {
        return fmaf(w, x, sum);
    }
    volatile float product = w * x;
    return sum + product;
}

size_t nwo_genome_stride_bytes(size_t action_count) {
    /* dynamic_layout.hpp:30-36: tail offset 301,056 B, 76 B per row, 2-byte alignment */
    if (action_count == 0) {
        return 0;
    }
    size_t bytes = (size_t)POLICY_END * 2u + action_count * NWO_TAIL_DIM * 2u;
    return (bytes + 1u) & ~(size_t)1u;
}

/* ---- Wordle rules ---- */

static int valid_word(const uint8_t w[5]) {
    for (int p = 0; p < 5; ++p) {
        if (w[p] >= 26) {
            return 0;
        }
    }
    return 1;
}

/* wordle/feedback.hpp:103-136: greens first, then yellows from the unmatched solution-letter counts. */
int nwo_feedback(const uint8_t guess[5], const uint8_t solution[5], uint8_t feedback[5]) {
    if (!valid_word(guess) || !valid_word(solution)) {
        return 0;
    }
    uint8_t unmatched[26];
    memset(unmatched, 0, sizeof unmatched);
    for (int p = 0; p < 5; ++p) {
        if (guess[p] == solution[p]) {
            feedback[p] = 0; /* green */
            continue;
        }
        feedback[p] = 2; /* grey */
        ++unmatched[solution[p]];
    }
    for (int p = 0; p < 5; ++p) {
        if (feedback[p] == 0) {
            continue;
        }
        if (unmatched[guess[p]] == 0) {
            continue;
        }
        feedback[p] = 1; /* yellow */
        --unmatched[guess[p]];
    }
    return 1;
}

typedef struct {
    uint8_t solution[5];
    uint8_t guess[6][5];
    uint8_t feedback[6][5];
    int32_t guess_index[6];
    size_t turn_count;
} grid_t;

static int words_equal(const uint8_t a[5], const uint8_t b[5]) { return memcmp(a, b, 5) == 0; }

/* wordle/wordle_grid.hpp:20-34 */
static int grid_won(const grid_t *g) {
    size_t n = g->turn_count < 6 ? g->turn_count : 6;
    for (size_t t = 0; t < n; ++t) {
        if (words_equal(g->guess[t], g->solution)) {
            return 1;
        }
    }
    return 0;
}

static int grid_finished(const grid_t *g) { return grid_won(g) || g->turn_count >= 6; }

/* wordle/wordle_grid.hpp:69-77 */
static int grid_append(grid_t *g, const uint8_t guess[5], int32_t index) {
    if (!valid_word(guess) || grid_finished(g)) {
        return 0;
    }
    memcpy(g->guess[g->turn_count], guess, 5);
    (void)nwo_feedback(guess, g->solution, g->feedback[g->turn_count]);
    g->guess_index[g->turn_count] = index;
    ++g->turn_count;
    return 1;
}

/* ---- model forward ---- */

/* turn_features.hpp:28-49 + shared_encoder.hpp:94-117 (one-hot layout: 5x26 letters then 5x3 tiles). */
void nwo_encode_turn(const uint16_t *genome, const uint8_t guess[5], const uint8_t feedback[5], float out[64]) {
    float x[145];
    memset(x, 0, sizeof x);
    for (int p = 0; p < 5; ++p) {
        x[p * 26 + guess[p]] = 1.0f;
        x[130 + p * 3 + feedback[p]] = 1.0f;
    }
    float hidden[128];
    for (int o = 0; o < 128; ++o) {
        float sum = h2f(genome[ENC_B1 + o]);
        for (int i = 0; i < 145; ++i) {
            sum = mac(h2f(genome[ENC_W1 + o * 145 + i]), x[i], sum);
        }
        hidden[o] = sum < 0.0f ? 0.0f : sum;
    }
    for (int o = 0; o < 64; ++o) {
        float sum = h2f(genome[ENC_B2 + o]);
        for (int i = 0; i < 128; ++i) {
            sum = mac(h2f(genome[ENC_W2 + o * 128 + i]), hidden[i], sum);
        }
        out[o] = sum;
    }
}

static void dense(const uint16_t *genome, int w_off, int b_off, int in_size, int out_size, const float *in, float *out,
                  int relu) {
    for (int o = 0; o < out_size; ++o) {
        float sum = h2f(genome[b_off + o]);
        const uint16_t *row = genome + w_off + (size_t)o * in_size;
        for (int i = 0; i < in_size; ++i) {
            sum = mac(h2f(row[i]), in[i], sum);
        }
        out[o] = (relu && sum < 0.0f) ? 0.0f : sum;
    }
}

/* model_input/wordle_grid_state.hpp:39-66 (virgin flag + five 64-wide turn slots, zeros past turn_count)
 * and dense_trunk.hpp:102-114 (321 -> 256 ReLU -> 128 ReLU -> 64). */
int nwo_policy_forward(const uint16_t *genome, size_t turn_count, const uint8_t *guesses, const uint8_t *feedbacks,
                       int finished, float out[64]) {
    if (turn_count > 5 || finished) {
        return 0;
    }
    float input[321];
    memset(input, 0, sizeof input);
    input[0] = (turn_count == 0) ? 1.0f : 0.0f;
    for (size_t t = 0; t < turn_count; ++t) {
        nwo_encode_turn(genome, guesses + 5 * t, feedbacks + 5 * t, input + 1 + 64 * t);
    }
    float h0[256];
    float h1[128];
    dense(genome, TR_W1, TR_B1, 321, 256, input, h0, 1);
    dense(genome, TR_W2, TR_B2, 256, 128, h0, h1, 1);
    dense(genome, TR_W3, TR_B3, 128, 64, h1, out, 0);
    return 1;
}

/* output_embedding.hpp:59-73 (letter counts, -1 when absent) and :98-119 (fixed dims then tail dims). */
float nwo_score_action(const float policy[64], const uint8_t word[5], const uint16_t tail[38]) {
    uint8_t counts[26];
    memset(counts, 0, sizeof counts);
    for (int p = 0; p < 5; ++p) {
        ++counts[word[p]];
    }
    float score = 0.0f;
    for (int l = 0; l < 26; ++l) {
        float fixed = counts[l] == 0 ? -1.0f : (float)counts[l];
        score = mac(policy[l], fixed, score);
    }
    for (int k = 0; k < 38; ++k) {
        score = mac(policy[26 + k], h2f(tail[k]), score);
    }
    return score;
}

/* inference/dynamic_policy.hpp:51-64 (mask by word equality) and :67-151 (max score, lowest index on ties). */
static int select_next_guess(const uint16_t *genome, size_t action_count, const uint8_t *catalog, const grid_t *g,
                             float policy_out[64], int32_t *best_index) {
    float policy[64];
    if (!nwo_policy_forward(genome, g->turn_count, &g->guess[0][0], &g->feedback[0][0], grid_finished(g), policy)) {
        return 3; /* kPolicyForwardFailed */
    }
    if (policy_out) {
        memcpy(policy_out, policy, sizeof policy);
    }
    const uint16_t *tails = genome + POLICY_END;
    int found = 0;
    float best = 0.0f;
    int32_t best_i = 0;
    for (size_t a = 0; a < action_count; ++a) {
        const uint8_t *word = catalog + 5 * a;
        int masked = 0;
        for (size_t t = 0; t < g->turn_count; ++t) {
            if (words_equal(g->guess[t], word)) {
                masked = 1;
                break;
            }
        }
        if (masked) {
            continue;
        }
        float s = nwo_score_action(policy, word, tails + 38 * a);
        if (!found || s > best) {
            found = 1;
            best = s;
            best_i = (int32_t)a;
        }
    }
    if (!found) {
        return 4; /* kActionSelectionFailed */
    }
    *best_index = best_i;
    return 0;
}

/* evaluation_ops.cuh:239-242 */
static float score_completed_episode(const grid_t *g) {
    return grid_won(g) ? (10.0f + (float)(6 - (int)g->turn_count)) : 0.0f;
}

/* evaluation_ops.cuh:203-237 (episode e: secret e/3; variant e%3 prefills words e/3+1,+2 or +3,+4 mod W). */
static int init_episode(const uint8_t *catalog, size_t catalog_count, const uint32_t *cell_words, size_t w,
                        size_t episode, grid_t *g) {
    memset(g, 0, sizeof *g);
    for (int t = 0; t < 6; ++t) {
        g->guess_index[t] = -1;
    }
    size_t entry = episode / 3;
    size_t variant = episode % 3;
    uint32_t solution_index = cell_words[entry];
    if (solution_index >= catalog_count) {
        return 1; /* kInvalidTrainingShard */
    }
    memcpy(g->solution, catalog + 5 * solution_index, 5);
    if (variant == 0) {
        return 0;
    }
    size_t first = (variant == 1) ? entry + 1 : entry + 3;
    uint32_t i0 = cell_words[first % w];
    uint32_t i1 = cell_words[(first + 1) % w];
    if (i0 >= catalog_count || i1 >= catalog_count) {
        return 1;
    }
    if (!grid_append(g, catalog + 5 * i0, (int32_t)i0) || !grid_append(g, catalog + 5 * i1, (int32_t)i1)) {
        return 2; /* kGuessAppendFailed */
    }
    return 0;
}

int nwo_evaluate_individual(const uint16_t *genome, size_t action_count, const uint8_t *catalog_letters,
                            size_t catalog_count, const uint32_t *cell_words, size_t word_count,
                            float *raw_fitness_out, uint64_t *steps_out, float *episode_scores, int32_t *episode_turns,
                            int32_t *episode_guesses, float *policy_trace) {
    *raw_fitness_out = 0.0f;
    *steps_out = 0;
    if (word_count == 0 || action_count == 0 || action_count > catalog_count) {
        return 1;
    }
    float raw = 0.0f;
    uint64_t steps = 0;
    for (size_t e = 0; e < 3 * word_count; ++e) {
        grid_t g;
        int status = init_episode(catalog_letters, catalog_count, cell_words, word_count, e, &g);
        if (status != 0) {
            return status;
        }
        int step = 0;
        while (!grid_finished(&g)) {
            int32_t best = 0;
            float *trace = policy_trace ? policy_trace + ((size_t)e * 6 + (size_t)step) * 64 : NULL;
            status = select_next_guess(genome, action_count, catalog_letters, &g, trace, &best);
            if (status != 0) {
                return status;
            }
            if (!grid_append(&g, catalog_letters + 5 * (size_t)best, best)) {
                return 2;
            }
            ++steps;
            ++step;
        }
        float score = score_completed_episode(&g);
        raw += score;
        if (episode_scores) {
            episode_scores[e] = score;
        }
        if (episode_turns) {
            episode_turns[e] = (int32_t)g.turn_count;
        }
        if (episode_guesses) {
            for (int t = 0; t < 6; ++t) {
                episode_guesses[e * 6 + t] = g.guess_index[t];
            }
        }
    }
    *raw_fitness_out = raw;
    *steps_out = steps;
    return 0;
}

/* evaluation_ops.cuh:87-111; floor from spatial/grid.hpp:14 */
float nwo_normalize_fitness(float raw_fitness, size_t training_word_count) {
    const float floor_value = 1.40129846e-45f;
    float maximum = 3.0f * 15.0f * (float)training_word_count;
    if (maximum <= 0.0f) {
        return floor_value;
    }
    float normalized = raw_fitness / maximum;
    if (normalized >= 1.0f) {
        return 1.0f;
    }
    return normalized > floor_value ? normalized : floor_value;
}

/* ---- spatial grid (spatial/grid.hpp:119-168) ---- */

static size_t axis_distance(size_t a, size_t b, size_t side) {
    size_t forward = a >= b ? a - b : b - a;
    size_t wrapped = side - forward;
    return forward < wrapped ? forward : wrapped;
}

static size_t chebyshev(size_t rows, size_t cols, size_t a, size_t b) {
    size_t dr = axis_distance(a / cols, b / cols, rows);
    size_t dc = axis_distance(a % cols, b % cols, cols);
    return dr > dc ? dr : dc;
}

/* training_data.hpp:135-143 + :208-223 (validity is judged against the 4,739-word catalog capacity). */
static int shard_covers(const nwo_shard *s, size_t rows, size_t cols, size_t cell) {
    const uint64_t capacity = 4739;
    if (s->word_count == 0 || s->first_catalog_word_index >= capacity ||
        s->word_count > capacity - s->first_catalog_word_index) {
        return 0;
    }
    if (!s->global_from_outset && (s->center_row >= rows || s->center_column >= cols)) {
        return 0;
    }
    if (cell >= rows * cols) {
        return 0;
    }
    if (s->global_from_outset) {
        return 1;
    }
    size_t center = (size_t)s->center_row * cols + (size_t)s->center_column;
    return chebyshev(rows, cols, center, cell) <= s->radius;
}

/* evaluation_ops.cuh:122-169: local word j is the j-th word of the concatenated covering shard ranges. */
size_t nwo_cell_words_from_shards(const nwo_shard *shards, size_t shard_count, size_t rows, size_t cols,
                                  size_t cell_index, uint32_t *out, size_t capacity) {
    size_t n = 0;
    for (size_t s = 0; s < shard_count; ++s) {
        if (!shard_covers(&shards[s], rows, cols, cell_index)) {
            continue;
        }
        for (uint64_t k = 0; k < shards[s].word_count; ++k) {
            if (n < capacity) {
                out[n] = (uint32_t)(shards[s].first_catalog_word_index + k);
            }
            ++n;
        }
    }
    return n < capacity ? n : capacity;
}

/* ---- selection (genetic_algorithm/device/selection_ops.cuh) ---- */

static uint64_t mix_key(uint64_t value) { /* selection_ops.cuh:32-37 (splitmix64 finaliser) */
    value += 0x9E3779B97F4A7C15ULL;
    value = (value ^ (value >> 30)) * 0xBF58476D1CE4E5B9ULL;
    value = (value ^ (value >> 27)) * 0x94D049BB133111EBULL;
    return value ^ (value >> 31);
}

/* selection_ops.cuh:43-57 */
static int ranks_before(float lf, size_t li, float rf, size_t ri, uint64_t seed) {
    if (lf < rf) {
        return 1;
    }
    if (lf > rf) {
        return 0;
    }
    uint64_t lk = mix_key(seed ^ (uint64_t)li);
    uint64_t rk = mix_key(seed ^ (uint64_t)ri);
    return (lk < rk) || (lk == rk && li < ri);
}

#define NWO_NO_INDEX ((size_t)-1)
#define NWO_MAX_CANDIDATES 4096

/* selection_ops.cuh:68-89 / :91-113 (the candidate set is passed explicitly in its iteration order). */
static size_t rank_within(const float *f, const uint8_t *has, const size_t *cand, size_t count, size_t ranked,
                          uint64_t seed, size_t excluded) {
    size_t rank = 1;
    for (size_t k = 0; k < count; ++k) {
        size_t c = cand[k];
        if (c == ranked || c == excluded || has[c] == 0) {
            continue;
        }
        if (ranks_before(f[c], c, f[ranked], ranked, seed)) {
            ++rank;
        }
    }
    return rank;
}

/* selection_ops.cuh:115-161 / :163-216 */
static int select_rank_weighted(const float *f, const uint8_t *has, const size_t *cand, size_t count,
                                uint64_t seed, float uniform, const float *weights, size_t max_rank, size_t excluded,
                                size_t *selected) {
    float total = 0.0f;
    int found = 0;
    size_t fallback = 0;
    for (size_t k = 0; k < count; ++k) {
        size_t c = cand[k];
        if (c == excluded || has[c] == 0) {
            continue;
        }
        size_t rank = rank_within(f, has, cand, count, c, seed, excluded);
        if (rank > max_rank) {
            return 0;
        }
        total += weights[rank];
        fallback = c;
        found = 1;
    }
    if (!found || total <= 0.0f) {
        return 0;
    }
    float threshold = uniform * total;
    float cumulative = 0.0f;
    for (size_t k = 0; k < count; ++k) {
        size_t c = cand[k];
        if (c == excluded || has[c] == 0) {
            continue;
        }
        size_t rank = rank_within(f, has, cand, count, c, seed, excluded);
        cumulative += weights[rank];
        if (threshold <= cumulative) {
            *selected = c;
            return 1;
        }
    }
    *selected = fallback;
    return 1;
}

static float bits_to_float(uint32_t bits) {
    float f;
    memcpy(&f, &bits, sizeof f);
    return f;
}

/* selection_ops.cuh:218-263 with spatial/grid.hpp:181-218 (Moore list for radius <= 2; every cell within the
 * toroidal Chebyshev radius, in index order, above that). */
int nwo_select_parent_pair(const float *fitness, const uint8_t *has_fitness, size_t rows, size_t cols,
                           size_t next_rows, size_t child_index, size_t radius, const uint32_t draws[6],
                           const float *rank_weights, size_t max_rank, uint32_t *first_parent, uint32_t *second_parent) {
    if (rows == 0 || cols == 0 || next_rows > rows || child_index >= next_rows * cols || radius == 0) {
        return 0;
    }
    size_t cand[NWO_MAX_CANDIDATES];
    size_t count = 0;
    size_t focal = (child_index / cols) * cols + (child_index % cols);
    if (radius <= 2) {
        long r = (long)radius;
        long fr = (long)(focal / cols), fc = (long)(focal % cols);
        for (long dr = -r; dr <= r; ++dr) {
            for (long dc = -r; dc <= r; ++dc) {
                long nr = (fr + dr) % (long)rows;
                if (nr < 0) nr += (long)rows;
                long nc = (fc + dc) % (long)cols;
                if (nc < 0) nc += (long)cols;
                size_t idx = (size_t)nr * cols + (size_t)nc;
                int dup = 0;
                for (size_t k = 0; k < count; ++k) {
                    if (cand[k] == idx) {
                        dup = 1;
                        break;
                    }
                }
                if (!dup) {
                    cand[count++] = idx;
                }
            }
        }
    } else {
        for (size_t c = 0; c < rows * cols; ++c) {
            if (chebyshev(rows, cols, focal, c) <= radius) {
                if (count >= NWO_MAX_CANDIDATES) {
                    return 0;
                }
                cand[count++] = c;
            }
        }
    }
    uint64_t seed1 = ((uint64_t)draws[0] << 32) ^ (uint64_t)draws[1];
    size_t p1 = 0, p2 = 0;
    if (!select_rank_weighted(fitness, has_fitness, cand, count, seed1, bits_to_float(draws[2]), rank_weights,
                              max_rank, NWO_NO_INDEX, &p1)) {
        return 0;
    }
    uint64_t seed2 = ((uint64_t)draws[3] << 32) ^ (uint64_t)draws[4];
    if (!select_rank_weighted(fitness, has_fitness, cand, count, seed2, bits_to_float(draws[5]), rank_weights,
                              max_rank, p1, &p2)) {
        return 0;
    }
    *first_parent = (uint32_t)p1;
    *second_parent = (uint32_t)p2;
    return 1;
}

/* ---- breeding (genetic_algorithm/device/genome_ops.cuh) ---- */

static float tape_uniform(nwo_draw_tape *t) {
    if (t->position >= t->length) {
        t->overflow = 1;
        return 1.0f;
    }
    return t->uniform[t->position++];
}

static uint32_t tape_u32(nwo_draw_tape *t) {
    if (t->position >= t->length) {
        t->overflow = 1;
        return 0;
    }
    return t->raw[t->position++];
}

/* One standard normal: a fresh pair consumes two raw outputs and keeps its second value for the next call. */
static float tape_normal(nwo_draw_tape *t) {
    if (t->has_cached_normal) {
        t->has_cached_normal = 0;
        return t->cached_normal;
    }
    if (t->position + 1 >= t->length) {
        t->overflow = 1;
        t->position = t->length;
        return 0.0f;
    }
    float first = t->normal_pair[2 * t->position];
    t->cached_normal = t->normal_pair[2 * t->position + 1];
    t->has_cached_normal = 1;
    t->position += 2;
    return first;
}

/* genome_ops.cuh:35-44 */
static int bernoulli(nwo_draw_tape *t, float p) {
    if (p <= 0.0f) {
        return 0;
    }
    if (p >= 1.0f) {
        return 1;
    }
    return tape_uniform(t) < p;
}

/* genome_ops.cuh:46-52 */
static size_t sample_index(nwo_draw_tape *t, size_t n) {
    if (n <= 1) {
        return 0;
    }
    return (size_t)(tape_u32(t) % (uint32_t)n);
}

typedef struct {
    int w_off, b_off, in_size, out_size;
} layer_t;

static const layer_t k_layers[5] = {
    {ENC_W1, ENC_B1, 145, 128}, {ENC_W2, ENC_B2, 128, 64}, {TR_W1, TR_B1, 321, 256},
    {TR_W2, TR_B2, 256, 128},   {TR_W3, TR_B3, 128, 64},
};

static void copy_layer(const uint16_t *src, uint16_t *dst, const layer_t *l) {
    memcpy(dst + l->w_off, src + l->w_off, (size_t)l->in_size * l->out_size * 2);
    memcpy(dst + l->b_off, src + l->b_off, (size_t)l->out_size * 2);
}

/* genome_ops.cuh:210-221 */
static void recombine_layer(const uint16_t *p1, const uint16_t *p2, uint16_t *child, const layer_t *l,
                            nwo_draw_tape *t, const nwo_breed_config *c, int source_first) {
    copy_layer(source_first ? p1 : p2, child, l);
    if (bernoulli(t, c->crossover_l3)) {
        size_t neuron = sample_index(t, (size_t)l->out_size);
        const uint16_t *src = source_first ? p2 : p1; /* the other parent */
        memcpy(child + l->w_off + neuron * l->in_size, src + l->w_off + neuron * l->in_size, (size_t)l->in_size * 2);
        child[l->b_off + neuron] = src[l->b_off + neuron];
    }
}

/* genome_ops.cuh:259-262 */
static int maybe_alternate(nwo_draw_tape *t, float p, int base_first) { return bernoulli(t, p) ? !base_first : base_first; }

/* genome_ops.cuh:153-167 */
static void mutate_buffer(uint16_t *buf, size_t n, nwo_draw_tape *t, const nwo_breed_config *c) {
    if (c->mutation_probability <= 0.0f || c->mutation_sigma <= 0.0f) {
        return;
    }
    for (size_t i = 0; i < n; ++i) {
        if (bernoulli(t, c->mutation_probability)) {
            float n_value = tape_normal(t);
            buf[i] = f2h(mac(c->mutation_sigma, n_value, h2f(buf[i])));
        }
    }
}

/* genome_ops.cuh:237-257 */
static void mutate_tail_row(uint16_t *row, nwo_draw_tape *t, const nwo_breed_config *c) {
    for (int i = 0; i < 38; ++i) {
        if (c->mutation_probability > 0.0f && bernoulli(t, c->mutation_probability) && c->mutation_sigma > 0.0f) {
            float n_value = tape_normal(t);
            row[i] = f2h(mac(c->mutation_sigma, n_value, h2f(row[i])));
        }
    }
    if (c->row_scale_probability > 0.0f && bernoulli(t, c->row_scale_probability)) {
        float scale = bernoulli(t, 0.5f) ? 1.02f : 0.98f; /* output_tail_ops.hpp:7-12 */
        for (int i = 0; i < 38; ++i) {
            row[i] = f2h(h2f(row[i]) * scale);
        }
    }
}

/* genome_ops.cuh:386-407 with :264-299 (policy recombination), :301-309, :344-376 (tail rows). */
int nwo_breed_and_mutate(const uint16_t *p1, const uint16_t *p2, size_t action_count, uint16_t *child,
                         nwo_draw_tape *t, const nwo_breed_config *c) {
    int enc_first = !bernoulli(t, c->crossover_l1);
    for (int l = 0; l < 2; ++l) {
        int src = maybe_alternate(t, c->crossover_l2, enc_first);
        recombine_layer(p1, p2, child, &k_layers[l], t, c, src);
    }
    int trunk_first = !bernoulli(t, c->crossover_l1);
    for (int l = 2; l < 5; ++l) {
        int src = maybe_alternate(t, c->crossover_l2, trunk_first);
        recombine_layer(p1, p2, child, &k_layers[l], t, c, src);
    }
    for (int l = 0; l < 5; ++l) {
        mutate_buffer(child + k_layers[l].w_off, (size_t)k_layers[l].in_size * k_layers[l].out_size, t, c);
        mutate_buffer(child + k_layers[l].b_off, (size_t)k_layers[l].out_size, t, c);
    }

    const uint16_t *t1 = p1 + POLICY_END;
    const uint16_t *t2 = p2 + POLICY_END;
    uint16_t *tc = child + POLICY_END;
    int rows_first = !bernoulli(t, c->crossover_l1);
    memcpy(tc, rows_first ? t1 : t2, action_count * 38 * 2);
    int has_swap = 0;
    size_t swap_index = 0;
    if (action_count > 0 && bernoulli(t, c->crossover_l2)) {
        has_swap = 1;
        swap_index = sample_index(t, action_count);
        memcpy(tc + 38 * swap_index, (rows_first ? t2 : t1) + 38 * swap_index, 76);
    }
    if (action_count > 0 && bernoulli(t, c->crossover_l3)) {
        size_t splice = sample_index(t, action_count);
        int row_first = (has_swap && splice == swap_index) ? !rows_first : rows_first;
        size_t point = 1 + sample_index(t, 37); /* genome_ops.cuh:335-342 */
        for (size_t k = 0; k < 38; ++k) {
            int from_first = (k < point) ? row_first : !row_first;
            tc[38 * splice + k] = from_first ? t1[38 * splice + k] : t2[38 * splice + k];
        }
    }
    for (size_t a = 0; a < action_count; ++a) {
        mutate_tail_row(tc + 38 * a, t, c);
    }
    return !t->overflow;
}

/* ---- bootstrap (genome_ops.cuh:61-143) ---- */

static const float k_fan_in[5] = {145.0f, 128.0f, 321.0f, 256.0f, 128.0f};

size_t nwo_bootstrap_normals_per_thread(size_t action_count, size_t tid) {
    size_t n = 0;
    for (int l = 0; l < 5; ++l) {
        size_t size = (size_t)k_layers[l].in_size * k_layers[l].out_size;
        if (tid < size) {
            n += (size - tid + 255) / 256;
        }
    }
    size_t tail = action_count * 38;
    if (tid < tail) {
        n += (tail - tid + 255) / 256;
    }
    return n;
}

void nwo_bootstrap_genome(uint16_t *genome, size_t action_count, const float *normals, size_t normals_per_thread) {
    for (size_t tid = 0; tid < 256; ++tid) {
        const float *stream = normals + tid * normals_per_thread;
        size_t k = 0;
        for (int l = 0; l < 5; ++l) {
            float stddev = 1.0f * sqrtf(2.0f / k_fan_in[l]);
            size_t size = (size_t)k_layers[l].in_size * k_layers[l].out_size;
            for (size_t i = tid; i < size; i += 256) {
                genome[k_layers[l].w_off + i] = f2h(stddev * stream[k++]);
            }
            for (size_t i = tid; i < (size_t)k_layers[l].out_size; i += 256) {
                genome[k_layers[l].b_off + i] = f2h(0.0f);
            }
        }
        for (size_t i = tid; i < action_count * 38; i += 256) {
            genome[POLICY_END + i] = f2h(0.05f * stream[k++]);
        }
    }
}

/* slab_runtime.cu:588-631 (best: ties to the lower index; mean: sequential fp32 sum). */
void nwo_summarize(const float *fitness, size_t count, float *best, float *average, size_t *best_index) {
    int found = 0;
    float b = 0.0f;
    size_t bi = 0;
    float sum = 0.0f;
    for (size_t i = 0; i < count; ++i) {
        sum += fitness[i];
        if (!found || fitness[i] > b || (fitness[i] == b && i < bi)) {
            found = 1;
            b = fitness[i];
            bi = i;
        }
    }
    *best = b;
    *average = count ? sum / (float)count : 0.0f;
    *best_index = bi;
}

/* ---- output-embedding injection for action-space growth ---- */

static void rotate_word_left(const uint8_t w[5], size_t rotation, uint8_t out[5]) { /* hint_grid.hpp:19-27 */
    for (size_t p = 0; p < 5; ++p) {
        out[p] = w[(p + rotation) % 5];
    }
}

static size_t count_tiles(const uint8_t fb[5], uint8_t tile) { /* hint_grid.hpp:39-50 */
    size_t n = 0;
    for (size_t p = 0; p < 5; ++p) {
        n += fb[p] == tile;
    }
    return n;
}

/* hint_grid.hpp:76-105: the solution's left rotations whose feedback is all yellow, in rotation order. */
static int build_cyclic_hint_grid(const uint8_t solution[5], grid_t *g) {
    memset(g, 0, sizeof *g);
    if (!valid_word(solution)) {
        return 0;
    }
    memcpy(g->solution, solution, 5);
    uint8_t appended[4][5];
    size_t appended_count = 0;
    for (size_t rotation = 1; rotation < 5; ++rotation) {
        uint8_t guess[5];
        rotate_word_left(solution, rotation, guess);
        int seen = words_equal(guess, solution);
        for (size_t k = 0; k < appended_count; ++k) {
            seen |= words_equal(appended[k], guess);
        }
        if (seen) {
            continue;
        }
        uint8_t fb[5];
        if (!nwo_feedback(guess, solution, fb) || count_tiles(fb, 1) != 5) {
            continue;
        }
        if (!grid_append(g, guess, -1)) {
            return 0;
        }
        memcpy(appended[appended_count++], guess, 5);
    }
    return 1;
}

/* hint_grid.hpp:107-125: the solution with two different letters swapped, if that reads 3 green + 2 yellow. */
static int build_swap_hint_grid(const uint8_t solution[5], size_t first, size_t second, grid_t *g) {
    memset(g, 0, sizeof *g);
    if (!valid_word(solution) || first >= 5 || second >= 5 || first == second || solution[first] == solution[second]) {
        return 0;
    }
    uint8_t guess[5];
    memcpy(guess, solution, 5);
    guess[first] = solution[second];
    guess[second] = solution[first];
    uint8_t fb[5];
    if (!nwo_feedback(guess, solution, fb) || count_tiles(fb, 0) != 3 || count_tiles(fb, 1) != 2) {
        return 0;
    }
    memcpy(g->solution, solution, 5);
    return grid_append(g, guess, -1);
}

/* hint_grid.hpp:127-162: the cyclic grid, then the first two swap grids with different guesses. */
int nwo_hint_grid_group(const uint8_t solution[5], size_t turn_counts[3], uint8_t guesses[3][4][5],
                        uint8_t feedbacks[3][4][5]) {
    grid_t grids[3];
    memset(grids, 0, sizeof grids);
    memset(turn_counts, 0, 3 * sizeof(size_t));
    memset(guesses, 0, 3 * 4 * 5);
    memset(feedbacks, 0, 3 * 4 * 5);
    if (!build_cyclic_hint_grid(solution, &grids[0])) {
        return 0;
    }
    size_t selected = 0;
    int ok = 0;
    for (size_t first = 0; first < 5 && !ok; ++first) {
        for (size_t second = first + 1; second < 5 && !ok; ++second) {
            grid_t swap;
            if (!build_swap_hint_grid(solution, first, second, &swap)) {
                continue;
            }
            int seen = 0;
            for (size_t k = 0; k < selected; ++k) {
                seen |= words_equal(grids[1 + k].guess[0], swap.guess[0]);
            }
            if (seen) {
                continue;
            }
            grids[1 + selected] = swap;
            ++selected;
            ok = selected == 2;
        }
    }
    if (!ok) {
        return 0;
    }
    for (size_t g = 0; g < 3; ++g) {
        turn_counts[g] = grids[g].turn_count;
        for (size_t t = 0; t < grids[g].turn_count; ++t) {
            memcpy(guesses[g][t], grids[g].guess[t], 5);
            memcpy(feedbacks[g][t], grids[g].feedback[t], 5);
        }
    }
    return 1;
}

/* output_embedding_injection.hpp:66-75 (the device build contracts `sum += v * v`). */
static float trainable_tail_norm(const uint16_t row[NWO_TAIL_DIM]) {
    float sum = 0.0f;
    for (size_t k = 0; k < NWO_TAIL_DIM; ++k) {
        const float v = h2f(row[k]);
        sum = mac(v, v, sum);
    }
    return sqrtf(sum);
}

static int cmp_float(const void *a, const void *b) {
    const float x = *(const float *)a;
    const float y = *(const float *)b;
    return (x > y) - (x < y);
}

/* output_embedding_injection.hpp:77-102: median of the rows' norms (mean of the two middle ones). */
float nwo_median_tail_norm(const uint16_t *genome, size_t row_count) {
    float *norms = (float *)malloc(row_count * sizeof(float));
    for (size_t a = 0; a < row_count; ++a) {
        norms[a] = trainable_tail_norm(genome + POLICY_END + NWO_TAIL_DIM * a);
    }
    qsort(norms, row_count, sizeof(float), cmp_float);
    const size_t upper = row_count / 2;
    const float median = (row_count % 2) != 0 ? norms[upper] : 0.5f * (norms[upper - 1] + norms[upper]);
    free(norms);
    return median;
}

/* device/injection_ops.cuh:22-64 with output_embedding_injection.hpp:117-199: for each new word, the mean of
 * the policy's 38 trainable outputs over its three hint grids (rounded to FP16), rescaled to the median norm
 * of the genome's existing rows. */
int nwo_inject_tails(uint16_t *genome, size_t parent_action_count, const uint8_t *catalog_letters,
                     size_t catalog_count, size_t first, size_t count) {
    if (genome == NULL || parent_action_count == 0 || count == 0 || first != parent_action_count) {
        return 2;
    }
    if (first >= catalog_count || count > catalog_count - first) {
        return 1;
    }
    const float target = nwo_median_tail_norm(genome, parent_action_count);
    const float third = 1.0f / 3.0f;
    for (size_t i = 0; i < count; ++i) {
        size_t turns[3];
        uint8_t guesses[3][4][5];
        uint8_t feedbacks[3][4][5];
        if (!nwo_hint_grid_group(catalog_letters + 5 * (first + i), turns, guesses, feedbacks)) {
            return 2;
        }
        float sums[NWO_TAIL_DIM];
        memset(sums, 0, sizeof sums);
        for (size_t g = 0; g < 3; ++g) {
            float policy[64];
            if (!nwo_policy_forward(genome, turns[g], &guesses[g][0][0], &feedbacks[g][0][0], 0, policy)) {
                return 2;
            }
            for (size_t k = 0; k < NWO_TAIL_DIM; ++k) {
                sums[k] += policy[26 + k];
            }
        }
        uint16_t *row = genome + POLICY_END + NWO_TAIL_DIM * (parent_action_count + i);
        for (size_t k = 0; k < NWO_TAIL_DIM; ++k) {
            row[k] = f2h(sums[k] * third);
        }
        float scale = 0.0f;
        if (target > 1.0e-6f) {
            const float current = trainable_tail_norm(row);
            if (!(current > 1.0e-6f)) {
                return 2;
            }
            scale = target / current;
        }
        for (size_t k = 0; k < NWO_TAIL_DIM; ++k) {
            row[k] = f2h(h2f(row[k]) * scale);
        }
    }
    return 0;
}
