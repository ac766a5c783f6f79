// Surrogate-screened generation step (no reference counterpart): every cell breeds several candidate children, a
// learned model ranks them from their behaviour, and only the best of each cell (plus an audit sample) is played.
//
// One step, for a population of P cells whose per-cell word lists are set (CSR):
//   1. selection: the reference's cellular rank roulette (select.cu) drawn `candidates_per_cell` times with
//      planning seeds seed ^ 0xA341316C + k * 0x9E3779B9 (k = 0 is the plain step's plan);
//   2. breeding: all k * P children at once (breed.cu) into the slab of an evaluator runtime owned here, child
//      k * P + i being candidate k of cell i; candidate set 0 is exactly the plain step's children;
//   3. descriptors: each child's policy vectors on 128 fixed probe states (eval_fp32.cu, BF16);
//   4. inference: the MLP (surrogate_mlp.cu) scores every child;
//   5. screening: when the model is trained and its last audit rank correlation is at least the floor, the best-
//      scored child of each cell is played, plus an audit sample of the others; otherwise every child is played
//      (full evaluation) and the best-played child of each cell wins;
//   6. evaluation: the played children on the evaluator runtime in the configured form (default: FP16 tensor-core
//      trunk), each with its cell's words;
//   7. the audit: Spearman rank correlation between predicted score and fitness over the audit sample (or over
//      all played children on a full-evaluation step), before the model sees them;
//   8. learning: the played (descriptor, fitness) pairs enter a replay ring; a few Adam steps on minibatches drawn
//      from it, targets standardised per minibatch;
//   9. the winners become the population's next generation with their measured fitness.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <new>
#include <numeric>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"

using namespace nwg;

struct nwg_surrogate {
    nwg_runtime *rt = nullptr;    // the population (not owned)
    nwg_runtime *eval = nullptr;  // candidate slab and evaluator (owned)
    nwg_mlp *mlp = nullptr;
    nwg_surrogate_config cfg{};
    std::size_t P = 0, A = 0, cols = 0, candidates = 0, padded = 0;
    std::uint8_t *slab = nullptr;  // the evaluator's slab
    std::size_t pitch = 0;
    std::uint32_t *d_probe_codes = nullptr;
    std::uint16_t *d_probe_tiles = nullptr;
    std::uint8_t *d_probe_turns = nullptr;
    float scale = 0.0f;
    float *desc_scratch = nullptr;
    int desc_ctas = 0;
    std::uint16_t *descriptors = nullptr;  // [padded][8192]
    float *pred = nullptr;                 // [padded]
    std::uint32_t *pairs = nullptr;        // [candidates][2]
    std::uint32_t *identity = nullptr;     // [candidates]: candidate c sits in evaluator slot c
    std::uint16_t *replay_x = nullptr;     // [replay_capacity][8192]
    std::vector<float> replay_t;
    std::size_t replay_size = 0, replay_next = 0;
    std::uint16_t *batch_x = nullptr;
    float *batch_t = nullptr;
    std::uint32_t *d_rows = nullptr;       // row lists for the gathers
    std::uint32_t *d_rows2 = nullptr;
    std::vector<std::uint32_t> cell_offsets, cell_words;
    bool trained = false;
    float last_rho = std::numeric_limits<float>::quiet_NaN();
    std::uint64_t rng = 0;
};

namespace {

constexpr std::size_t kRow = kDescriptorWidth;  // descriptor values per row

std::uint64_t NextRandom(std::uint64_t &state) {  // splitmix64
    std::uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// rows dst_rows[i] of dst = rows src_rows[i] of src (kRow BF16 values each, 16-byte vectors)
__global__ void GatherRowsKernel(const std::uint16_t *src, const std::uint32_t *src_rows, std::uint16_t *dst,
                                 const std::uint32_t *dst_rows, std::uint32_t n) {
    constexpr int kVectors = static_cast<int>(kRow * 2 / 16);
    for (std::uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
        const uint4 *s = reinterpret_cast<const uint4 *>(src + static_cast<std::size_t>(src_rows[i]) * kRow);
        uint4 *d = reinterpret_cast<uint4 *>(dst + static_cast<std::size_t>(dst_rows != nullptr ? dst_rows[i] : i) *
                                                       kRow);
        for (int v = threadIdx.x; v < kVectors; v += blockDim.x) {
            d[v] = s[v];
        }
    }
}

// Spearman rank correlation with average ranks for ties.
float Spearman(const std::vector<float> &a, const std::vector<float> &b) {
    const std::size_t n = a.size();
    if (n < 3) {
        return std::numeric_limits<float>::quiet_NaN();
    }
    const auto ranks = [n](const std::vector<float> &v) {
        std::vector<std::size_t> order(n);
        std::iota(order.begin(), order.end(), std::size_t{0});
        std::stable_sort(order.begin(), order.end(), [&](std::size_t x, std::size_t y) { return v[x] < v[y]; });
        std::vector<double> r(n);
        for (std::size_t i = 0; i < n;) {
            std::size_t j = i;
            while (j + 1 < n && v[order[j + 1]] == v[order[i]]) {
                ++j;
            }
            const double avg = 0.5 * static_cast<double>(i + j);
            for (std::size_t k = i; k <= j; ++k) {
                r[order[k]] = avg;
            }
            i = j + 1;
        }
        return r;
    };
    const std::vector<double> ra = ranks(a), rb = ranks(b);
    const double ma = std::accumulate(ra.begin(), ra.end(), 0.0) / n;
    const double mb = std::accumulate(rb.begin(), rb.end(), 0.0) / n;
    double sab = 0.0, saa = 0.0, sbb = 0.0;
    for (std::size_t i = 0; i < n; ++i) {
        sab += (ra[i] - ma) * (rb[i] - mb);
        saa += (ra[i] - ma) * (ra[i] - ma);
        sbb += (rb[i] - mb) * (rb[i] - mb);
    }
    return (saa > 0.0 && sbb > 0.0) ? static_cast<float>(sab / std::sqrt(saa * sbb)) : 0.0f;
}

double Now() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

void FreeSurrogate(nwg_surrogate *s) {
    if (s == nullptr) {
        return;
    }
    if (s->eval != nullptr) {
        nwg_destroy(s->eval);
    }
    if (s->mlp != nullptr) {
        nwg_mlp_destroy(s->mlp);
    }
    void *ptrs[] = {s->d_probe_codes, s->d_probe_tiles, s->d_probe_turns, s->desc_scratch, s->descriptors, s->pred,
                    s->pairs,         s->identity,      s->replay_x,      s->batch_x,      s->batch_t,     s->d_rows,
                    s->d_rows2};
    for (void *p : ptrs) {
        cudaFree(p);
    }
    delete s;
}

int Descriptors(nwg_surrogate *s, cudaStream_t stream) {
    DescriptorParams q{};
    q.slab = s->slab;
    q.pitch = s->pitch;
    q.slots = s->identity;
    q.count = static_cast<std::uint32_t>(s->candidates);
    q.probe_codes = s->d_probe_codes;
    q.probe_tiles = s->d_probe_tiles;
    q.probe_turns = s->d_probe_turns;
    q.scale = s->scale;
    q.scratch = s->desc_scratch;
    q.out = s->descriptors;
    q.out_ld = kRow;
    return LaunchDescriptors(q, s->desc_ctas, stream) == cudaSuccess && cudaStreamSynchronize(stream) == cudaSuccess
               ? kOk
               : kCudaFailure;
}

}  // namespace

extern "C" {

int nwg_surrogate_create(nwg_runtime *rt, const nwg_surrogate_config *config, const uint8_t *catalog_letters,
                         size_t catalog_count, const uint32_t *secret_pool, size_t pool_count,
                         nwg_surrogate **out) {
    if (out == nullptr) {
        return kInvalidRuntimeConfig;
    }
    *out = nullptr;
    GenerationView v{};
    if (rt == nullptr || config == nullptr || catalog_letters == nullptr || ReadGenerationView(rt, &v) != kOk) {
        return kInvalidRuntimeConfig;
    }
    const nwg_surrogate_config &c = *config;
    if (v.generation_size == 0 || v.cell_count != v.generation_size || c.candidates_per_cell == 0 ||
        c.candidates_per_cell > 16 || c.batch_rows == 0 || c.batch_rows % 128 != 0 ||
        c.replay_capacity < c.batch_rows || catalog_count < v.action_count || !(c.audit_fraction >= 0.0f) ||
        c.audit_fraction > 1.0f) {
        return kInvalidRuntimeConfig;  // the population needs per-cell word lists (nwg_set_cell_words)
    }
    nwg_surrogate *s = new (std::nothrow) nwg_surrogate();
    if (s == nullptr) {
        return kCudaFailure;
    }
    s->rt = rt;
    s->cfg = c;
    s->P = v.generation_size;
    s->A = v.action_count;
    s->cols = v.grid_column_count;
    s->candidates = c.candidates_per_cell * s->P;
    s->padded = (s->candidates + 127) / 128 * 128;
    s->rng = 0x243f6a8885a308d3ULL ^ (static_cast<std::uint64_t>(c.seed) << 1);
    // the per-cell word lists of the population, for the played children's cells
    s->cell_offsets.resize(s->P + 1);
    bool ok = cudaStreamSynchronize(v.stream) == cudaSuccess &&
              cudaMemcpy(s->cell_offsets.data(), v.cell_offsets, (s->P + 1) * 4, cudaMemcpyDeviceToHost) == cudaSuccess;
    if (ok) {
        s->cell_words.resize(s->cell_offsets[s->P]);
        ok = cudaMemcpy(s->cell_words.data(), v.cell_words, s->cell_words.size() * 4, cudaMemcpyDeviceToHost) ==
             cudaSuccess;
    }
    // the evaluator: one column (any number of played children), a slot per candidate
    nwg_runtime_config ec{};
    ec.genotype_slab_byte_budget_bytes = s->candidates * v.stride;
    ec.generation_byte_budget_bytes = s->candidates * v.stride;
    ec.action_count = s->A;
    ec.population_size_ceiling = s->candidates;
    ec.grid_column_count = 1;
    ok = ok && nwg_create(&ec, &s->eval) == kOk && nwg_set_evaluation_form(s->eval, c.evaluation_form) == kOk &&
         (c.evaluation_form < NWG_FORM_TC_TRUNK_BF16 || nwg_set_margin_guard(s->eval, c.margin_tau) == kOk);
    void *slab = nullptr;
    ok = ok && nwg_device_slab(s->eval, &slab, &s->pitch) == kOk && s->pitch == v.pitch;
    s->slab = static_cast<std::uint8_t *>(slab);
    ok = ok && nwg_mlp_create(std::max(s->padded, c.batch_rows), c.seed, c.learning_rate, &s->mlp) == kOk;
    // probe states: a pool secret, 0..4 turns of catalog guesses (none the secret), their feedback
    std::vector<std::uint32_t> codes(kProbeStates * kProbeMaxTurns, 0);
    std::vector<std::uint16_t> tiles(kProbeStates * kProbeMaxTurns, 0);
    std::vector<std::uint8_t> turns(kProbeStates, 0);
    std::uint64_t prng = 0x13198a2e03707344ULL ^ c.seed;
    for (int p = 0; ok && p < kProbeStates; ++p) {
        const std::size_t si = secret_pool != nullptr ? secret_pool[NextRandom(prng) % pool_count]
                                                      : NextRandom(prng) % s->A;
        if (si >= catalog_count) {
            ok = false;
            break;
        }
        const std::uint32_t secret = PackWord(catalog_letters + 5 * si);
        turns[p] = static_cast<std::uint8_t>(NextRandom(prng) % (kProbeMaxTurns + 1));
        for (int u = 0; u < turns[p]; ++u) {
            std::uint32_t guess = secret;
            while (guess == secret) {
                guess = PackWord(catalog_letters + 5 * (NextRandom(prng) % s->A));
            }
            codes[p * kProbeMaxTurns + u] = guess;
            tiles[p * kProbeMaxTurns + u] = static_cast<std::uint16_t>(FeedbackPacked(guess, secret));
        }
    }
    std::vector<std::uint32_t> identity(s->candidates);
    std::iota(identity.begin(), identity.end(), 0u);
    s->desc_ctas = EvalCtaCount(static_cast<std::uint32_t>(s->candidates));
    ok = ok && cudaMalloc(&s->d_probe_codes, codes.size() * 4) == cudaSuccess &&
         cudaMalloc(&s->d_probe_tiles, tiles.size() * 2) == cudaSuccess &&
         cudaMalloc(&s->d_probe_turns, turns.size()) == cudaSuccess &&
         cudaMemcpy(s->d_probe_codes, codes.data(), codes.size() * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->d_probe_tiles, tiles.data(), tiles.size() * 2, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->d_probe_turns, turns.data(), turns.size(), cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMalloc(&s->desc_scratch, static_cast<std::size_t>(s->desc_ctas) * EvalScratchFloatsPerCta() * 4) ==
             cudaSuccess &&
         cudaMalloc(&s->descriptors, s->padded * kRow * 2) == cudaSuccess &&
         cudaMemset(s->descriptors, 0, s->padded * kRow * 2) == cudaSuccess &&
         cudaMalloc(&s->pred, s->padded * 4) == cudaSuccess &&
         cudaMalloc(&s->pairs, s->candidates * 2 * 4) == cudaSuccess &&
         cudaMalloc(&s->identity, s->candidates * 4) == cudaSuccess &&
         cudaMemcpy(s->identity, identity.data(), s->candidates * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMalloc(&s->replay_x, c.replay_capacity * kRow * 2) == cudaSuccess &&
         cudaMalloc(&s->batch_x, c.batch_rows * kRow * 2) == cudaSuccess &&
         cudaMalloc(&s->batch_t, c.batch_rows * 4) == cudaSuccess &&
         cudaMalloc(&s->d_rows, std::max(s->candidates, c.batch_rows) * 4) == cudaSuccess &&
         cudaMalloc(&s->d_rows2, std::max(s->candidates, c.batch_rows) * 4) == cudaSuccess;
    if (!ok) {
        FreeSurrogate(s);
        return kCudaFailure;
    }
    s->replay_t.assign(c.replay_capacity, 0.0f);
    *out = s;
    return kOk;
}

void nwg_surrogate_destroy(nwg_surrogate *s) { FreeSurrogate(s); }

int nwg_surrogate_advance(nwg_surrogate *s, uint32_t generation_seed, const nwg_runtime_word_counts *counts,
                          const nwg_generation_assembly_config *config, nwg_surrogate_stats *stats) {
    if (s == nullptr || counts == nullptr || config == nullptr) {
        return kInvalidRuntimeConfig;
    }
    nwg_surrogate_stats st{};
    const double t0 = Now();
    GenerationView v{};
    if (ReadGenerationView(s->rt, &v) != kOk || v.generation_size != s->P || v.action_count != s->A) {
        return kInvalidGeneration;
    }
    if (!v.evaluated) {
        const int e = nwg_evaluate(s->rt, counts, nullptr);
        if (e != kOk) {
            return e;
        }
        ReadGenerationView(s->rt, &v);
    }
    const nwg_surrogate_config &c = s->cfg;
    const std::size_t P = s->P, K = c.candidates_per_cell, N = s->candidates;
    cudaStream_t stream = v.stream;

    // 1-2. selection and breeding of every candidate
    for (std::size_t k = 0; k < K; ++k) {
        SelectParams sp{};
        sp.fitness = v.fitness;
        sp.has_fitness = v.has_fitness;
        sp.rows = static_cast<std::uint32_t>(P / s->cols);
        sp.cols = static_cast<std::uint32_t>(s->cols);
        sp.child_count = static_cast<std::uint32_t>(P);
        sp.generation_index = v.generation_index;
        sp.radius = config->parent_selection.cellular_breeding_radius;
        sp.rank_exponent = config->parent_selection.rank_exponent;
        sp.planning_seed = (generation_seed ^ 0xA341316Cu) + static_cast<std::uint32_t>(k) * 0x9E3779B9u;
        sp.pairs = s->pairs + 2 * P * k;
        sp.status = v.status;
        if (LaunchSelect(sp, stream) != cudaSuccess) {
            return kCudaFailure;
        }
    }
    BreedParams bp{};
    bp.parent_slab = v.slab;
    bp.parent_pitch = v.pitch;
    bp.parent_slots = v.slots;
    bp.child_slab = s->slab;
    bp.child_pitch = s->pitch;
    bp.child_slots = nullptr;
    bp.pairs = s->pairs;
    bp.child_count = static_cast<std::uint32_t>(N);
    bp.action_count = static_cast<std::uint32_t>(s->A);
    bp.generation_seed = generation_seed;
    bp.generation_index = v.generation_index;
    bp.crossover_l1 = config->breeding.crossover_temperature_level1;
    bp.crossover_l2 = config->breeding.crossover_temperature_level2;
    bp.crossover_l3 = config->breeding.crossover_temperature_level3;
    bp.mutation_probability = config->mutation.mutation_probability;
    bp.mutation_sigma = config->mutation.mutation_sigma;
    bp.row_scale_probability = config->mutation.output_tail_row_scale_mutation_probability;
    bp.status = v.status;
    int status = 0;
    if (LaunchBreed(bp, stream) != cudaSuccess || cudaStreamSynchronize(stream) != cudaSuccess ||
        nwg_read_status(s->rt, &status) != kOk) {
        return kCudaFailure;
    }
    if (status != kOk) {
        return status;
    }
    const double t1 = Now();

    // 3. descriptors (the first brood also fixes the input scale: 1 / RMS of its values)
    if (s->scale == 0.0f) {
        s->scale = 1.0f;
        if (Descriptors(s, stream) != kOk) {
            return kCudaFailure;
        }
        const std::size_t sample = std::min<std::size_t>(N, 256);
        std::vector<std::uint16_t> h(sample * kRow);
        if (cudaMemcpy(h.data(), s->descriptors, h.size() * 2, cudaMemcpyDeviceToHost) != cudaSuccess) {
            return kCudaFailure;
        }
        double sq = 0.0;
        for (const std::uint16_t b : h) {
            const std::uint32_t bits = static_cast<std::uint32_t>(b) << 16;
            float f;
            std::memcpy(&f, &bits, 4);
            sq += static_cast<double>(f) * f;
        }
        const double rms = std::sqrt(sq / static_cast<double>(h.size()));
        s->scale = rms > 0.0 ? static_cast<float>(1.0 / rms) : 1.0f;
    }
    if (Descriptors(s, stream) != kOk) {
        return kCudaFailure;
    }
    const double t2 = Now();

    // 4. inference
    std::vector<float> pred(N);
    if (nwg_mlp_set_stream(s->mlp, stream) != kOk || nwg_mlp_forward(s->mlp, s->descriptors, s->padded, s->pred) != kOk ||
        cudaMemcpy(pred.data(), s->pred, N * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        return kCudaFailure;
    }
    const double t3 = Now();

    // 5. who plays
    const bool screen = s->trained && s->replay_size >= c.warmup_pairs && s->last_rho >= c.spearman_floor;
    std::vector<std::uint32_t> chosen(P), played;
    std::vector<std::uint8_t> is_audit;
    if (screen) {
        for (std::size_t i = 0; i < P; ++i) {
            std::size_t best = 0;
            for (std::size_t k = 1; k < K; ++k) {
                best = pred[k * P + i] > pred[best * P + i] ? k : best;
            }
            chosen[i] = static_cast<std::uint32_t>(best * P + i);
        }
        std::vector<std::uint8_t> taken(N, 0);
        for (const std::uint32_t ch : chosen) {
            taken[ch] = 1;
        }
        std::vector<std::uint32_t> others;
        for (std::uint32_t ci = 0; ci < N; ++ci) {
            if (!taken[ci]) {
                others.push_back(ci);
            }
        }
        const std::size_t audit = std::min(others.size(), static_cast<std::size_t>(std::lround(c.audit_fraction * N)));
        for (std::size_t a = 0; a < audit; ++a) {  // partial Fisher-Yates
            std::swap(others[a], others[a + NextRandom(s->rng) % (others.size() - a)]);
        }
        played = chosen;
        played.insert(played.end(), others.begin(), others.begin() + static_cast<std::ptrdiff_t>(audit));
        is_audit.assign(played.size(), 0);
        std::fill(is_audit.begin() + static_cast<std::ptrdiff_t>(P), is_audit.end(), 1);
    } else {
        played.resize(N);
        std::iota(played.begin(), played.end(), 0u);
        is_audit.assign(N, 1);
    }

    // 6. play them on the evaluator, each with its cell's words
    const std::size_t m = played.size();
    std::vector<std::uint32_t> offsets(m + 1, 0), words;
    for (std::size_t j = 0; j < m; ++j) {
        const std::size_t cell = played[j] % P;
        words.insert(words.end(), s->cell_words.begin() + s->cell_offsets[cell],
                     s->cell_words.begin() + s->cell_offsets[cell + 1]);
        offsets[j + 1] = static_cast<std::uint32_t>(words.size());
    }
    std::vector<float> fit(m);
    std::vector<std::uint32_t> slots(m), evals(m);
    std::vector<std::uint8_t> has(m);
    std::vector<float> rates(m);
    std::size_t got = 0, gen = 0;
    double mean_rate = 0.0;
    int e = nwg_upload_current_generation(s->eval, played.data(), m, v.generation_index + 1);
    e = e == kOk ? nwg_set_cell_words(s->eval, offsets.data(), words.data(), m) : e;
    e = e == kOk ? nwg_evaluate(s->eval, counts, nullptr) : e;
    e = e == kOk ? nwg_download_current_generation(s->eval, slots.data(), fit.data(), evals.data(), has.data(), m, &got,
                                                   &gen)
                 : e;
    e = e == kOk ? nwg_read_solve_rates(s->eval, rates.data(), m, &got, &mean_rate) : e;
    if (e != kOk) {
        return e;
    }
    nwg_evaluation_stats es{};
    nwg_read_evaluation_stats(s->eval, &es);
    const double t4 = Now();

    // 7. the audit, before the model sees these children
    std::vector<float> audit_pred, audit_fit;
    for (std::size_t j = 0; j < m; ++j) {
        if (is_audit[j]) {
            audit_pred.push_back(pred[played[j]]);
            audit_fit.push_back(fit[j]);
        }
    }
    const float rho = s->trained ? Spearman(audit_pred, audit_fit) : std::numeric_limits<float>::quiet_NaN();
    s->last_rho = rho;
    // what the model would gain: on a full-evaluation step every child's fitness is known, so the model's pick,
    // candidate 0 (the plain step's child) and the best child of each cell can be compared on the same brood
    double model_pick = 0.0, first_pick = 0.0, best_pick = 0.0;
    const bool all_played = !screen;
    std::vector<float> chosen_fit(P), chosen_rate(P);
    std::vector<std::int64_t> where(N, -1);
    for (std::size_t j = 0; j < m; ++j) {
        where[played[j]] = static_cast<std::int64_t>(j);
    }
    for (std::size_t i = 0; i < P; ++i) {
        if (all_played) {
            std::size_t best = 0, model = 0;
            for (std::size_t k = 1; k < K; ++k) {
                best = fit[where[k * P + i]] > fit[where[best * P + i]] ? k : best;
                model = pred[k * P + i] > pred[model * P + i] ? k : model;
            }
            chosen[i] = static_cast<std::uint32_t>(best * P + i);
            best_pick += fit[where[best * P + i]];
            model_pick += fit[where[model * P + i]];
            first_pick += fit[where[i]];
        }
        chosen_fit[i] = fit[where[chosen[i]]];
        chosen_rate[i] = rates[where[chosen[i]]];
    }

    // 8. learning: the played pairs enter the replay ring, then Adam steps on minibatches from it
    std::vector<std::uint32_t> src(m), dst(m);
    for (std::size_t j = 0; j < m; ++j) {
        src[j] = played[j];
        dst[j] = static_cast<std::uint32_t>(s->replay_next);
        s->replay_t[s->replay_next] = fit[j];
        s->replay_next = (s->replay_next + 1) % c.replay_capacity;
        s->replay_size = std::min(s->replay_size + 1, c.replay_capacity);
    }
    bool ok = true;
    for (std::size_t b = 0; ok && b < m; b += N) {  // m <= N: one gather
        ok = cudaMemcpy(s->d_rows, src.data(), m * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
             cudaMemcpy(s->d_rows2, dst.data(), m * 4, cudaMemcpyHostToDevice) == cudaSuccess;
        if (ok) {
            GatherRowsKernel<<<512, 256, 0, stream>>>(s->descriptors, s->d_rows, s->replay_x, s->d_rows2,
                                                      static_cast<std::uint32_t>(m));
            ok = cudaGetLastError() == cudaSuccess;
        }
    }
    float loss = 0.0f;
    std::size_t steps = 0;
    if (ok && s->replay_size >= c.batch_rows) {
        std::vector<std::uint32_t> rows(c.batch_rows);
        std::vector<float> t(c.batch_rows);
        for (std::size_t step = 0; ok && step < c.train_steps; ++step) {
            double mean = 0.0, sq = 0.0;
            for (std::size_t r = 0; r < c.batch_rows; ++r) {
                rows[r] = static_cast<std::uint32_t>(NextRandom(s->rng) % s->replay_size);
                t[r] = s->replay_t[rows[r]];
                mean += t[r];
            }
            mean /= static_cast<double>(c.batch_rows);
            for (const float x : t) {
                sq += (x - mean) * (x - mean);
            }
            const double sd = std::sqrt(sq / static_cast<double>(c.batch_rows)) + 1e-6;
            for (float &x : t) {
                x = static_cast<float>((x - mean) / sd);
            }
            ok = cudaMemcpyAsync(s->d_rows, rows.data(), c.batch_rows * 4, cudaMemcpyHostToDevice, stream) ==
                     cudaSuccess &&
                 cudaMemcpyAsync(s->batch_t, t.data(), c.batch_rows * 4, cudaMemcpyHostToDevice, stream) == cudaSuccess;
            if (ok) {
                GatherRowsKernel<<<512, 256, 0, stream>>>(s->replay_x, s->d_rows, s->batch_x, nullptr,
                                                          static_cast<std::uint32_t>(c.batch_rows));
                ok = cudaGetLastError() == cudaSuccess &&
                     nwg_mlp_train_step(s->mlp, s->batch_x, s->batch_t, c.batch_rows) == kOk &&
                     cudaStreamSynchronize(stream) == cudaSuccess;
                ++steps;
            }
        }
        if (ok && steps > 0) {
            // the loss on the last minibatch after its step
            ok = nwg_mlp_gradients(s->mlp, s->batch_x, s->batch_t, c.batch_rows, nullptr, &loss) == kOk;
            s->trained = true;
        }
    }
    if (!ok) {
        return kCudaFailure;
    }
    const double t5 = Now();

    // 9. the winners become the next generation
    e = InstallGeneration(s->rt, s->slab, s->pitch, chosen, chosen_fit, v.generation_index + 1);
    if (e != kOk) {
        return e;
    }
    const double t6 = Now();
    if (stats != nullptr) {
        st.generation = v.generation_index + 1;
        st.candidates = N;
        st.evaluated = m;
        st.screened = screen;
        st.spearman = rho;
        st.train_loss = loss;
        st.train_steps = steps;
        st.replay_size = s->replay_size;
        double fsum = 0.0, rsum = 0.0;
        for (std::size_t i = 0; i < P; ++i) {
            fsum += chosen_fit[i];
            rsum += chosen_rate[i];
        }
        st.mean_fitness = fsum / static_cast<double>(P);
        const double nan = std::numeric_limits<double>::quiet_NaN();
        const bool compared = all_played && s->trained && !std::isnan(rho);
        st.mean_fitness_model_pick = compared ? model_pick / static_cast<double>(P) : nan;
        st.mean_fitness_first_candidate = all_played ? first_pick / static_cast<double>(P) : nan;
        st.mean_fitness_best_candidate = all_played ? best_pick / static_cast<double>(P) : nan;
        st.mean_solve_rate = rsum / static_cast<double>(P);
        st.game_steps = es.game_steps;
        st.ms_select_breed = static_cast<float>(t1 - t0);
        st.ms_descriptors = static_cast<float>(t2 - t1);
        st.ms_inference = static_cast<float>(t3 - t2);
        st.ms_evaluation = static_cast<float>(t4 - t3);
        st.ms_training = static_cast<float>(t5 - t4);
        st.ms_install = static_cast<float>(t6 - t5);
        st.ms_total = static_cast<float>(t6 - t0);
        *stats = st;
    }
    return kOk;
}

}  // extern "C"
