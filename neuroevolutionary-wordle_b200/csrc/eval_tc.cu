// Fitness evaluation, tensor-core scoring form: action scores on tcgen05, decisions re-scored exactly.
//
// Same chunk structure, encoder and FP32 trunk as the plain form (eval_common.cuh, or trunk_fp32.cuh when the
// exact trunk tables are built); only the scoring phase differs. Per game step and chunk of up to 128 games:
//   1. the FP32 policy vectors are rounded to 16-bit (BF16, or FP16) into a K-major operand tile;
//   2. the individual's embedding table, kept as a 16-bit copy in the tensor-core layout
//      (BuildTcTablesKernel), streams through shared memory 128 actions at a time by bulk copies;
//   3. tcgen05.mma (M = 128 games, N = 128 actions, K = 64) fills two TMEM accumulators in turn; all eight warps
//      read a buffer back (tcgen05.ld) and keep, per game, the four largest 32-action chunk maxima; the first warp
//      to see a tile's MMAs complete refills its stage, and the last warp to read its buffer issues the tile two
//      ahead into it;
//   4. every chunk whose maximum lies within 2 * eps of the best chunk free of guessed words is re-scored
//      in FP32 with the plain form's own fused-multiply-add chain, and the game's guess is the exact FP32
//      argmax (ties to the lower index, guessed words masked).
//      eps bounds |tensor-core score - FP32 score|. FP16 operands: sum_k |fp16(p_k) - p_k| max_a |e_ak| (the
//      embeddings are exact in FP16) plus both 64-term FP32 accumulations; BF16 operands: kappa sum_k |p_k|
//      max_a |e_ak|, kappa covering both roundings and the accumulations. When the four tracked chunks cannot
//      prove that no other chunk reaches the window, the game is re-scored over every action. The guesses are
//      therefore identical to the plain form's.
// Every mbarrier wait is bounded; a wait that gives up records NWG_TIMEOUT and the kernel winds down.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tc_common.cuh"
#include "trunk_fp32.cuh"

namespace nwg {
namespace {

using namespace evalx;
using namespace tcx;

constexpr int kTileN = 128;                  // actions per MMA tile
constexpr std::uint32_t kTmemColumns = 256;  // two 128-column FP32 accumulators
constexpr std::uint32_t kDrainLimit = 1u << 22;  // polls of each wind-down wait after a failure
constexpr int kTileBytes = kTileN * kPolicy * 2;  // 16 KB of 16-bit embeddings per tile
constexpr int kMaxTasks = 2048;

// Shared-memory arena (floats) during the scoring phase: the FP32 policy vectors (arena[0 .. kTile)), the
// 16-bit policy operand and three 16 KB embedding tiles; once the tile loop ends, the candidate lists, task
// list and per-game keys reuse the embedding tiles' space.
constexpr int kStages = 3;
constexpr int kOffA = kTile;                          // 16-bit policy operand tile, 16 KB
constexpr int kOffB = kOffA + 4096;                   // kStages 16 KB embedding tiles
static_assert(kOffB + kStages * 4096 <= kArenaFloats, "embedding tiles must fit in the arena");
constexpr int kOffCand = kOffB;                       // [128 games][2 halves][4] values, then ids
constexpr int kOffTask = kOffCand + 2 * kChunkGames * 2 * kTopK;  // task list: (game << 16) | chunk
constexpr int kOffKeys = kOffTask + kMaxTasks;        // per game: packed (exact score, action) maximum
constexpr int kOffWindow = kOffKeys + 2 * kChunkGames;  // per game: best tensor-core score minus eps
constexpr int kOffFull = kOffWindow + kChunkGames;    // games re-scored over every action
constexpr int kOffEnd = kOffFull + kChunkGames;
static_assert(kOffEnd <= kArenaFloats, "scoring buffers must fit in the arena");
// FP16 operands: the policy vectors again as contiguous [game][64] rows for the exact re-scores (the embedding
// stages' space, free once the tile loop ends)
constexpr int kOffPvRows = kOffEnd;
static_assert(kOffPvRows + kChunkGames * kPolicy <= kArenaFloats, "policy rows must fit in the arena");
static_assert((kOffPvRows * 4) % 16 == 0, "policy rows are read 16 bytes at a time");
static_assert((kOffKeys * 4) % 8 == 0, "64-bit keys need 8-byte alignment");

struct TcState {
    std::uint64_t mbar_load[kStages];
    std::uint64_t mbar_mma[2];
    std::uint64_t mbar_drain[kEvalThreads / 32];  // wind-down after a failure: each warp's MMAs have completed
    unsigned int loads_issued[kStages];  // bulk copies issued on each stage barrier (one per phase)
    std::uint32_t readers[2];            // warps that have read each accumulator buffer (8 per tile)
    std::uint32_t waiters[2];            // warps that have seen each buffer's MMAs complete (8 per tile)
    int task_count;
    int full_count;
    std::uint32_t tmem_base;
    int failed;
};

struct TcParams {
    EvalParams base;
    const std::uint8_t *tables;  // per individual: 256-byte header (emax[64]) + A_pad x 64 16-bit values
    std::size_t table_pitch;
    float kappa;
    int fp16_operands;
    unsigned long long *tc_counters;  // [0] re-scored chunks, [1] games re-scored over every action
    std::uint32_t wait_limit;         // polls of a bounded mbarrier wait before it gives up (NWG_TIMEOUT)
};

// Failure protocol: a wait that gives up (q.wait_limit polls, or earlier once another thread has recorded a failure)
// marks its thread dead (`alive`) and the CTA failed; a dead thread issues nothing and no copy or MMA is issued once
// the CTA has failed, so every barrier phase still gets exactly one copy or commit, and the kernel's wind-down waits
// for the copies issued on each barrier (counted) and for every issuing warp's MMAs.
template <bool kFp16>
__device__ __forceinline__ void ScoreTensorCores(const TcParams &q, ChunkState &cs, TcState &ts, const __half *gh,
                                                 float *arena, int t, std::uint32_t &load_phase,
                                                 std::uint32_t &acc_phase, bool &alive) {
    const EvalParams &p = q.base;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const float *pv = arena;
    unsigned char *a_tile = reinterpret_cast<unsigned char *>(arena + kOffA);
    unsigned char *b_tile = reinterpret_cast<unsigned char *>(arena + kOffB);
    float *cand_v = arena + kOffCand;
    int *cand_id = reinterpret_cast<int *>(arena + kOffCand + kChunkGames * 2 * kTopK);
    std::uint32_t *task_list = reinterpret_cast<std::uint32_t *>(arena + kOffTask);
    unsigned long long *best_key = reinterpret_cast<unsigned long long *>(arena + kOffKeys);
    float *window_low = arena + kOffWindow;
    int *full_rows = reinterpret_cast<int *>(arena + kOffFull);
    const std::uint32_t ind = static_cast<std::uint32_t>(cs.individual);
    const std::uint8_t *table = q.tables + static_cast<std::size_t>(ind) * q.table_pitch;
    const float *emax = reinterpret_cast<const float *>(table);
    const std::uint8_t *embed = table + 256;
    const int n_tiles = static_cast<int>((p.action_count + kTileN - 1) / kTileN);

    const std::uint32_t idesc = kFp16 ? (umma::InstrDescBf16(128, kTileN) & ~((7u << 7) | (7u << 10)))
                                      : umma::InstrDescBf16(128, kTileN);
    const std::uint64_t a_desc0 = umma::SmemDescriptor(umma::SmemAddress(a_tile), 128, 1024);
    const std::uint32_t b_addr0 = umma::SmemAddress(b_tile);
    auto failed_now = [&]() { return *reinterpret_cast<volatile int *>(&ts.failed) != 0; };
    auto can_issue = [&]() { return alive && !failed_now(); };
    auto wait_bar = [&](std::uint64_t *bar, std::uint32_t parity) -> bool {
        if (alive && umma::MbarTest(bar, parity)) {
            return true;
        }
        if (alive && !failed_now() && umma::MbarWaitOrStop(bar, parity, q.wait_limit, &ts.failed)) {
            return true;
        }
        *reinterpret_cast<volatile int *>(&ts.failed) = 1;
        alive = false;
        return false;
    };
    auto issue_load = [&](int stage, int tile) {  // the issuing thread
        if (can_issue()) {
            BulkLoad(b_tile + stage * kTileBytes, embed + static_cast<std::size_t>(tile) * kTileBytes, kTileBytes,
                     &ts.mbar_load[stage]);
            atomicAdd(&ts.loads_issued[stage], 1u);
        }
    };
    // accumulator buffer: tile & 1; embedding stage: tile % kStages
    auto issue_mma = [&](int tile) {  // the issuing thread, once tile's stage has landed
        if (!can_issue()) {
            return;
        }
        const int acc = tile & 1;
        const int stage = tile % kStages;
        const std::uint32_t d = ts.tmem_base + static_cast<std::uint32_t>(acc * kTileN);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const std::uint64_t ad = a_desc0 + static_cast<std::uint64_t>((s * 256) >> 4);
            const std::uint64_t bd = umma::SmemDescriptor(b_addr0 + stage * kTileBytes + s * 256, 128, 1024);
            umma::Mma(d, ad, bd, idesc, s > 0);
        }
        umma::Commit(&ts.mbar_mma[acc]);
    };
    auto wait_stage_and_issue = [&](int tile) {
        const int stage = tile % kStages;
        if (wait_bar(&ts.mbar_load[stage], (load_phase >> stage) & 1u)) {
            umma::FenceAfterSync();
            issue_mma(tile);
        }
    };
    // The first embedding tiles stream in while the 16-bit policy operand is built: the stages are free (the trunk's
    // last reads of this memory ended before its final barrier).
    if (tid == 0) {
        umma::FenceProxyAsyncShared();
        for (int tile = 0; tile < kStages && tile < n_tiles; ++tile) {
            issue_load(tile, tile);
        }
    }

    // 16-bit policy operand, K-major tile [128 games][64]
    for (int idx = tid; idx < kChunkGames * kPolicy; idx += kEvalThreads) {
        const int g = idx & 127;
        const int k = idx >> 7;
        const float v = pv[k * kLd + g];
        std::uint16_t bits;
        if constexpr (kFp16) {
            bits = __half_as_ushort(__float2half_rn(v));
        } else {
            bits = __bfloat16_as_ushort(__float2bfloat16_rn(v));
        }
        *reinterpret_cast<std::uint16_t *>(a_tile + umma::TileOffset(g, k, kPolicy)) = bits;
    }
    if (tid == 0) {
        ts.task_count = 0;
        ts.full_count = 0;
    }
    umma::FenceProxyAsyncShared();
    __syncthreads();

    // No block barrier inside the tile loop. Thread 0 issues tiles 0 and 1; after that, the first warp to see tile
    // k's MMAs complete (an arrival counter per buffer) refills tile k's embedding stage with tile k + kStages, and
    // the last warp to read tile k's accumulator buffer (a second counter) issues tile k + 2 into the buffer it has
    // just released, while the other warps read the other buffer. The stage parities advance alike in every thread,
    // tile by tile.
    for (int tile = 0; tile < 2 && tile < n_tiles; ++tile) {
        if (tid == 0) {
            wait_stage_and_issue(tile);
        }
        load_phase ^= 1u << (tile % kStages);
    }
    const int quadrant = warp & 3;
    const int half = warp >> 2;
    const int row = quadrant * 32 + lane;
    float tv[kTopK];
    int ti[kTopK];
#pragma unroll
    for (int j = 0; j < kTopK; ++j) {
        tv[j] = -INFINITY;
        ti[j] = -1;
    }
    for (int tile = 0; tile < n_tiles; ++tile) {
        const int buf = tile & 1;
        const bool acc_ok = wait_bar(&ts.mbar_mma[buf], (acc_phase >> buf) & 1u);
        acc_phase ^= 1u << buf;
        umma::FenceAfterSync();
        __syncwarp();
        {
            float v[64];
            umma::Load64(ts.tmem_base + static_cast<std::uint32_t>(buf * kTileN + half * 64) +
                             (static_cast<std::uint32_t>(quadrant * 32) << 16),
                         v);
            if (lane == 0) {
                // the first warp to see tile's MMAs complete refills its embedding stage, a whole epilogue earlier
                // than the buffer's last reader could
                const std::uint32_t prior = atomicAdd(&ts.waiters[buf], 1u);
                if ((prior & 7u) == 0u && acc_ok && tile + kStages < n_tiles) {
                    issue_load(tile % kStages, tile + kStages);
                }
            }
            if (tile + 1 == n_tiles) {
#pragma unroll
                for (int j = 0; j < 64; ++j) {
                    if (static_cast<std::uint32_t>(tile * kTileN + half * 64 + j) >= p.action_count) {
                        v[j] = -INFINITY;
                    }
                }
            }
            const float m0 = Max32(v, 0);
            const float m1 = Max32(v, 32);
            InsertTop4(tv, ti, m0, tile * 4 + half * 2);
            InsertTop4(tv, ti, m1, tile * 4 + half * 2 + 1);
        }
        umma::FenceBeforeSync();
        __syncwarp();
        if (lane == 0) {
            // one acquire-release add: releases this warp's reads, and the last reader acquires the others'
            std::uint32_t prior = 0;
            asm volatile("atom.acq_rel.cta.shared::cta.add.u32 %0, [%1], %2;"
                         : "=r"(prior)
                         : "r"(umma::SmemAddress(&ts.readers[buf])), "r"(1u)
                         : "memory");
            if ((prior & 7u) == 7u && acc_ok && tile + 2 < n_tiles) {  // every warp has read tile's buffer
                wait_stage_and_issue(tile + 2);
            }
        }
        if (tile + 2 < n_tiles) {
            load_phase ^= 1u << ((tile + 2) % kStages);
        }
    }
#pragma unroll
    for (int j = 0; j < kTopK; ++j) {
        cand_v[(row * 2 + half) * kTopK + j] = tv[j];
        cand_id[(row * 2 + half) * kTopK + j] = ti[j];
    }
    if (tid < kChunkGames) {
        best_key[tid] = 0;
    }
    __syncthreads();

    if constexpr (kFp16) {
        float *pv_rows = arena + kOffPvRows;
        for (int idx = tid; idx < kChunkGames * kPolicy; idx += kEvalThreads) {
            pv_rows[idx] = pv[(idx & (kPolicy - 1)) * kLd + (idx >> 6)];  // game idx / 64, value idx % 64
        }
    }

    // ---- candidate chunks per game ----
    const int turns_now = t;
    if (tid < kChunkGames && !cs.done[tid]) {
        const int g = tid;
        int masked_chunk[kMaxTurns];
        for (int u = 0; u < kMaxTurns; ++u) {
            masked_chunk[u] = (u < turns_now && cs.word_index[u][g] >= 0) ? cs.word_index[u][g] / 32 : -1;
        }
        auto is_masked_chunk = [&](int chunk) {
            bool m = false;
            for (int u = 0; u < kMaxTurns; ++u) {
                m |= masked_chunk[u] == chunk;
            }
            return m;
        };
        float s_sum = 0.0f;
        float s_dev = 0.0f;
        bool finite = true;
        for (int k = 0; k < kPolicy; ++k) {
            const float pk = pv[k * kLd + g];
            finite &= fabsf(pk) < (kFp16 ? 60000.0f : 3.0e38f);
            s_sum = __fmaf_rn(fabsf(pk), emax[k], s_sum);
            if constexpr (kFp16) {
                // the operand's own rounding error: p and its FP16 value are within a factor of two of each
                // other (or the FP16 value is 0), so the difference is exact
                s_dev = __fmaf_rn(fabsf(__half2float(__float2half_rn(pk)) - pk), emax[k], s_dev);
            }
        }
        // |tensor-core score - FP32 score| <= sum_k |p~_k - p_k| |e_ak| + both 64-term FP32 accumulations. FP16 operands
        // hold every embedding exactly, so the first term is s_dev (the actual rounding of this game's policy) and
        // the accumulations are covered by 2e-5 sum_k |p_k| max_a |e_ak| (64 x 2^-23 = 7.6e-6 each, tensor core
        // and FP32 chain). BF16 operands also round the embeddings: kappa bounds both roundings relative to |p||e|.
        const float eps = kFp16 ? (s_dev + 2.0e-5f * s_sum) * 1.0001f : q.kappa * s_sum * 1.0001f;
        bool full = !finite || !(eps < INFINITY);
        float top = -INFINITY;
        for (int h = 0; h < 2; ++h) {
            bool found = false;
            for (int j = 0; j < kTopK && !found; ++j) {
                const int id = cand_id[(g * 2 + h) * kTopK + j];
                if (id >= 0 && !is_masked_chunk(id)) {
                    top = fmaxf(top, cand_v[(g * 2 + h) * kTopK + j]);
                    found = true;
                }
            }
            if (!found && cand_id[(g * 2 + h) * kTopK + kTopK - 1] >= 0) {
                full = true;  // every tracked chunk of this half holds a guessed word
            }
        }
        const float window = top - 2.0f * eps;
        if (!(top > -INFINITY)) {
            full = true;
        }
        for (int h = 0; h < 2 && !full; ++h) {
            const int last_id = cand_id[(g * 2 + h) * kTopK + kTopK - 1];
            if (last_id >= 0 && cand_v[(g * 2 + h) * kTopK + kTopK - 1] >= window) {
                full = true;  // more chunks of this half may reach the window
            }
        }
        window_low[g] = top - eps;
        if (full) {
            const int slot = atomicAdd(&ts.full_count, 1);
            full_rows[slot] = g;
        } else {
            for (int h = 0; h < 2; ++h) {
                for (int j = 0; j < kTopK; ++j) {
                    const int id = cand_id[(g * 2 + h) * kTopK + j];
                    if (id >= 0 && cand_v[(g * 2 + h) * kTopK + j] >= window && !is_masked_chunk(id)) {
                        const int slot = atomicAdd(&ts.task_count, 1);
                        if (slot < kMaxTasks) {
                            task_list[slot] = (static_cast<std::uint32_t>(g) << 16) | static_cast<std::uint32_t>(id);
                        }
                    }
                }
            }
            // A chunk holding a guessed word matters only when its maximum reaches the window: tracked chunks
            // are compared directly; an untracked chunk lies below the tracked list's last entry, which
            // (no overflow) is below the window.
            for (int h = 0; h < 2; ++h) {
                for (int j = 0; j < kTopK; ++j) {
                    const int id = cand_id[(g * 2 + h) * kTopK + j];
                    if (id >= 0 && cand_v[(g * 2 + h) * kTopK + j] >= window && is_masked_chunk(id)) {
                        const int slot = atomicAdd(&ts.task_count, 1);
                        if (slot < kMaxTasks) {
                            task_list[slot] = (static_cast<std::uint32_t>(g) << 16) | static_cast<std::uint32_t>(id);
                        }
                    }
                }
            }
        }
    }
    __syncthreads();

    // ---- exact re-scoring of the candidate chunks (a warp per chunk) ----
    const __half *tail = reinterpret_cast<const __half *>(reinterpret_cast<const std::uint8_t *>(gh) + kTailOffsetBytes);
    const int tasks = ts.task_count < kMaxTasks ? ts.task_count : kMaxTasks;
    const int first_full = ts.full_count;
    constexpr int kWarps = kEvalThreads / 32;
    if constexpr (kFp16) {
        // the FP16 table holds every embedding value exactly: two tasks per warp in flight
        for (int k0 = warp; k0 < tasks; k0 += 2 * kWarps) {
            const int k1 = k0 + kWarps;
            const std::uint32_t task0 = task_list[k0];
            const std::uint32_t task1 = k1 < tasks ? task_list[k1] : task0;
            const int g0 = static_cast<int>(task0 >> 16);
            const int g1 = static_cast<int>(task1 >> 16);
            unsigned long long key0 = 0;
            unsigned long long key1 = 0;
            const float *pv_rows = arena + kOffPvRows;
            ChunkKeyPairFp16<1>(p, cs, embed, pv_rows + g0 * kPolicy, g0, static_cast<int>(task0 & 0xFFFFu),
                                pv_rows + g1 * kPolicy, g1, static_cast<int>(task1 & 0xFFFFu), turns_now, key0, key1);
            FoldKeys(best_key + g0, key0);
            if (k1 < tasks) {
                FoldKeys(best_key + g1, key1);
            }
        }
    } else {
        for (int k = warp; k < tasks; k += kWarps) {
            const std::uint32_t task = task_list[k];
            const int tg = static_cast<int>(task >> 16);
            RescoreChunk(p, cs, best_key + tg, pv + tg, kLd, tail, tg, static_cast<int>(task & 0xFFFFu), turns_now);
        }
    }
    __syncthreads();
    // a game whose exact best stays below top - eps, or whose task list overflowed, is re-scored in full
    if (tid < kChunkGames && !cs.done[tid]) {
        const int g = tid;
        const unsigned long long key = best_key[g];
        bool in_full = false;
        for (int i = 0; i < first_full; ++i) {
            in_full |= full_rows[i] == g;
        }
        if (!in_full && (ts.task_count > kMaxTasks || key == 0 ||
                         FromOrderedBits(static_cast<std::uint32_t>(key >> 32)) < window_low[g])) {
            const int slot = atomicAdd(&ts.full_count, 1);
            full_rows[slot] = g;
        }
    }
    __syncthreads();
    const int full_count = ts.full_count;
    const int chunks_per_row = static_cast<int>((p.action_count + 31) / 32);
    for (int i = 0; i < full_count; ++i) {
        const int g = full_rows[i];
        if constexpr (kFp16) {
            // each lane keeps its best key over the warp's chunks, two chunks in flight; one fold per warp
            unsigned long long best = 0;
            for (int c0 = warp; c0 < chunks_per_row; c0 += 2 * kWarps) {
                const int c1 = c0 + kWarps;
                unsigned long long key0 = 0;
                unsigned long long key1 = 0;
                const float *row = arena + kOffPvRows + g * kPolicy;
                ChunkKeyPairFp16<1>(p, cs, embed, row, g, c0, row, g, c1 < chunks_per_row ? c1 : c0, turns_now, key0,
                                    key1);
                best = key0 > best ? key0 : best;
                best = c1 < chunks_per_row && key1 > best ? key1 : best;
            }
            FoldKeys(best_key + g, best);
        } else {
            for (int chunk = warp; chunk < chunks_per_row; chunk += kWarps) {
                RescoreChunk(p, cs, best_key + g, pv + g, kLd, tail, g, chunk, turns_now);
            }
        }
    }
    __syncthreads();
    if (tid < kChunkGames) {
        const unsigned long long key = best_key[tid];
        cs.best[tid] = key == 0 ? -1 : static_cast<int>(0xFFFFFFFFu - static_cast<std::uint32_t>(key & 0xFFFFFFFFull));
    }
    if (tid == 0 && q.tc_counters != nullptr) {
        atomicAdd(q.tc_counters, static_cast<unsigned long long>(tasks));
        atomicAdd(q.tc_counters + 1, static_cast<unsigned long long>(full_count));
    }
    __syncthreads();
}

// kStreamed: the FP32 encoder and trunk stream their weights from the exact trunk tables (q.base.xt).
template <bool kFp16, bool kStreamed>
__global__ void __launch_bounds__(kEvalThreads, 2) EvalTcKernel(const TcParams q) {
    extern __shared__ __align__(1024) float arena[];
    __shared__ ChunkState cs;
    __shared__ TcState ts;
    const EvalParams &p = q.base;
    const int tid = threadIdx.x;
    float *scratch = p.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats;
    unsigned long long decisions = 0;
    unsigned long long encoded = 0;
    unsigned long long episodes = 0;
    // parity of the next wait on each stage barrier (bit per stage) and accumulator barrier (bit per buffer); every
    // thread advances them alike, tile by tile
    std::uint32_t load_phase = 0;
    std::uint32_t acc_phase = 0;
    bool alive = true;
    const std::uint32_t total_chunks = p.chunk_start[p.population];

    if (tid < 32) {
        umma::Alloc(&ts.tmem_base, kTmemColumns);
    }
    if (tid == 0) {
        for (int b = 0; b < kStages; ++b) {
            umma::MbarInit(&ts.mbar_load[b], 1);
        }
        for (int b = 0; b < 2; ++b) {
            umma::MbarInit(&ts.mbar_mma[b], 1);
        }
        for (int w = 0; w < kEvalThreads / 32; ++w) {
            umma::MbarInit(&ts.mbar_drain[w], 1);
        }
        for (int b = 0; b < kStages; ++b) {
            ts.loads_issued[b] = 0;
        }
        ts.readers[0] = 0;
        ts.readers[1] = 0;
        ts.waiters[0] = 0;
        ts.waiters[1] = 0;
        ts.failed = 0;
    }
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();

    for (std::uint32_t chunk = blockIdx.x; chunk < total_chunks; chunk += gridDim.x) {
        if (!BeginChunk(p, cs, chunk) || ts.failed) {
            break;
        }
        const std::uint32_t ind = static_cast<std::uint32_t>(cs.individual);
        const __half *gh = reinterpret_cast<const __half *>(p.slab + static_cast<std::size_t>(cs.slot) * p.pitch);
        const std::uint8_t *xt = kStreamed ? p.xt + static_cast<std::size_t>(ind) * p.xt_pitch : nullptr;
        auto encode = [&](int u) {
            if constexpr (kStreamed) {
                EncodeRoundX(cs, gh, xt, arena, scratch, u);
            } else {
                EncodeRound(cs, gh, arena, scratch, u);
            }
        };
        SetupGames(p, cs, gh, scratch);
        if (cs.cls == 1 && CountActive(cs) > 0) {
            encode(0);
            encode(1);
            encoded += tid == 0 ? 2ull * cs.active : 0ull;
        }
        for (int step = 0; step < kMaxTurns; ++step) {
            if (CountActive(cs) == 0 || ts.failed) {
                break;
            }
            const int t = cs.cls == 0 ? step : step + 2;
            if (step > 0) {
                encode(t - 1);
                encoded += tid == 0 ? static_cast<unsigned long long>(cs.active) : 0ull;
            }
            if constexpr (kStreamed) {
                TrunkForwardX(p, cs, gh, xt, arena, scratch, t, step, ind);
            } else {
                TrunkForward(p, cs, gh, arena, scratch, t, step, ind);
            }
            ScoreTensorCores<kFp16>(q, cs, ts, gh, arena, t, load_phase, acc_phase, alive);
            if (ts.failed) {
                break;
            }
            AppendGuesses(p, cs, step, decisions);
        }
        FinishChunk(p, cs, ind, episodes);
    }
    FlushCounters(p, decisions, encoded, episodes);
    __syncthreads();
    if (ts.failed) {  // read after the barrier: uniform
        // every warp's MMAs (a commit tracks all of its thread's earlier tensor-core operations; lane 0 of each warp
        // is the only issuer in it), then the last copy issued on each stage barrier (the n-th copy completes phase
        // n - 1), before the columns and the CTA are released
        const int warp = tid >> 5;
        if ((tid & 31) == 0) {
            umma::Commit(&ts.mbar_drain[warp]);
            (void)umma::MbarWait(&ts.mbar_drain[warp], 0, kDrainLimit);
        }
        if (tid == 0) {
            SetStatus(p.status, kTimeout);
            for (int b = 0; b < kStages; ++b) {
                const unsigned int n = ts.loads_issued[b];
                if (n != 0) {
                    (void)umma::MbarWait(&ts.mbar_load[b], (n - 1u) & 1u, kDrainLimit);
                }
            }
        }
    }
    umma::FenceBeforeSync();
    __syncthreads();
    if (tid < 32) {
        umma::Dealloc(ts.tmem_base, kTmemColumns);
    }
}

// Per individual: emax[k] = max over the selectable actions of |e_ak| (header), the embeddings as 16-bit
// values in the K-major core-matrix layout, 1 KB per 8 actions, zero past the last action, and after the
// last tile, per tile, the column moments (sum_a e_ak, sum_a e_ak^2) over the tile's actions as float2[64].
// One CTA per individual walks its tiles. Thread (a, part) builds action a's four 16-byte segments of columns
// 32 part .. 32 part + 31 (the fixed features from the catalog, the tail from the genome); each warp's stores
// fill whole 128-byte lines. The values also go to shared memory ([action][65], conflict-free both ways), where
// thread (column, quarter) sums its quarter of the tile's actions (values and their squares, each operation
// rounded on its own) in ascending order; the quarters are then combined in a fixed order, so every run gets the
// same bits. kMoments false (the scoring form, which reads no moments) skips them: each thread keeps the maxima of
// its 32 columns in registers, and a warp and then the CTA reduce them once at the end (a maximum is order-free).
template <bool kFp16, bool kMoments>
__global__ void __launch_bounds__(256, kMoments ? 4 : 3) BuildTcTablesKernel(const std::uint8_t *slab, std::size_t pitch,
                                                           const std::uint32_t *slots, const float *fixed_t,
                                                           std::uint32_t action_pad, std::uint32_t action_count,
                                                           std::uint32_t tiles, std::uint8_t *tables,
                                                           std::size_t table_pitch) {
    constexpr int kLd = kPolicy + 1;
    __shared__ float vals[kMoments ? kTileN * kLd : 1];
    __shared__ float2 part_sum[4][kPolicy];
    __shared__ float part_max[4][kPolicy];
    const std::uint32_t ind = blockIdx.x;
    const std::uint8_t *tail = slab + static_cast<std::size_t>(slots[ind]) * pitch + kTailOffsetBytes;
    std::uint8_t *table = tables + static_cast<std::size_t>(ind) * table_pitch;
    float2 *moments = reinterpret_cast<float2 *>(table + 256 + static_cast<std::size_t>(tiles) * kTileBytes);
    const int t = static_cast<int>(threadIdx.x);
    const int a_local = t & (kTileN - 1);
    const int part = t >> 7;     // columns 32 part .. 32 part + 31
    const int col = t & (kPolicy - 1);
    const int quarter = t >> 6;  // actions 32 quarter .. 32 quarter + 31 of the tile
    float run_max = 0.0f;
    float col_max[32];  // without moments: this thread's columns 32 part + j over its actions
#pragma unroll
    for (int j = 0; j < 32; ++j) {
        col_max[j] = 0.0f;
    }
    for (std::uint32_t tile = 0; tile < tiles; ++tile) {
        const std::uint32_t a = tile * kTileN + static_cast<std::uint32_t>(a_local);
        const bool valid = a < action_count;
        const std::uint32_t *row =
            reinterpret_cast<const std::uint32_t *>(tail + static_cast<std::size_t>(valid ? a : 0u) * kTailRowBytes);
        float v[32];
        if (part == 0) {
#pragma unroll
            for (int k = 0; k < kFixedDim; ++k) {
                v[k] = valid ? __ldg(fixed_t + static_cast<std::size_t>(k) * action_pad + a) : 0.0f;
            }
#pragma unroll
            for (int i = 0; i < 3; ++i) {  // tail values 0 .. 5 (columns 26 .. 31)
                const std::uint32_t w = valid ? __ldg(row + i) : 0u;
                const __half2 h = *reinterpret_cast<const __half2 *>(&w);
                v[kFixedDim + 2 * i] = __low2float(h);
                v[kFixedDim + 2 * i + 1] = __high2float(h);
            }
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) {  // tail values 6 .. 37 (columns 32 .. 63)
                const std::uint32_t w = valid ? __ldg(row + 3 + i) : 0u;
                const __half2 h = *reinterpret_cast<const __half2 *>(&w);
                v[2 * i] = __low2float(h);
                v[2 * i + 1] = __high2float(h);
            }
        }
        std::uint8_t *out = table + 256 + static_cast<std::size_t>(tile) * kTileBytes;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            std::uint32_t w[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float x = v[8 * s + 2 * i];
                const float y = v[8 * s + 2 * i + 1];
                if constexpr (kFp16) {
                    w[i] = static_cast<std::uint32_t>(__half_as_ushort(__float2half_rn(x))) |
                           (static_cast<std::uint32_t>(__half_as_ushort(__float2half_rn(y))) << 16);
                } else {
                    w[i] = static_cast<std::uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(x))) |
                           (static_cast<std::uint32_t>(__bfloat16_as_ushort(__float2bfloat16_rn(y))) << 16);
                }
            }
            *reinterpret_cast<uint4 *>(out + umma::TileOffset(a_local, part * 32 + 8 * s, kPolicy)) =
                make_uint4(w[0], w[1], w[2], w[3]);
        }
        if constexpr (!kMoments) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                col_max[j] = fmaxf(col_max[j], fabsf(v[j]));
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                vals[a_local * kLd + part * 32 + j] = v[j];
            }
            __syncthreads();
            float sum = 0.0f;
            float sum_sq = 0.0f;
            for (int i = 0; i < 32; ++i) {
                const float x = vals[(quarter * 32 + i) * kLd + col];
                sum = __fadd_rn(sum, x);
                sum_sq = __fadd_rn(sum_sq, __fmul_rn(x, x));
                run_max = fmaxf(run_max, fabsf(x));
            }
            part_sum[quarter][col] = make_float2(sum, sum_sq);
            __syncthreads();
            if (t < kPolicy) {
                moments[tile * kPolicy + t] =
                    make_float2(((part_sum[0][t].x + part_sum[1][t].x) + part_sum[2][t].x) + part_sum[3][t].x,
                                ((part_sum[0][t].y + part_sum[1][t].y) + part_sum[2][t].y) + part_sum[3][t].y);
            }
        }
    }
    if constexpr (!kMoments) {
        // warp maxima of each column (the warp's 32 actions share `part`), then the four warps of each part
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            float m = col_max[j];
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, d));
            }
            col_max[j] = m;
        }
        const int w = (t >> 5) & 3;  // the warp within its part
        if ((t & 31) == 0) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                part_max[w][part * 32 + j] = col_max[j];
            }
        }
    } else {
        part_max[quarter][col] = run_max;
    }
    __syncthreads();
    if (t < kPolicy) {
        reinterpret_cast<float *>(table)[t] =
            fmaxf(fmaxf(part_max[0][t], part_max[1][t]), fmaxf(part_max[2][t], part_max[3][t]));
    }
}

}  // namespace

std::size_t TcTablePitch(std::uint32_t action_count) {
    const std::size_t tiles = (action_count + kTileN - 1) / kTileN;
    return 256 + tiles * static_cast<std::size_t>(kTileBytes + kPolicy * sizeof(float2));
}

cudaError_t LaunchBuildTcTables(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                std::uint32_t population, const float *fixed_t, std::uint32_t action_pad,
                                std::uint32_t action_count, std::uint8_t *tables, bool fp16, bool with_moments,
                                cudaStream_t stream) {
    if (population == 0) {
        return cudaSuccess;
    }
    const std::size_t table_pitch = TcTablePitch(action_count);
    const std::uint32_t tiles = (action_count + kTileN - 1) / kTileN;
    if (fp16 && with_moments) {
        BuildTcTablesKernel<true, true><<<population, 256, 0, stream>>>(slab, pitch, slots, fixed_t, action_pad,
                                                                        action_count, tiles, tables, table_pitch);
    } else if (fp16) {
        BuildTcTablesKernel<true, false><<<population, 256, 0, stream>>>(slab, pitch, slots, fixed_t, action_pad,
                                                                         action_count, tiles, tables, table_pitch);
    } else if (with_moments) {
        BuildTcTablesKernel<false, true><<<population, 256, 0, stream>>>(slab, pitch, slots, fixed_t, action_pad,
                                                                         action_count, tiles, tables, table_pitch);
    } else {
        BuildTcTablesKernel<false, false><<<population, 256, 0, stream>>>(slab, pitch, slots, fixed_t, action_pad,
                                                                          action_count, tiles, tables, table_pitch);
    }
    return cudaGetLastError();
}

cudaError_t LaunchEvalTc(const EvalParams &params, const std::uint8_t *tables, std::size_t table_pitch, float kappa,
                         bool fp16, unsigned long long *tc_counters, int cta_count, cudaStream_t stream,
                         std::uint32_t wait_limit) {
    const int arena_bytes = kArenaFloats * static_cast<int>(sizeof(float));
    static std::atomic<unsigned long long> configured[4]{{0}, {0}, {0}, {0}};
    const bool streamed = params.xt != nullptr;
    cudaError_t e = cudaSuccess;
    if (fp16) {
        e = streamed ? RaiseSharedLimit(EvalTcKernel<true, true>, arena_bytes, configured[3])
                     : RaiseSharedLimit(EvalTcKernel<true, false>, arena_bytes, configured[1]);
    } else {
        e = streamed ? RaiseSharedLimit(EvalTcKernel<false, true>, arena_bytes, configured[2])
                     : RaiseSharedLimit(EvalTcKernel<false, false>, arena_bytes, configured[0]);
    }
    if (e != cudaSuccess) {
        return e;
    }
    if (cta_count <= 0) {
        return cudaSuccess;
    }
    TcParams q{};
    q.base = params;
    q.tables = tables;
    q.table_pitch = table_pitch;
    q.kappa = kappa;
    q.fp16_operands = fp16 ? 1 : 0;
    q.tc_counters = tc_counters;
    q.wait_limit = wait_limit;
    if (fp16) {
        if (streamed) {
            EvalTcKernel<true, true><<<cta_count, kEvalThreads, arena_bytes, stream>>>(q);
        } else {
            EvalTcKernel<true, false><<<cta_count, kEvalThreads, arena_bytes, stream>>>(q);
        }
    } else if (streamed) {
        EvalTcKernel<false, true><<<cta_count, kEvalThreads, arena_bytes, stream>>>(q);
    } else {
        EvalTcKernel<false, false><<<cta_count, kEvalThreads, arena_bytes, stream>>>(q);
    }
    return cudaGetLastError();
}

}  // namespace nwg
