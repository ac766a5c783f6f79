// Fitness evaluation, tensor-core trunk form: encoder, trunk and action scoring on tcgen05 with 16-bit
// operands (FP16 or BF16) and FP32 accumulation in tensor memory; a margin guard sends every uncertain
// game step through the exact FP32 path.
//
// A CTA of 256 threads owns a chunk of up to 128 games of one individual (the same chunks as the plain
// form). Per game step, with t turns on the board:
//   encoder   the new turn's 145 one-hot features x W_e1 (K = 160), + bias, ReLU, x W_e2 -> 64 values,
//             kept as a 16-bit operand tile in the CTA's global scratch (one 16 KB tile per turn);
//   layer 1   sum over the t turn tiles of enc_u x W1[:, 1 + 64u .. 64 + 64u]^T (N = 256), + bias, ReLU;
//             with no turn on the board every row is relu(b1 + W1[:, 0]);
//   layer 2   (K = 256, N = 128), + bias, ReLU;  layer 3  (K = 128, N = 64), + bias -> policy p~;
//   scoring   p~ (16-bit) against the individual's 16-bit embedding table, 128 actions per MMA tile,
//             keeping per game the four largest 32-action chunk maxima of each half of the columns.
// Decision: the chunks within the guard bound of the best chunk free of guessed words are re-scored on
// CUDA cores from the same 16-bit operands; the guess is the best unguessed action when its margin over
// every other unguessed action is positive and at least tau * spread, where the spread
// sqrt(sum_k p~_k^2 var_a(e_ak)) estimates the standard deviation of the game's scores over the actions
// (the per-column embedding variances come with the embedding table; unlike the best score's magnitude the
// spread ignores a shift common to every action). Otherwise (and whenever the tracked chunks cannot certify
// the margin) the game step
// falls back: its policy is recomputed with the plain form's exact FP32 chains and its guess is the
// exact FP32 argmax, found by re-scoring every chunk that the tensor-core maxima cannot rule out
// (|s~ - s| <= sum_k |p~_k - p_k| max_a |e_ak| + accumulation slack).
// All weight operands come from a per-individual table in the tensor-core layout (BuildTrunkTables);
// every mbarrier wait is bounded and a wait that gives up records NWG_TIMEOUT.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "tc_common.cuh"

namespace nwg {
namespace {

using namespace evalx;
using namespace tcx;

constexpr int kPageBytes = 16384;
constexpr int kPages = 6;
constexpr int kSmemBytes = kPages * kPageBytes;
constexpr int kTileN = 128;
constexpr int kEmbedStages = 5;  // scoring stages live in pages 1..5
constexpr std::uint32_t kTmemColumns = 256;
constexpr std::uint32_t kDrainLimit = 1u << 22;  // polls of each wind-down wait after a failure
constexpr int kKe1 = 160;  // encoder input features (145) padded to a multiple of 16
constexpr int kFallbackBatch = 8;

// Per-individual trunk table (bytes): K-major canonical operand tiles, rows = output neurons.
constexpr int kTblWe1 = 0;                                          // [128][160]
constexpr int kTblWe2 = kTblWe1 + kEncoderHidden * kKe1 * 2;        // [64][128]
constexpr int kTblW1 = kTblWe2 + kEncoderOut * kEncoderHidden * 2;  // 5 x [256][64]
constexpr int kW1SlotBytes = kHidden0 * kEncoderOut * 2;
constexpr int kTblW2 = kTblW1 + 5 * kW1SlotBytes;                   // 4 x [128][64]
constexpr int kW2ChunkBytes = kHidden1 * 64 * 2;
constexpr int kTblW3 = kTblW2 + 4 * kW2ChunkBytes;                  // [64][128]
constexpr int kTrunkTableBytes = kTblW3 + kPolicy * kHidden1 * 2;
static_assert(kTrunkTableBytes == 303104, "trunk table layout");
static_assert(kTrunkTableBytes % (16 * 256) == 0, "table build grid covers whole 16-byte segments");

// Post-scoring shared-memory layout (byte offsets into the page arena; page 0 keeps the policy operand).
constexpr int kOffCandV = 1 * kPageBytes;                            // [128 games][2 halves][4] floats
constexpr int kOffCandId = kOffCandV + kChunkGames * 2 * kTopK * 4;  // ids
constexpr int kOffExcl = kOffCandId + kChunkGames * 2 * kTopK * 4;   // [128] max score outside the candidates
constexpr int kOffTaskOff = kOffExcl + kChunkGames * 4;              // [128] first task of each game
constexpr int kOffTaskCnt = kOffTaskOff + kChunkGames * 4;           // [128] candidate chunks per game
constexpr int kOffFbKey = kOffTaskCnt + kChunkGames * 4;             // [8] exact best keys (u64)
constexpr int kOffFbWin = kOffFbKey + kFallbackBatch * 8;            // [8] exact window low ends
constexpr int kOffFbFull = kOffFbWin + kFallbackBatch * 4;           // [8] full re-score flags
constexpr int kOffFbTasks = kOffFbFull + kFallbackBatch * 4;         // [64] exact tasks (batch game << 16 | chunk)
constexpr int kOffFbCount = kOffFbTasks + kFallbackBatch * 2 * kTopK * 4;
constexpr int kMaxCandTasks = kChunkGames * 2 * kTopK;
constexpr int kOffTasks = 2 * kPageBytes;                   // [1024] (game << 16) | chunk
constexpr int kOffResults = kOffTasks + kMaxCandTasks * 4;  // [1024][2] u64 top-2 keys
static_assert(kOffResults + kMaxCandTasks * 16 <= kSmemBytes, "task buffers");
// exact fallback buffers (reuse the task region once the approximate decisions are made)
constexpr int kOffXEnc = 26624;                                                 // [8][5][64] f32
constexpr int kOffXHid = kOffXEnc + kFallbackBatch * 5 * kEncoderOut * 4;       // [8][5][128] f32
constexpr int kOffXH0 = kOffXHid;                                               // [8][256], once hid is dead
constexpr int kOffXH1 = kOffXH0 + kFallbackBatch * kHidden0 * 4;                // [8][128]
constexpr int kOffXP = kOffXH1 + kFallbackBatch * kHidden1 * 4;                 // [8][64]
constexpr int kOffXStage = kOffXHid + kFallbackBatch * 5 * kEncoderHidden * 4;  // staged encoder weights
static_assert(kOffFbCount + 16 <= kOffXEnc, "decision buffers overlap the fallback buffers");
static_assert(kOffXP + kFallbackBatch * kPolicy * 4 <= kOffXStage, "fallback buffers");
static_assert(kOffXStage + kEncoderHidden * kTurnFeatures * 2 <= kSmemBytes, "staged encoder weights");
static_assert((kEncoderHidden * kTurnFeatures * 2) % 16 == 0, "W_e1 copies as 16-byte words");
constexpr int kStageLd = 66;   // halfs per staged 64-wide weight row (33 words: conflict-free column reads)
constexpr int kStageLd3 = 130; // halfs per staged W3 row (65 words)
static_assert(kOffXStage + kHidden0 * kStageLd * 2 <= kSmemBytes, "staged layer-1 slice");
static_assert(kOffXStage + kPolicy * kStageLd3 * 2 <= kSmemBytes, "staged W3");
// FP16 form: the exact path streams its weights from the trunk table (the genome's FP16 values in K-major
// canonical tiles) through a ring of three 16 KB buffers: page 0 (its 16-bit policy rows saved first) and two
// buffers in the staging area; the saved rows follow them.
constexpr int kRing = 3;
constexpr int kRingTileBytes = 16384;
constexpr int kOffRing1 = kOffXStage;
constexpr int kOffRing2 = kOffRing1 + kRingTileBytes;
constexpr int kOffSavedRows = kOffRing2 + kRingTileBytes;  // [games][64] 16-bit policy values
constexpr int kMaxSavedRows = (kSmemBytes - kOffSavedRows) / (kPolicy * 2);
static_assert(kOffXP + kFallbackBatch * kPolicy * 4 <= kOffRing1, "ring buffers after the fallback activations");
static_assert(kMaxSavedRows >= 64, "saved policy rows");
constexpr int kWe1GroupBytes = 8 * kKe1 * 2;  // 8 rows of W_e1 in the canonical layout

struct TctState {
    std::uint64_t bar_load[kPages];  // bulk loads into page p (at most one outstanding per barrier)
    std::uint64_t bar_free[2];       // trunk operand stages released by completed MMAs
    std::uint64_t bar_mma;           // a trunk phase's MMAs have completed
    std::uint64_t bar_acc[2];        // scoring accumulator buffers: MMAs completed
    std::uint64_t bar_drain[kEvalThreads / 32];  // wind-down after a failure: each warp's MMAs have completed
    std::uint64_t bar_ring[kRing];   // exact-path weight tiles (FP16 form)
    unsigned int loads_issued[kPages];  // bulk copies issued on each page barrier (one per phase)
    unsigned int ring_issued[kRing];
    std::uint32_t tmem_base;
    int failed;
    int n_fallback;
    int scan[4];
    std::uint8_t fallback_games[kChunkGames];  // game rows (< 128)
    float be1[kEncoderHidden];
    float be2[kEncoderOut];
    float b1[kHidden0];
    float b2[kHidden1];
    float b3[kPolicy];
    float virgin[kHidden0];  // relu(b1 + W1[:, 0])
    float emax[kPolicy];
    float var[kPolicy];  // per-column variance of the embeddings over the selectable actions
    float s_part[2][kChunkGames];
    std::uint32_t load_sync;             // thread 0's load phase bits, handed to every thread for the scoring loop
    std::uint32_t readers[2];            // warps that have read each scoring accumulator buffer (8 per tile)
};

struct TctParams {
    EvalParams base;
    const std::uint8_t *embed_tables;  // per individual: 256-byte header (emax[64]) + A_pad x 64 16-bit values
    std::size_t embed_pitch;
    const std::uint8_t *trunk_tables;  // per individual: kTrunkTableBytes
    std::size_t trunk_pitch;
    float tau;
    unsigned long long *counters;  // [0] candidate chunks, [1] fallback steps, [2] exact chunks, [3] exact rows
    std::uint32_t wait_limit;      // polls of a bounded mbarrier wait before it gives up (NWG_TIMEOUT)
};

template <bool kFp16>
__device__ __forceinline__ std::uint32_t Pack2(float a, float b) {
    if constexpr (kFp16) {
        const __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<const std::uint32_t *>(&h);
    } else {
        const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<const std::uint32_t *>(&h);
    }
}

template <bool kFp16>
__device__ __forceinline__ float2 Unpack2(std::uint32_t bits) {
    if constexpr (kFp16) {
        return __half22float2(*reinterpret_cast<const __half2 *>(&bits));
    } else {
        return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&bits));
    }
}

template <bool kFp16>
__device__ __forceinline__ std::uint16_t One16() {
    return kFp16 ? std::uint16_t{0x3C00} : std::uint16_t{0x3F80};
}

template <bool kFp16>
__host__ __device__ constexpr std::uint32_t InstrDesc(int m, int n) {
    return kFp16 ? (umma::InstrDescBf16(m, n) & ~((7u << 7) | (7u << 10))) : umma::InstrDescBf16(m, n);
}

// Stores 32 consecutive FP32 columns c0..c0+31 of row g, rounded to 16 bits, into a K-wide operand tile.
template <bool kFp16>
__device__ __forceinline__ void StoreRow32(std::uint8_t *tile, int g, int c0, int K, const float (&v)[32]) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        uint4 w;
        w.x = Pack2<kFp16>(v[8 * s + 0], v[8 * s + 1]);
        w.y = Pack2<kFp16>(v[8 * s + 2], v[8 * s + 3]);
        w.z = Pack2<kFp16>(v[8 * s + 4], v[8 * s + 5]);
        w.w = Pack2<kFp16>(v[8 * s + 6], v[8 * s + 7]);
        *reinterpret_cast<uint4 *>(tile + umma::TileOffset(g, c0 + 8 * s, K)) = w;
    }
}

// D (+)= A x B^T over K (a multiple of 16), both operands K-major canonical tiles; one thread issues.
__device__ __forceinline__ void MmaK(std::uint32_t d, const std::uint8_t *a, int a_k, const std::uint8_t *b, int b_k,
                                     int k_steps, std::uint32_t idesc, bool accumulate) {
    const std::uint32_t a_addr = umma::SmemAddress(a);
    const std::uint32_t b_addr = umma::SmemAddress(b);
    for (int s = 0; s < k_steps; ++s) {
        const std::uint64_t ad = umma::SmemDescriptor(a_addr + s * 256, 128, (a_k / 8) * 128);
        const std::uint64_t bd = umma::SmemDescriptor(b_addr + s * 256, 128, (b_k / 8) * 128);
        umma::Mma(d, ad, bd, idesc, accumulate || s > 0);
    }
}

// a x b + c with 16-bit factors (FP16 or BF16 bit patterns in the low 16 bits) and an FP32 addend, rounded once.
template <bool kFp16>
__device__ __forceinline__ float Fma16(std::uint32_t a, std::uint32_t b, float c) {
    float d;
    const unsigned short ha = static_cast<unsigned short>(a);
    const unsigned short hb = static_cast<unsigned short>(b);
    if constexpr (kFp16) {
        asm("fma.rn.f32.f16 %0, %1, %2, %3;" : "=f"(d) : "h"(ha), "h"(hb), "f"(c));
    } else {
        asm("fma.rn.f32.bf16 %0, %1, %2, %3;" : "=f"(d) : "h"(ha), "h"(hb), "f"(c));
    }
    return d;
}

// Approximate score (16-bit operands, FP32 accumulation) of an action for game g: the policy row of the
// operand tile against the action's embedding row e.
template <bool kFp16>
__device__ __forceinline__ float ApproxScore(const std::uint8_t *a_tile, int g, const uint4 (&e)[8]) {
    float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int kg = 0; kg < 8; ++kg) {
        const uint4 pw = *reinterpret_cast<const uint4 *>(a_tile + umma::TileOffset(g, kg * 8, kPolicy));
        const std::uint32_t pv[4] = {pw.x, pw.y, pw.z, pw.w};
        const std::uint32_t ev[4] = {e[kg].x, e[kg].y, e[kg].z, e[kg].w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            // both factors 16-bit: the product is formed exactly and added with one rounding, as fmaf does on the
            // converted values, without the conversions
            acc[i] = Fma16<kFp16>(pv[i] & 0xFFFFu, ev[i] & 0xFFFFu, acc[i]);
            acc[i] = Fma16<kFp16>(pv[i] >> 16, ev[i] >> 16, acc[i]);
        }
    }
    return (acc[0] + acc[1]) + (acc[2] + acc[3]);
}

// Copies `rows` rows of `cols` (a multiple of 32) 16-bit values, source row stride src_ld, destination row
// stride dst_ld, into shared memory: a warp per row so that each load instruction reads consecutive halfs,
// with 16 rows' loads issued before any store.
template <int kCols>
__device__ __forceinline__ void StageRows(__half *__restrict__ dst, int dst_ld, const __half *__restrict__ src,
                                          int src_ld, int rows) {
    constexpr int kBatch = 16;
    constexpr int kPer = kCols / 32;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    for (int r0 = warp; r0 < rows; r0 += kBatch * (kEvalThreads / 32)) {
        __half v[kBatch][kPer];
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
            const int r = r0 + i * (kEvalThreads / 32);
#pragma unroll
            for (int c = 0; c < kPer; ++c) {
                v[i][c] = r < rows ? __ldg(src + static_cast<std::size_t>(r) * src_ld + c * 32 + lane)
                                   : __float2half_rn(0.0f);
            }
        }
#pragma unroll
        for (int i = 0; i < kBatch; ++i) {
            const int r = r0 + i * (kEvalThreads / 32);
            if (r < rows) {
#pragma unroll
                for (int c = 0; c < kPer; ++c) {
                    dst[r * dst_ld + c * 32 + lane] = v[i][c];
                }
            }
        }
    }
}

template <bool kFp16>
__global__ void __launch_bounds__(kEvalThreads, 2) EvalTctKernel(const TctParams q) {
    extern __shared__ __align__(1024) std::uint8_t smem[];
    __shared__ ChunkState cs;
    __shared__ TctState ts;
    const EvalParams &p = q.base;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const int lane = tid & 31;
    const int quad = warp & 3;
    const int half = warp >> 2;
    const int row = quad * 32 + lane;  // TMEM lane = game row this thread reads back
    const std::uint32_t lane_bits = static_cast<std::uint32_t>(quad * 32) << 16;
    auto page = [&](int i) { return smem + i * kPageBytes; };
    std::uint8_t *enc_scratch =
        reinterpret_cast<std::uint8_t *>(p.scratch + static_cast<std::size_t>(blockIdx.x) * kScratchFloats);
    unsigned long long decisions = 0, encoded = 0, episodes = 0;
    unsigned long long cand_chunks = 0, fallback_steps = 0, exact_chunks = 0, exact_rows = 0;
    // Barrier bookkeeping as one bit per barrier in registers (each barrier has at most one copy or commit
    // outstanding): the parity of the next wait.
    // thread 0 only: page loads, stage commits mod 2
    std::uint32_t load_phase = 0;
    std::uint32_t free_parity = 0;
    // every thread: ring waits, phase commits, accumulator waits
    std::uint32_t ring_phase = 0;
    std::uint32_t mma_commits = 0;
    std::uint32_t acc_phase = 0;
    const std::uint32_t total_chunks = p.chunk_start[p.population];
    const std::uint32_t idesc128 = InstrDesc<kFp16>(128, 128);
    const std::uint32_t idesc64 = InstrDesc<kFp16>(128, 64);
    const std::uint32_t idesc256 = InstrDesc<kFp16>(128, 256);
    const int n_tiles = static_cast<int>((p.action_count + kTileN - 1) / kTileN);

    if (tid < 32) {
        umma::Alloc(&ts.tmem_base, kTmemColumns);
    }
    if (tid == 0) {
        for (int b = 0; b < kPages; ++b) {
            umma::MbarInit(&ts.bar_load[b], 1);
        }
        umma::MbarInit(&ts.bar_free[0], 1);
        umma::MbarInit(&ts.bar_free[1], 1);
        umma::MbarInit(&ts.bar_mma, 1);
        umma::MbarInit(&ts.bar_acc[0], 1);
        umma::MbarInit(&ts.bar_acc[1], 1);
        ts.readers[0] = 0;
        ts.readers[1] = 0;
        for (int w = 0; w < kEvalThreads / 32; ++w) {
            umma::MbarInit(&ts.bar_drain[w], 1);
        }
        for (int b = 0; b < kRing; ++b) {
            umma::MbarInit(&ts.bar_ring[b], 1);
            ts.ring_issued[b] = 0;
        }
        for (int b = 0; b < kPages; ++b) {
            ts.loads_issued[b] = 0;
        }
        ts.failed = 0;
    }
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    const std::uint32_t tmem = ts.tmem_base;

    // Failure protocol. A wait that gives up (q.wait_limit polls, or earlier once another thread has recorded a
    // failure) marks its thread dead and the CTA failed. From then on the thread issues nothing, and no thread issues
    // anything once it sees the CTA failed: every copy or MMA that is issued follows successful waits of its own
    // thread, so each barrier phase still gets exactly one copy or commit. Threads keep their uniform control flow
    // (results are discarded) until the chunk's next uniform check; the wind-down then waits for the copies issued
    // on each barrier (counted) and for every warp's MMAs before tensor memory is released.
    bool alive = true;
    auto failed_now = [&]() { return *reinterpret_cast<volatile int *>(&ts.failed) != 0; };
    auto can_issue = [&]() { return alive && !failed_now(); };
    auto wait_bar = [&](std::uint64_t *bar, std::uint32_t parity) -> bool {
        // a completed phase is taken at once; the failure flag is read only for a phase still open
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
    auto issue_load = [&](int b, void *dst, const void *src, std::uint32_t bytes) {  // any issuing thread
        if (can_issue()) {
            BulkLoad(dst, src, bytes, &ts.bar_load[b]);
            atomicAdd(&ts.loads_issued[b], 1u);
        }
    };
    // thread 0 only
    auto load = [&](int b, void *dst, const void *src, std::uint32_t bytes) { issue_load(b, dst, src, bytes); };
    auto wait_load = [&](int b) -> bool {
        const bool ok = wait_bar(&ts.bar_load[b], (load_phase >> b) & 1u);
        load_phase ^= 1u << b;
        return ok;
    };
    auto commit_free = [&](int s) {
        if (can_issue()) {
            umma::Commit(&ts.bar_free[s]);
        }
        free_parity ^= 1u << s;
    };
    auto wait_free = [&](int s) { return wait_bar(&ts.bar_free[s], ((free_parity >> s) & 1u) ^ 1u); };
    // every thread (uniform control flow)
    auto commit_mma = [&]() {
        if (tid == 0 && can_issue()) {
            umma::Commit(&ts.bar_mma);
        }
        ++mma_commits;
    };
    auto wait_mma = [&]() {
        wait_bar(&ts.bar_mma, (mma_commits - 1u) & 1u);
        umma::FenceAfterSync();
    };
    auto phase_sync = [&]() {  // generic smem writes -> visible to the tensor core; TMEM reads ordered
        umma::FenceProxyAsyncShared();
        umma::FenceBeforeSync();
        __syncthreads();
        umma::FenceAfterSync();
    };

    for (std::uint32_t chunk = blockIdx.x; chunk < total_chunks; chunk += gridDim.x) {
        if (!BeginChunk(p, cs, chunk) || ts.failed) {
            break;
        }
        const std::uint32_t ind = static_cast<std::uint32_t>(cs.individual);
        const __half *gh = reinterpret_cast<const __half *>(p.slab + static_cast<std::size_t>(cs.slot) * p.pitch);
        const std::uint8_t *ttab = q.trunk_tables + static_cast<std::size_t>(ind) * q.trunk_pitch;
        const std::uint8_t *etab = q.embed_tables + static_cast<std::size_t>(ind) * q.embed_pitch;
        const std::uint8_t *embed = etab + 256;
        SetupGames(p, cs, gh, nullptr);
        for (int i = tid; i < kHidden0; i += kEvalThreads) {
            const float b = H2F(gh, kTrB1 + i);
            ts.b1[i] = b;
            const float v = __fmaf_rn(H2F(gh, kTrW1 + i * kModelInput), 1.0f, b);
            ts.virgin[i] = v < 0.0f ? 0.0f : v;
            if (i < kEncoderHidden) {
                ts.be1[i] = H2F(gh, kEncB1 + i);
                ts.b2[i] = H2F(gh, kTrB2 + i);
            }
            if (i < kPolicy) {
                ts.be2[i] = H2F(gh, kEncB2 + i);
                ts.b3[i] = H2F(gh, kTrB3 + i);
                ts.emax[i] = reinterpret_cast<const float *>(etab)[i];
                const float2 *moments = reinterpret_cast<const float2 *>(embed + static_cast<std::size_t>(n_tiles) *
                                                                                     kPageBytes);
                float sum = 0.0f;
                float sum_sq = 0.0f;
                for (int tile = 0; tile < n_tiles; ++tile) {
                    const float2 m = moments[tile * kPolicy + i];
                    sum += m.x;
                    sum_sq += m.y;
                }
                const float mean = sum / static_cast<float>(p.action_count);
                ts.var[i] = fmaxf(sum_sq / static_cast<float>(p.action_count) - mean * mean, 0.0f);
            }
        }
        __syncthreads();

        // ---- encoder: turn u of every game -> 16-bit tile in page 2 and in the CTA's scratch slot u ----
        auto encode_turn = [&](int u) {
            std::uint8_t *onehot = page(0);                // [128][160], 40 KB
            std::uint8_t *we1 = page(0) + 128 * kKe1 * 2;  // [128][160], 40 KB (pages 2.5 .. 5)
            std::uint8_t *a_h = page(0);                   // [128][128] hidden operand, after the first MMA
            std::uint8_t *enc = page(2);                   // [128][64]
            if (tid == 0) {
                umma::FenceProxyAsyncShared();
                load(2, we1, ttab + kTblWe1, 128 * kKe1 * 2);
                load(5, page(5), ttab + kTblWe2, kEncoderOut * kEncoderHidden * 2);
            }
            for (int i = tid; i < 128 * kKe1 * 2 / 16; i += kEvalThreads) {
                reinterpret_cast<uint4 *>(onehot)[i] = make_uint4(0, 0, 0, 0);
            }
            __syncthreads();
            for (int i = tid; i < kChunkGames * 10; i += kEvalThreads) {
                const int g = i / 10;
                const int f = i - g * 10;
                const std::uint32_t code = cs.guess[u][g];
                const std::uint32_t tiles = cs.tiles[u][g];
                const int feature = f < kWordLength ? f * kAlphabet + static_cast<int>(WordLetter(code, f))
                                                    : kWordLength * kAlphabet + (f - kWordLength) * 3 +
                                                          static_cast<int>((tiles >> (2 * (f - kWordLength))) & 3u);
                *reinterpret_cast<std::uint16_t *>(onehot + umma::TileOffset(g, feature, kKe1)) = One16<kFp16>();
            }
            phase_sync();
            if (tid == 0 && wait_load(2) && can_issue()) {
                umma::FenceAfterSync();
                MmaK(tmem, onehot, kKe1, we1, kKe1, kKe1 / 16, idesc128, false);
            }
            commit_mma();
            wait_mma();
            {
                float v[32];
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int c0 = half * 64 + j * 32;
                    umma::Load32(tmem + static_cast<std::uint32_t>(c0) + lane_bits, v);
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const float h = v[i] + ts.be1[c0 + i];
                        v[i] = h < 0.0f ? 0.0f : h;
                    }
                    StoreRow32<kFp16>(a_h, row, c0, kEncoderHidden, v);
                }
            }
            phase_sync();
            if (tid == 0 && wait_load(5) && can_issue()) {
                umma::FenceAfterSync();
                MmaK(tmem + 128, a_h, kEncoderHidden, page(5), kEncoderHidden, kEncoderHidden / 16, idesc64, false);
            }
            commit_mma();
            wait_mma();
            {
                float v[32];
                const int c0 = half * 32;
                umma::Load32(tmem + 128u + static_cast<std::uint32_t>(c0) + lane_bits, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    v[i] += ts.be2[c0 + i];
                }
                StoreRow32<kFp16>(enc, row, c0, kEncoderOut, v);
                StoreRow32<kFp16>(enc_scratch + u * kPageBytes, row, c0, kEncoderOut, v);
            }
            asm volatile("fence.proxy.async.global;" ::: "memory");
            phase_sync();
        };

        // ---- trunk at turn count t: leaves the 16-bit policy operand in page 0 ----
        // ---- trunk at turn count t: leaves the 16-bit policy operand in page 0 ----
        // Layer 1's 16-bit activations h0 stay in tensor memory as layer 2's A operand: the thread that reads row
        // r's accumulator columns 128 h .. 128 h + 127 writes their activations, two per column, into columns
        // 128 h .. 128 h + 63 it has already read, so shared memory holds all of W2 and W3 before layer 2 starts.
        // Layer 2 then accumulates outputs 0-63 in columns 64-127 and 64-127 in columns 192-255 (N = 64 each).
        auto load_layer23 = [&]() {  // thread 0: W2's four K-chunks into pages 0-3, W3 into page 4
            umma::FenceProxyAsyncShared();
            for (int kc = 0; kc < 4; ++kc) {
                load(kc, page(kc), ttab + kTblW2 + kc * kW2ChunkBytes, kW2ChunkBytes);
            }
            load(4, page(4), ttab + kTblW3, kPolicy * kHidden1 * 2);
        };
        auto store_h0 = [&](int j, const float (&v)[32]) {  // K = 128 half + 32 j .. + 31
            std::uint32_t r[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                r[i] = Pack2<kFp16>(v[2 * i], v[2 * i + 1]);
            }
            umma::Store16(tmem + static_cast<std::uint32_t>(half * 128 + j * 16) + lane_bits, r);
        };
        auto trunk = [&](int t, int step) {
            if (t == 0) {
                if (tid == 0) {
                    load_layer23();
                }
                float v[32];
#pragma unroll 1
                for (int j = 0; j < 4; ++j) {
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        v[i] = ts.virgin[half * 128 + j * 32 + i];
                    }
                    store_h0(j, v);
                }
                umma::WaitStore();
                phase_sync();
            } else {
                // layer 1: stage 0 = {enc page 2, W1 pages 3-4}, stage 1 = {enc page 5, W1 pages 0-1};
                // turn t-1's tile is already in page 2
                if (tid == 0) {
                    umma::FenceProxyAsyncShared();
                    load(3, page(3), ttab + kTblW1 + (t - 1) * kW1SlotBytes, kW1SlotBytes);
                    if (t >= 2) {
                        load(5, page(5), enc_scratch + (t - 2) * kPageBytes, kPageBytes);
                        load(0, page(0), ttab + kTblW1 + (t - 2) * kW1SlotBytes, kW1SlotBytes);
                    }
                    for (int i = 0; i < t; ++i) {
                        const int u = t - 1 - i;
                        const int st = i & 1;
                        const int enc_b = st == 0 ? 2 : 5;
                        const int w_b = st == 0 ? 3 : 0;
                        bool ok = wait_load(w_b);
                        if (i > 0) {
                            ok = wait_load(enc_b) && ok;
                        }
                        if (ok && can_issue()) {
                            umma::FenceAfterSync();
                            MmaK(tmem, page(enc_b), kEncoderOut, page(w_b), kEncoderOut, kEncoderOut / 16, idesc256,
                                 i > 0);
                        }
                        commit_free(st);
                        if (i + 2 < t) {
                            wait_free(st);
                            load(enc_b, page(enc_b), enc_scratch + (u - 2) * kPageBytes, kPageBytes);
                            load(w_b, page(w_b), ttab + kTblW1 + (u - 2) * kW1SlotBytes, kW1SlotBytes);
                        }
                    }
                }
                commit_mma();
                wait_mma();
                if (tid == 0) {
                    load_layer23();  // every page is free once layer 1's MMAs are done
                }
                float v[32];
#pragma unroll 1
                for (int j = 0; j < 4; ++j) {
                    const int c0 = half * 128 + j * 32;
                    umma::Load32(tmem + static_cast<std::uint32_t>(c0) + lane_bits, v);
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const float h = v[i] + ts.b1[c0 + i];
                        v[i] = h < 0.0f ? 0.0f : h;
                    }
                    store_h0(j, v);
                }
                umma::WaitStore();
                phase_sync();
            }
            // layer 2: A (h0) from tensor memory, 16 K-steps per half of the outputs
            if (tid == 0) {
                for (int kc = 0; kc < 4; ++kc) {
                    if (!wait_load(kc) || !can_issue()) {
                        continue;
                    }
                    umma::FenceAfterSync();
                    const std::uint32_t b_addr = umma::SmemAddress(page(kc));
#pragma unroll
                    for (int g = 0; g < 2; ++g) {
#pragma unroll
                        for (int s4 = 0; s4 < 4; ++s4) {
                            const int s = 4 * kc + s4;
                            const std::uint32_t a_col = s < 8 ? 8u * s : 128u + 8u * (s - 8);
                            const std::uint64_t bd = umma::SmemDescriptor(b_addr + g * 8 * 1024 + s4 * 256, 128,
                                                                          (64 / 8) * 128);
                            umma::MmaTs(tmem + 64u + 128u * g, tmem + a_col, bd, idesc64, s > 0);
                        }
                    }
                }
            }
            commit_mma();
            wait_mma();
            if (tid == 0) {
                // the first embedding tiles whose pages are free already (stage s lives in page 1 + s)
                umma::FenceProxyAsyncShared();
                for (int e = 1; e < kEmbedStages; ++e) {
                    if (e != 3 && e < n_tiles) {  // stage 3 (page 4) still holds W3
                        load(1 + e, page(1 + e), embed + static_cast<std::size_t>(e) * kPageBytes, kPageBytes);
                    }
                }
            }
            {
                std::uint8_t *h1 = page(0);  // [128][128]
                float v[32];
#pragma unroll 1
                for (int j = 0; j < 2; ++j) {
                    const int c0 = half * 64 + j * 32;
                    umma::Load32(tmem + static_cast<std::uint32_t>(64 + 128 * half + j * 32) + lane_bits, v);
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        const float h = v[i] + ts.b2[c0 + i];
                        v[i] = h < 0.0f ? 0.0f : h;
                    }
                    StoreRow32<kFp16>(h1, row, c0, kHidden1, v);
                }
            }
            phase_sync();
            // layer 3
            if (tid == 0 && wait_load(4) && can_issue()) {
                umma::FenceAfterSync();
                MmaK(tmem + 128, page(0), kHidden1, page(4), kHidden1, kHidden1 / 16, idesc64, false);
            }
            commit_mma();
            wait_mma();
            if (tid == 0) {
                umma::FenceProxyAsyncShared();
                if (n_tiles > 0) {
                    load(1, page(1), embed, kPageBytes);
                }
                if (n_tiles > 3) {
                    load(4, page(4), embed + 3 * static_cast<std::size_t>(kPageBytes), kPageBytes);
                }
            }
            {
                float v[32];
                const int c0 = half * 32;
                umma::Load32(tmem + 128u + static_cast<std::uint32_t>(c0) + lane_bits, v);
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    v[i] += ts.b3[c0 + i];
                }
                const std::int32_t e = cs.episode[row];
                if (p.trace_policy != nullptr && !cs.done[row] && e >= 0 &&
                    static_cast<std::uint32_t>(e) < p.trace_episodes) {
                    const std::size_t slot = static_cast<std::size_t>(ind) * p.trace_episodes + e;
                    float *dst = p.trace_policy + (slot * kMaxTurns + step) * kPolicy + c0;
#pragma unroll
                    for (int i = 0; i < 32; ++i) {
                        dst[i] = v[i];
                    }
                }
                StoreRow32<kFp16>(page(0), row, c0, kPolicy, v);
                // squared score spread; a policy value beyond the 16-bit range makes it infinite, which sends
                // the game step to the exact path
                float s = 0.0f;
                bool in_range = true;
#pragma unroll
                for (int i = 0; i < 32; i += 2) {
                    const float2 r = Unpack2<kFp16>(Pack2<kFp16>(v[i], v[i + 1]));
                    in_range &= fabsf(v[i]) < (kFp16 ? 65504.0f : 3.0e38f);
                    in_range &= fabsf(v[i + 1]) < (kFp16 ? 65504.0f : 3.0e38f);
                    s = __fmaf_rn(r.x * r.x, ts.var[c0 + i], s);
                    s = __fmaf_rn(r.y * r.y, ts.var[c0 + i + 1], s);
                }
                ts.s_part[half][row] = in_range ? s : INFINITY;
            }
            phase_sync();
        };

        // ---- scoring: per game, the four largest 32-action chunk maxima of each half of the columns ----
        // No block barrier inside the tile loop. Thread 0 issues tiles 0 and 1; after that, the last warp to finish
        // reading tile k's accumulator buffer (an arrival counter per buffer) refills tile k's embedding stage with
        // tile k + kEmbedStages and issues tile k + 2 into the buffer it has just released. Issuing stalls the
        // issuing thread while the tensor core takes the instructions, and the last reader of a buffer would wait
        // for the buffer's next tile in any case, so the stall stays off the critical path while the other warps
        // read the other buffer. The load counters advance alike in every thread, which keeps thread 0's exact for
        // the phases that follow.
        auto score_tiles = [&]() {
            const std::uint8_t *a_tile = page(0);
            if (tid == 0) {
                ts.load_sync = load_phase;
            }
            __syncthreads();
            load_phase = ts.load_sync;
            auto issue = [&](int tile) {  // one thread
                const int acc = tile & 1;
                const int b = 1 + tile % kEmbedStages;
                if (wait_bar(&ts.bar_load[b], (load_phase >> b) & 1u) && can_issue()) {
                    umma::FenceAfterSync();
                    MmaK(tmem + static_cast<std::uint32_t>(acc * kTileN), a_tile, kPolicy, page(b), kPolicy,
                         kPolicy / 16, idesc128, false);
                    umma::Commit(&ts.bar_acc[acc]);
                }
            };
            for (int k = 0; k < 2 && k < n_tiles; ++k) {
                if (tid == 0) {
                    issue(k);
                }
                load_phase ^= 1u << (1 + k % kEmbedStages);
            }
            float tv[kTopK];
            int ti[kTopK];
#pragma unroll
            for (int j = 0; j < kTopK; ++j) {
                tv[j] = -INFINITY;
                ti[j] = -1;
            }
            for (int tile = 0; tile < n_tiles; ++tile) {
                const int buf = tile & 1;
                wait_bar(&ts.bar_acc[buf], (acc_phase >> buf) & 1u);
                acc_phase ^= 1u << buf;
                umma::FenceAfterSync();
                __syncwarp();
                const bool last = tile + 1 == n_tiles;
                {
                    float v[64];
                    umma::Load64(tmem + static_cast<std::uint32_t>(buf * kTileN + half * 64) + lane_bits, v);
                    if (last) {
#pragma unroll
                        for (int j = 0; j < 64; ++j) {
                            if (static_cast<std::uint32_t>(tile * kTileN + half * 64 + j) >= p.action_count) {
                                v[j] = -INFINITY;
                            }
                        }
                    }
                    v[0] = Max32(v, 0);
                    v[32] = Max32(v, 32);
                    InsertTop4(tv, ti, v[0], tile * 4 + half * 2);
                    InsertTop4(tv, ti, v[32], tile * 4 + half * 2 + 1);
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
                    if ((prior & 7u) == 7u) {  // every warp has read tile's buffer
                        if (tile + kEmbedStages < n_tiles) {
                            const int b = 1 + tile % kEmbedStages;  // tile's MMAs have completed: its stage is free
                            issue_load(b, page(b), embed + static_cast<std::size_t>(tile + kEmbedStages) * kPageBytes,
                                       kPageBytes);
                        }
                        if (tile + 2 < n_tiles) {
                            issue(tile + 2);
                        }
                    }
                }
                if (tile + 2 < n_tiles) {
                    load_phase ^= 1u << (1 + (tile + 2) % kEmbedStages);
                }
            }
            float *cand_v = reinterpret_cast<float *>(smem + kOffCandV);
            int *cand_id = reinterpret_cast<int *>(smem + kOffCandId);
#pragma unroll
            for (int j = 0; j < kTopK; ++j) {
                cand_v[(row * 2 + half) * kTopK + j] = tv[j];
                cand_id[(row * 2 + half) * kTopK + j] = ti[j];
            }
            __syncthreads();
        };

        // Best tracked chunk maximum free of guessed words (by catalog index); `covered` turns false when the
        // tracked lists cannot stand in for every chunk.
        auto best_free_chunk = [&](int g, int t, bool &covered) {
            const float *cand_v = reinterpret_cast<const float *>(smem + kOffCandV);
            const int *cand_id = reinterpret_cast<const int *>(smem + kOffCandId);
            float top = -INFINITY;
            covered = true;
            for (int h = 0; h < 2; ++h) {
                bool found = false;
                for (int j = 0; j < kTopK && !found; ++j) {
                    const int id = cand_id[(g * 2 + h) * kTopK + j];
                    bool masked = false;
                    for (int u = 0; u < t; ++u) {
                        masked |= cs.word_index[u][g] >= 0 && cs.word_index[u][g] / 32 == id;
                    }
                    if (id >= 0 && !masked) {
                        top = fmaxf(top, cand_v[(g * 2 + h) * kTopK + j]);
                        found = true;
                    }
                }
                if (!found && cand_id[(g * 2 + h) * kTopK + kTopK - 1] >= 0) {
                    covered = false;  // every tracked chunk of this half holds a guessed word
                }
            }
            if (!(top > -INFINITY)) {
                covered = false;
            }
            return top;
        };
        // Whether an untracked chunk may reach `floor`: a half whose list is full must end below it.
        auto full_list_reaches = [&](int g, float floor) {
            const float *cand_v = reinterpret_cast<const float *>(smem + kOffCandV);
            const int *cand_id = reinterpret_cast<const int *>(smem + kOffCandId);
            bool r = false;
            for (int h = 0; h < 2; ++h) {
                r |= cand_id[(g * 2 + h) * kTopK + kTopK - 1] >= 0 &&
                     !(cand_v[(g * 2 + h) * kTopK + kTopK - 1] < floor);
            }
            return r;
        };

        // ---- decision from the 16-bit scores, certified by the top-2 margin ----
        auto decide = [&](int t) {
            const float *cand_v = reinterpret_cast<const float *>(smem + kOffCandV);
            const int *cand_id = reinterpret_cast<const int *>(smem + kOffCandId);
            float *excl = reinterpret_cast<float *>(smem + kOffExcl);
            int *task_off = reinterpret_cast<int *>(smem + kOffTaskOff);
            int *task_cnt = reinterpret_cast<int *>(smem + kOffTaskCnt);
            std::uint32_t *tasks = reinterpret_cast<std::uint32_t *>(smem + kOffTasks);
            unsigned long long *results = reinterpret_cast<unsigned long long *>(smem + kOffResults);
            int n = 0;
            float theta = 0.0f;
            bool fallback = false;
            if (tid == 0) {
                ts.n_fallback = 0;
            }
            if (tid < kChunkGames) {
                const int g = tid;
                if (!cs.done[g]) {
                    bool covered = true;
                    const float top = best_free_chunk(g, t, covered);
                    const float spread = sqrtf(ts.s_part[0][g] + ts.s_part[1][g]);
                    theta = top - q.tau * spread;
                    if (!(theta > -INFINITY) || full_list_reaches(g, theta)) {
                        covered = false;
                    }
                    float x = -INFINITY;
                    if (covered) {
                        for (int e = 0; e < 2 * kTopK; ++e) {
                            const int id = cand_id[g * 2 * kTopK + e];
                            const float v = cand_v[g * 2 * kTopK + e];
                            if (id >= 0) {
                                if (v >= theta) {
                                    ++n;
                                } else {
                                    x = fmaxf(x, v);
                                }
                            }
                        }
                    }
                    excl[g] = x;
                    fallback = !covered;
                }
            }
            // block prefix sum of the candidate counts (threads 0..127)
            int incl = n;
            for (int off = 1; off < 32; off <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) {
                    incl += y;
                }
            }
            if (lane == 31 && warp < 4) {
                ts.scan[warp] = incl;
            }
            __syncthreads();
            int total = 0;
            int before = 0;
            for (int w = 0; w < 4; ++w) {
                before += w < warp ? ts.scan[w] : 0;
                total += ts.scan[w];
            }
            if (tid < kChunkGames) {
                const int g = tid;
                const int first = before + incl - n;
                task_off[g] = first;
                task_cnt[g] = n;
                int k = first;
                for (int e = 0; e < 2 * kTopK && n > 0; ++e) {
                    const int id = cand_id[g * 2 * kTopK + e];
                    if (id >= 0 && cand_v[g * 2 * kTopK + e] >= theta) {
                        tasks[k++] = (static_cast<std::uint32_t>(g) << 16) | static_cast<std::uint32_t>(id);
                    }
                }
                if (fallback) {
                    ts.fallback_games[atomicAdd(&ts.n_fallback, 1)] = static_cast<std::uint8_t>(g);
                }
            }
            __syncthreads();
            // re-score each candidate chunk from the 16-bit operands: a warp per chunk (two chunks in flight),
            // top-2 keys by (score, lower action index) from 32-bit warp reductions
            auto task_action = [&](std::uint32_t task) {
                return (task & 0xFFFFu) * 32u + static_cast<std::uint32_t>(lane);
            };
            auto task_bits = [&](std::uint32_t task, const uint4 (&e)[8], std::uint32_t code) {
                const int g = static_cast<int>(task >> 16);
                const bool valid = task_action(task) < p.action_count;
                const float s = ApproxScore<kFp16>(page(0), g, e);
                bool masked = !valid;
                for (int u = 0; u < t; ++u) {
                    masked |= cs.guess[u][g] == code;
                }
                return masked ? 0u : OrderedBits(s);
            };
            auto store_top2 = [&](int k, std::uint32_t task, std::uint32_t ob) {
                const std::uint32_t a0 = (task & 0xFFFFu) * 32u;
                const std::uint32_t m1 = __reduce_max_sync(0xffffffffu, ob);
                const unsigned b1 = __ballot_sync(0xffffffffu, ob == m1 && m1 != 0u);
                const int l1 = b1 != 0u ? __ffs(b1) - 1 : 0;
                const std::uint32_t ob2 = lane == l1 ? 0u : ob;
                const std::uint32_t m2 = __reduce_max_sync(0xffffffffu, ob2);
                const unsigned b2 = __ballot_sync(0xffffffffu, ob2 == m2 && m2 != 0u);
                if (lane == 0) {
                    results[2 * k] = b1 != 0u ? (static_cast<unsigned long long>(m1) << 32) |
                                                    (0xFFFFFFFFu - (a0 + static_cast<std::uint32_t>(l1)))
                                              : 0ull;
                    results[2 * k + 1] =
                        b2 != 0u ? (static_cast<unsigned long long>(m2) << 32) |
                                       (0xFFFFFFFFu - (a0 + static_cast<std::uint32_t>(__ffs(b2) - 1)))
                                 : 0ull;
                }
            };
            constexpr int kWarps = kEvalThreads / 32;
            for (int k0 = warp; k0 < total; k0 += 2 * kWarps) {
                const int k1 = k0 + kWarps;
                const std::uint32_t task0 = tasks[k0];
                const std::uint32_t task1 = k1 < total ? tasks[k1] : task0;
                // both chunks' embedding rows and codes are in flight before either dot product
                const std::uint32_t a0 = task_action(task0);
                const std::uint32_t a1 = task_action(task1);
                const bool v0 = a0 < p.action_count;
                const bool v1 = a1 < p.action_count;
                uint4 e0[8];
                uint4 e1[8];
                LoadEmbedRow(embed, v0 ? a0 : 0u, e0);
                LoadEmbedRow(embed, v1 ? a1 : 0u, e1);
                const std::uint32_t code0 = v0 ? __ldg(p.codes + a0) : 0u;
                const std::uint32_t code1 = v1 ? __ldg(p.codes + a1) : 0u;
                const std::uint32_t ob0 = task_bits(task0, e0, code0);
                const std::uint32_t ob1 = task_bits(task1, e1, code1);
                store_top2(k0, task0, ob0);
                if (k1 < total) {
                    store_top2(k1, task1, ob1);
                }
            }
            __syncthreads();
            if (tid < kChunkGames && !cs.done[tid] && !fallback) {
                const int g = tid;
                unsigned long long best = 0;
                int best_task = -1;
                for (int k = task_off[g]; k < task_off[g] + task_cnt[g]; ++k) {
                    if (results[2 * k] > best) {
                        best = results[2 * k];
                        best_task = k;
                    }
                }
                unsigned long long second = 0;
                for (int k = task_off[g]; k < task_off[g] + task_cnt[g]; ++k) {
                    const unsigned long long c = k == best_task ? results[2 * k + 1] : results[2 * k];
                    second = c > second ? c : second;
                }
                bool ok = best != 0;
                if (ok) {
                    const float s1 = KeyScore(best);
                    const float s2 = fmaxf(second != 0 ? KeyScore(second) : -INFINITY, excl[g]);
                    const float spread = sqrtf(ts.s_part[0][g] + ts.s_part[1][g]);
                    ok = s1 - s2 > 0.0f && s1 - s2 >= q.tau * spread;
                }
                if (ok) {
                    cs.best[g] = KeyAction(best);
                } else {
                    ts.fallback_games[atomicAdd(&ts.n_fallback, 1)] = static_cast<std::uint8_t>(g);
                }
            }
            cand_chunks += tid == 0 ? static_cast<unsigned long long>(total) : 0ull;
            __syncthreads();
        };

        // ---- exact FP32 path for the fallback games (the plain form's chains, bit for bit) ----
        auto exact_fallback = [&](int t, int step) {
            const int nf = ts.n_fallback;
            fallback_steps += tid == 0 ? static_cast<unsigned long long>(nf) : 0ull;
            float *hid = reinterpret_cast<float *>(smem + kOffXHid);  // [f][u][128]
            float *enc = reinterpret_cast<float *>(smem + kOffXEnc);  // [f][u][64]
            float *x0 = reinterpret_cast<float *>(smem + kOffXH0);    // [f][256]
            float *x1 = reinterpret_cast<float *>(smem + kOffXH1);    // [f][128]
            float *xp = reinterpret_cast<float *>(smem + kOffXP);     // [f][64]
            std::uint8_t *stage = smem + kOffXStage;
            unsigned long long *fb_key = reinterpret_cast<unsigned long long *>(smem + kOffFbKey);
            float *fb_win = reinterpret_cast<float *>(smem + kOffFbWin);
            int *fb_full = reinterpret_cast<int *>(smem + kOffFbFull);
            std::uint32_t *fb_tasks = reinterpret_cast<std::uint32_t *>(smem + kOffFbTasks);
            int *fb_count = reinterpret_cast<int *>(smem + kOffFbCount);
            const __half *tail =
                reinterpret_cast<const __half *>(reinterpret_cast<const std::uint8_t *>(gh) + kTailOffsetBytes);
            const float *cand_v = reinterpret_cast<const float *>(smem + kOffCandV);
            const int *cand_id = reinterpret_cast<const int *>(smem + kOffCandId);
            // FP16 form with few fallback games: weights streamed from the trunk table (see fallback_trunk_ring)
            const bool ring = kFp16 && nf <= kMaxSavedRows;
            std::uint8_t *saved = smem + kOffSavedRows;
            if (ring) {
                for (int i = tid; i < nf * 8; i += kEvalThreads) {
                    const int g = ts.fallback_games[i >> 3];
                    reinterpret_cast<uint4 *>(saved)[i] =
                        *reinterpret_cast<const uint4 *>(page(0) + umma::TileOffset(g, (i & 7) * 8, kPolicy));
                }
                __syncthreads();
            }
            // the 16-bit policy value pair (k, k + 1) of fallback game number fi, game row g
            auto policy16 = [&](int fi, int g, int k) {
                return ring ? *reinterpret_cast<const std::uint32_t *>(saved + fi * kPolicy * 2 + k * 2)
                            : *reinterpret_cast<const std::uint32_t *>(page(0) + umma::TileOffset(g, k, kPolicy));
            };
            // The exact trunk of batch games b0 .. b0 + nb - 1 into xp, the plain form's FP32 chains in their order,
            // with every weight tile copied in by bulk copies two tiles ahead of its use: W_e1 in three row
            // groups, W_e2, then per turn the two 128-row halves of its W1 slot, the four K-chunks of W2, and W3.
            auto fallback_trunk_ring = [&](int b0, int nb) {
                float *hid = reinterpret_cast<float *>(smem + kOffXHid);
                float *enc = reinterpret_cast<float *>(smem + kOffXEnc);
                float *x0 = reinterpret_cast<float *>(smem + kOffXH0);
                float *x1 = reinterpret_cast<float *>(smem + kOffXH1);
                float *xp = reinterpret_cast<float *>(smem + kOffXP);
                const int enc_tiles = t > 0 ? 4 : 0;
                const int n_tiles = enc_tiles + 2 * t + 5;
                auto buffer = [&](int i) { return i % kRing == 0 ? page(0) : smem + (i % kRing == 1 ? kOffRing1 : kOffRing2); };
                auto issue = [&](int i) {  // thread 0
                    int kind = i < enc_tiles ? (i < 3 ? 0 : 1) : (i - enc_tiles < 2 * t ? 2 : (i - enc_tiles - 2 * t < 4 ? 3 : 4));
                    std::size_t off = 0;
                    std::uint32_t bytes = kRingTileBytes;
                    if (kind == 0) {
                        off = kTblWe1 + static_cast<std::size_t>(i) * 6 * kWe1GroupBytes;
                        bytes = (i < 2 ? 6 : 4) * kWe1GroupBytes;
                    } else if (kind == 1) {
                        off = kTblWe2;
                    } else if (kind == 2) {
                        off = kTblW1 + static_cast<std::size_t>(i - enc_tiles) * kRingTileBytes;
                    } else if (kind == 3) {
                        off = kTblW2 + static_cast<std::size_t>(i - enc_tiles - 2 * t) * kW2ChunkBytes;
                    } else {
                        off = kTblW3;
                    }
                    if (can_issue()) {
                        BulkLoad(buffer(i), ttab + off, bytes, &ts.bar_ring[i % kRing]);
                        atomicAdd(&ts.ring_issued[i % kRing], 1u);
                    }
                };
                if (tid == 0) {
                    umma::FenceProxyAsyncShared();
                    for (int i = 0; i < kRing && i < n_tiles; ++i) {
                        issue(i);
                    }
                }
                // layer-1 accumulators: output o_local (+128 h) for games sub, sub + 2, sub + 4, sub + 6
                const int o_local = tid & 127;
                const int sub = tid >> 7;
                float acc1a[4], acc1b[4];  // rows o_local and 128 + o_local
                {
                    const float init_a = t == 0 ? __fmaf_rn(H2F(gh, kTrW1 + o_local * kModelInput), 1.0f,
                                                            ts.b1[o_local])
                                                : ts.b1[o_local];
                    const int ob = 128 + o_local;
                    const float init_b =
                        t == 0 ? __fmaf_rn(H2F(gh, kTrW1 + ob * kModelInput), 1.0f, ts.b1[ob]) : ts.b1[ob];
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        acc1a[r] = init_a;
                        acc1b[r] = init_b;
                    }
                }
                // a batch of at most two games needs one chain per thread (game sub), otherwise four
                const bool pair = nb <= 2;
                auto layer1_rows = [&](float (&acc)[4], const std::uint8_t *w, int u) {
                    const std::uint8_t *wrow = w + (o_local >> 3) * 1024 + (o_local & 7) * 16;
                    if (pair) {
                        const float *x = enc + ((sub < nb ? sub : 0) * 5 + u) * kEncoderOut;
                        for (int k8 = 0; k8 < kEncoderOut / 8; ++k8) {
                            const uint4 w8 = *reinterpret_cast<const uint4 *>(wrow + k8 * 128);
                            const __half *h8 = reinterpret_cast<const __half *>(&w8);
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                acc[0] = __fmaf_rn(x[k8 * 8 + e], __half2float(h8[e]), acc[0]);
                            }
                        }
                        return;
                    }
                    for (int k8 = 0; k8 < kEncoderOut / 8; ++k8) {
                        const uint4 w8 = *reinterpret_cast<const uint4 *>(wrow + k8 * 128);
                        const __half *h8 = reinterpret_cast<const __half *>(&w8);
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            const float wv = __half2float(h8[e]);
#pragma unroll
                            for (int r = 0; r < 4; ++r) {
                                const int f = sub + 2 * r;
                                const int fs = f < nb ? f : 0;
                                acc[r] = __fmaf_rn(enc[(fs * 5 + u) * kEncoderOut + k8 * 8 + e], wv, acc[r]);
                            }
                        }
                    }
                };
                auto store_x0 = [&]() {
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int f = sub + 2 * r;
                        if (f < nb) {
                            x0[f * kHidden0 + o_local] = acc1a[r] < 0.0f ? 0.0f : acc1a[r];
                            x0[f * kHidden0 + 128 + o_local] = acc1b[r] < 0.0f ? 0.0f : acc1b[r];
                        }
                    }
                };
                float acc2[4];
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    acc2[r] = ts.b2[o_local];
                }
                for (int i = 0; i < n_tiles; ++i) {
                    const int b = i % kRing;
                    wait_bar(&ts.bar_ring[b], (ring_phase >> b) & 1u);
                    ring_phase ^= 1u << b;
                    const std::uint8_t *w = buffer(i);
                    if (i < enc_tiles && i < 3) {
                        // encoder hidden rows of this group: EncodeRound's gather chain, ascending feature order
                        const int r0 = i * 48;
                        const int rows = i < 2 ? 48 : 32;
                        for (int idx = tid; idx < nb * t * rows; idx += kEvalThreads) {
                            const int ol = idx % rows;
                            const int fu = idx / rows;
                            const int f = fu / t;
                            const int u = fu - f * t;
                            const int o = r0 + ol;
                            const int g = ts.fallback_games[b0 + f];
                            const std::uint32_t code = cs.guess[u][g];
                            const std::uint32_t tiles = cs.tiles[u][g];
                            const std::uint8_t *row = w + (ol >> 3) * kWe1GroupBytes + (o & 7) * 16;
                            auto we1 = [&](int feature) {
                                return __half2float(*reinterpret_cast<const __half *>(row + (feature >> 3) * 128 +
                                                                                     (feature & 7) * 2));
                            };
                            float hsum = ts.be1[o];
                            for (int pos = 0; pos < kWordLength; ++pos) {
                                hsum = __fmaf_rn(we1(pos * kAlphabet + static_cast<int>(WordLetter(code, pos))), 1.0f,
                                                 hsum);
                            }
                            for (int pos = 0; pos < kWordLength; ++pos) {
                                hsum = __fmaf_rn(we1(kWordLength * kAlphabet + pos * 3 +
                                                     static_cast<int>((tiles >> (2 * pos)) & 3u)),
                                                 1.0f, hsum);
                            }
                            hid[(f * 5 + u) * kEncoderHidden + o] = hsum < 0.0f ? 0.0f : hsum;
                        }
                    } else if (i < enc_tiles) {
                        // encoder output: thread (j, group), five chains at once, 8 weights per 16-byte read
                        const int j = tid & (kEncoderOut - 1);
                        const int grp = tid >> 6;
                        const int pairs = nb * t;
                        const std::uint8_t *wrow = w + (j >> 3) * (kEncoderHidden / 8) * 128 + (j & 7) * 16;
                        for (int q0 = grp; q0 < pairs; q0 += 20) {
                            float acc[5];
                            int base[5];
#pragma unroll
                            for (int r = 0; r < 5; ++r) {
                                const int qq = q0 + 4 * r;
                                const int f = qq < pairs ? qq / t : 0;
                                const int u = qq < pairs ? qq - f * t : 0;
                                base[r] = (f * 5 + u) * kEncoderHidden;
                                acc[r] = ts.be2[j];
                            }
                            for (int o8 = 0; o8 < kEncoderHidden / 8; ++o8) {
                                const uint4 w8 = *reinterpret_cast<const uint4 *>(wrow + o8 * 128);
                                const __half *h8 = reinterpret_cast<const __half *>(&w8);
#pragma unroll
                                for (int e = 0; e < 8; ++e) {
                                    const float wv = __half2float(h8[e]);
#pragma unroll
                                    for (int r = 0; r < 5; ++r) {
                                        acc[r] = __fmaf_rn(hid[base[r] + o8 * 8 + e], wv, acc[r]);
                                    }
                                }
                            }
#pragma unroll
                            for (int r = 0; r < 5; ++r) {
                                const int qq = q0 + 4 * r;
                                if (qq < pairs) {
                                    const int f = qq / t;
                                    const int u = qq - f * t;
                                    enc[(f * 5 + u) * kEncoderOut + j] = acc[r];
                                }
                            }
                        }
                    } else if (i - enc_tiles < 2 * t) {
                        // layer 1, turn u, rows 128 h .. 128 h + 127: the chains continue in ascending input order
                        const int u = (i - enc_tiles) >> 1;
                        if (((i - enc_tiles) & 1) == 0) {
                            layer1_rows(acc1a, w, u);
                        } else {
                            layer1_rows(acc1b, w, u);
                            if (u == t - 1) {
                                store_x0();
                            }
                        }
                    } else if (i - enc_tiles - 2 * t < 4) {
                        // layer 2, K-chunk kc: thread (n, parity) over the batch games of its parity
                        const int kc = i - enc_tiles - 2 * t;
                        if (kc == 0 && t == 0) {  // no turn: every output is relu(b1 + W1[:, 0])
                            store_x0();
                            __syncthreads();
                        }
                        const std::uint8_t *wrow = w + (o_local >> 3) * 1024 + (o_local & 7) * 16;
                        if (pair) {
                            const float *x = x0 + (sub < nb ? sub : 0) * kHidden0 + kc * 64;
                            for (int k8 = 0; k8 < 8; ++k8) {
                                const uint4 w8 = *reinterpret_cast<const uint4 *>(wrow + k8 * 128);
                                const __half *h8 = reinterpret_cast<const __half *>(&w8);
#pragma unroll
                                for (int e = 0; e < 8; ++e) {
                                    acc2[0] = __fmaf_rn(x[k8 * 8 + e], __half2float(h8[e]), acc2[0]);
                                }
                            }
                        } else {
                            for (int k8 = 0; k8 < 8; ++k8) {
                                const uint4 w8 = *reinterpret_cast<const uint4 *>(wrow + k8 * 128);
                                const __half *h8 = reinterpret_cast<const __half *>(&w8);
#pragma unroll
                                for (int e = 0; e < 8; ++e) {
                                    const float wv = __half2float(h8[e]);
#pragma unroll
                                    for (int r = 0; r < 4; ++r) {
                                        const int f = sub + 2 * r;
                                        const int fs = f < nb ? f : 0;
                                        acc2[r] = __fmaf_rn(x0[fs * kHidden0 + kc * 64 + k8 * 8 + e], wv, acc2[r]);
                                    }
                                }
                            }
                        }
                        if (kc == 3) {
#pragma unroll
                            for (int r = 0; r < 4; ++r) {
                                const int f = sub + 2 * r;
                                if (f < nb) {
                                    x1[f * kHidden1 + o_local] = acc2[r] < 0.0f ? 0.0f : acc2[r];
                                }
                            }
                        }
                    } else {
                        // layer 3: thread (j, group of four) over two batch games
                        const int j = tid & 63;
                        const int grp = tid >> 6;
                        float acc[2] = {ts.b3[j], ts.b3[j]};
                        const std::uint8_t *wrow = w + (j >> 3) * (kHidden1 / 8) * 128 + (j & 7) * 16;
                        for (int k8 = 0; k8 < kHidden1 / 8; ++k8) {
                            const uint4 w8 = *reinterpret_cast<const uint4 *>(wrow + k8 * 128);
                            const __half *h8 = reinterpret_cast<const __half *>(&w8);
#pragma unroll
                            for (int e = 0; e < 8; ++e) {
                                const float wv = __half2float(h8[e]);
#pragma unroll
                                for (int r = 0; r < 2; ++r) {
                                    const int f = grp + 4 * r;
                                    const int fs = f < nb ? f : 0;
                                    acc[r] = __fmaf_rn(x1[fs * kHidden1 + k8 * 8 + e], wv, acc[r]);
                                }
                            }
                        }
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                            const int f = grp + 4 * r;
                            if (f < nb) {
                                xp[f * kPolicy + j] = acc[r];
                            }
                        }
                    }
                    __syncthreads();
                    if (tid == 0 && i + kRing < n_tiles) {
                        umma::FenceProxyAsyncShared();
                        issue(i + kRing);
                    }
                }
            };
            for (int b0 = 0; b0 < nf; b0 += kFallbackBatch) {
                const int nb = nf - b0 < kFallbackBatch ? nf - b0 : kFallbackBatch;
                if (ring) {
                    fallback_trunk_ring(b0, nb);
                } else {
                // encoder hidden layer of every turn (EncodeRound's gather chain), W_e1 staged in shared memory
                {
                    const uint4 *src = reinterpret_cast<const uint4 *>(gh + kEncW1);
                    uint4 *dst = reinterpret_cast<uint4 *>(stage);
                    for (int i = tid; i < kEncoderHidden * kTurnFeatures * 2 / 16; i += kEvalThreads) {
                        dst[i] = __ldg(src + i);
                    }
                }
                __syncthreads();
                {
                    const __half *we1 = reinterpret_cast<const __half *>(stage);
                    for (int i = tid; i < nb * t * kEncoderHidden; i += kEvalThreads) {
                        const int o = i & (kEncoderHidden - 1);
                        const int fu = i >> 7;
                        const int f = fu / t;
                        const int u = fu - f * t;
                        const int g = ts.fallback_games[b0 + f];
                        const std::uint32_t code = cs.guess[u][g];
                        const std::uint32_t tiles = cs.tiles[u][g];
                        const __half *wr = we1 + o * kTurnFeatures;
                        float h = ts.be1[o];
                        for (int pos = 0; pos < kWordLength; ++pos) {
                            h = __fmaf_rn(__half2float(wr[pos * kAlphabet + static_cast<int>(WordLetter(code, pos))]),
                                          1.0f, h);
                        }
                        for (int pos = 0; pos < kWordLength; ++pos) {
                            h = __fmaf_rn(__half2float(wr[kWordLength * kAlphabet + pos * 3 +
                                                          static_cast<int>((tiles >> (2 * pos)) & 3u)]),
                                          1.0f, h);
                        }
                        hid[(f * 5 + u) * kEncoderHidden + o] = h < 0.0f ? 0.0f : h;
                    }
                }
                __syncthreads();
                // encoder output layer: W_e2 staged transposed ([o][j]); thread (j, group) runs five chains at once
                {
                    __half *w2t = reinterpret_cast<__half *>(stage);
                    for (int i = tid; i < kEncoderOut * kEncoderHidden / 8; i += kEvalThreads) {
                        const int j = i & (kEncoderOut - 1);
                        const int o0 = (i >> 6) * 8;
                        const uint4 w4 = __ldg(reinterpret_cast<const uint4 *>(gh + kEncW2 + j * kEncoderHidden + o0));
                        const __half *h8 = reinterpret_cast<const __half *>(&w4);
#pragma unroll
                        for (int e = 0; e < 8; ++e) {
                            w2t[(o0 + e) * kEncoderOut + j] = h8[e];
                        }
                    }
                }
                __syncthreads();
                {
                    const __half *w2t = reinterpret_cast<const __half *>(stage);
                    const int j = tid & (kEncoderOut - 1);
                    const int grp = tid >> 6;
                    const int pairs = nb * t;
                    for (int q0 = grp; q0 < pairs; q0 += 20) {
                        float acc[5];
                        int base[5];
#pragma unroll
                        for (int r = 0; r < 5; ++r) {
                            const int qq = q0 + 4 * r;
                            const int f = qq < pairs ? qq / t : 0;
                            const int u = qq < pairs ? qq - f * t : 0;
                            base[r] = (f * 5 + u) * kEncoderHidden;
                            acc[r] = ts.be2[j];
                        }
#pragma unroll 4
                        for (int o = 0; o < kEncoderHidden; ++o) {
                            const float w = __half2float(w2t[o * kEncoderOut + j]);
#pragma unroll
                            for (int r = 0; r < 5; ++r) {
                                acc[r] = __fmaf_rn(hid[base[r] + o], w, acc[r]);
                            }
                        }
#pragma unroll
                        for (int r = 0; r < 5; ++r) {
                            const int qq = q0 + 4 * r;
                            if (qq < pairs) {
                                const int f = qq / t;
                                const int u = qq - f * t;
                                enc[(f * 5 + u) * kEncoderOut + j] = acc[r];
                            }
                        }
                    }
                }
                __syncthreads();
                // layer 1: thread o, all batch games side by side (the chains continue across the turns in
                // ascending input order); each turn's 256 x 64 weight slice is staged in shared memory first
                {
                    const int o = tid;
                    const __half *w1s = reinterpret_cast<const __half *>(stage);
                    float acc[kFallbackBatch];
                    int ebase[kFallbackBatch];
#pragma unroll
                    for (int r = 0; r < kFallbackBatch; ++r) {
                        ebase[r] = (r < nb ? r : 0) * 5 * kEncoderOut;
                        acc[r] = t == 0 ? __fmaf_rn(H2F(gh, kTrW1 + o * kModelInput), 1.0f, ts.b1[o]) : ts.b1[o];
                    }
                    for (int u = 0; u < t; ++u) {
                        __syncthreads();
                        StageRows<kEncoderOut>(reinterpret_cast<__half *>(stage), kStageLd, gh + kTrW1 + 1 + kEncoderOut * u,
                                               kModelInput, kHidden0);
                        __syncthreads();
                        if (nb <= 4) {
#pragma unroll 4
                            for (int k = 0; k < kEncoderOut; ++k) {
                                const float w = __half2float(w1s[o * kStageLd + k]);
#pragma unroll
                                for (int r = 0; r < 4; ++r) {
                                    acc[r] = __fmaf_rn(enc[ebase[r] + u * kEncoderOut + k], w, acc[r]);
                                }
                            }
                        } else {
#pragma unroll 2
                            for (int k = 0; k < kEncoderOut; ++k) {
                                const float w = __half2float(w1s[o * kStageLd + k]);
#pragma unroll
                                for (int r = 0; r < kFallbackBatch; ++r) {
                                    acc[r] = __fmaf_rn(enc[ebase[r] + u * kEncoderOut + k], w, acc[r]);
                                }
                            }
                        }
                    }
#pragma unroll
                    for (int r = 0; r < kFallbackBatch; ++r) {
                        if (r < nb) {
                            x0[r * kHidden0 + o] = acc[r] < 0.0f ? 0.0f : acc[r];
                        }
                    }
                }
                __syncthreads();
                // layer 2: thread (n, parity) over the batch games of its parity; 64 weights fetched per block
                {
                    const int n = tid & 127;
                    const int par = tid >> 7;
                    int xbase[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int f = par + 2 * r;
                        xbase[r] = (f < nb ? f : 0) * kHidden0;
                    }
                    float acc[4];
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        acc[r] = ts.b2[n];
                    }
                    const __half *w2s = reinterpret_cast<const __half *>(stage);
                    for (int k0 = 0; k0 < kHidden0; k0 += 64) {
                        __syncthreads();
                        StageRows<64>(reinterpret_cast<__half *>(stage), kStageLd, gh + kTrW2 + k0, kHidden0, kHidden1);
                        __syncthreads();
#pragma unroll 4
                        for (int k = 0; k < 64; ++k) {
                            const float w = __half2float(w2s[n * kStageLd + k]);
#pragma unroll
                            for (int r = 0; r < 4; ++r) {
                                acc[r] = __fmaf_rn(x0[xbase[r] + k0 + k], w, acc[r]);
                            }
                        }
                    }
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        const int f = par + 2 * r;
                        if (f < nb) {
                            x1[f * kHidden1 + n] = acc[r] < 0.0f ? 0.0f : acc[r];
                        }
                    }
                }
                __syncthreads();
                // layer 3: thread (j, group of four) over two batch games
                {
                    const int j = tid & 63;
                    const int grp = tid >> 6;
                    int xbase[2];
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        const int f = grp + 4 * r;
                        xbase[r] = (f < nb ? f : 0) * kHidden1;
                    }
                    float acc[2] = {ts.b3[j], ts.b3[j]};
                    StageRows<kHidden1>(reinterpret_cast<__half *>(stage), kStageLd3, gh + kTrW3, kHidden1, kPolicy);
                    __syncthreads();
                    const __half *w3s = reinterpret_cast<const __half *>(stage);
#pragma unroll 4
                    for (int k = 0; k < kHidden1; ++k) {
                        const float w = __half2float(w3s[j * kStageLd3 + k]);
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                            acc[r] = __fmaf_rn(x1[xbase[r] + k], w, acc[r]);
                        }
                    }
#pragma unroll
                    for (int r = 0; r < 2; ++r) {
                        const int f = grp + 4 * r;
                        if (f < nb) {
                            xp[f * kPolicy + j] = acc[r];
                        }
                    }
                }
                }  // existing staged path
                if (tid == 0) {
                    *fb_count = 0;
                }
                __syncthreads();
                // exact policy into the trace; exact argmax over every chunk the 16-bit maxima cannot rule out
                if (p.trace_policy != nullptr) {
                    for (int i = tid; i < nb * kPolicy; i += kEvalThreads) {
                        const int f = i >> 6;
                        const int g = ts.fallback_games[b0 + f];
                        const std::int32_t e = cs.episode[g];
                        if (e >= 0 && static_cast<std::uint32_t>(e) < p.trace_episodes) {
                            const std::size_t slot = static_cast<std::size_t>(ind) * p.trace_episodes + e;
                            p.trace_policy[(slot * kMaxTurns + step) * kPolicy + (i & 63)] = xp[i];
                        }
                    }
                }
                if (tid < nb) {
                    const int f = tid;
                    const int g = ts.fallback_games[b0 + f];
                    float dev = 0.0f;
                    float mag = 0.0f;
                    for (int k = 0; k < kPolicy; k += 2) {
                        const std::uint32_t bits = policy16(b0 + f, g, k);
                        const float2 r = Unpack2<kFp16>(bits);
                        dev = __fmaf_rn(fabsf(r.x - xp[f * kPolicy + k]), ts.emax[k], dev);
                        dev = __fmaf_rn(fabsf(r.y - xp[f * kPolicy + k + 1]), ts.emax[k + 1], dev);
                        mag = __fmaf_rn(fabsf(r.x), ts.emax[k], mag);
                        mag = __fmaf_rn(fabsf(r.y), ts.emax[k + 1], mag);
                    }
                    const float err = dev * 1.001f + 1.0e-4f * mag;
                    bool covered = true;
                    const float top = best_free_chunk(g, t, covered);
                    const float window = top - 2.0f * err;
                    const bool full =
                        !covered || !(err < INFINITY) || !(window > -INFINITY) || full_list_reaches(g, window);
                    fb_key[f] = 0;
                    fb_win[f] = top - err;
                    if (!full) {
                        for (int e = 0; e < 2 * kTopK; ++e) {
                            const int id = cand_id[g * 2 * kTopK + e];
                            if (id >= 0 && cand_v[g * 2 * kTopK + e] >= window) {
                                fb_tasks[atomicAdd(fb_count, 1)] =
                                    (static_cast<std::uint32_t>(f) << 16) | static_cast<std::uint32_t>(id);
                            }
                        }
                    }
                    fb_full[f] = full ? 1 : 0;
                }
                __syncthreads();
                const int n_tasks = *fb_count;
                constexpr int kWarps = kEvalThreads / 32;
                if constexpr (kFp16) {
                    // the FP16 table holds every embedding value exactly: two tasks per warp in flight
                    for (int k0 = warp; k0 < n_tasks; k0 += 2 * kWarps) {
                        const int k1 = k0 + kWarps;
                        const std::uint32_t task0 = fb_tasks[k0];
                        const std::uint32_t task1 = k1 < n_tasks ? fb_tasks[k1] : task0;
                        const int f0 = static_cast<int>(task0 >> 16);
                        const int f1 = static_cast<int>(task1 >> 16);
                        unsigned long long key0 = 0;
                        unsigned long long key1 = 0;
                        ChunkKeyPairFp16<1>(p, cs, embed, xp + f0 * kPolicy, ts.fallback_games[b0 + f0],
                                            static_cast<int>(task0 & 0xFFFFu), xp + f1 * kPolicy,
                                            ts.fallback_games[b0 + f1], static_cast<int>(task1 & 0xFFFFu), t, key0,
                                            key1);
                        FoldKeys(fb_key + f0, key0);
                        if (k1 < n_tasks) {
                            FoldKeys(fb_key + f1, key1);
                        }
                    }
                } else {
                    for (int k = warp; k < n_tasks; k += kWarps) {
                        const int f = static_cast<int>(fb_tasks[k] >> 16);
                        RescoreChunk(p, cs, fb_key + f, xp + f * kPolicy, 1, tail, ts.fallback_games[b0 + f],
                                     static_cast<int>(fb_tasks[k] & 0xFFFFu), t);
                    }
                }
                __syncthreads();
                if (tid < nb && !fb_full[tid]) {
                    const unsigned long long key = fb_key[tid];
                    if (key == 0 || KeyScore(key) < fb_win[tid]) {
                        fb_full[tid] = 1;  // the exact best stays below what the window guarantees
                    }
                }
                __syncthreads();
                const int chunks_per_row = static_cast<int>((p.action_count + 31) / 32);
                for (int f = 0; f < nb; ++f) {
                    if (fb_full[f]) {
                        // each lane keeps its best key over the warp's chunks; one fold per warp and row
                        unsigned long long key = 0;
                        const int g = ts.fallback_games[b0 + f];
                        if constexpr (kFp16) {
                            for (int c0 = warp; c0 < chunks_per_row; c0 += 2 * kWarps) {
                                const int c1 = c0 + kWarps;
                                unsigned long long key0 = 0;
                                unsigned long long key1 = 0;
                                ChunkKeyPairFp16<1>(p, cs, embed, xp + f * kPolicy, g, c0, xp + f * kPolicy, g,
                                                    c1 < chunks_per_row ? c1 : c0, t, key0, key1);
                                key = key0 > key ? key0 : key;
                                key = c1 < chunks_per_row && key1 > key ? key1 : key;
                            }
                        } else {
                            for (int c = warp; c < chunks_per_row; c += kWarps) {
                                const unsigned long long k = ChunkKey(p, cs, xp + f * kPolicy, 1, tail, g, c, t);
                                key = k > key ? k : key;
                            }
                        }
                        FoldKeys(fb_key + f, key);
                    }
                }
                __syncthreads();
                if (tid < nb) {
                    const unsigned long long key = fb_key[tid];
                    cs.best[ts.fallback_games[b0 + tid]] = key == 0 ? -1 : KeyAction(key);
                }
                if (tid == 0) {
                    exact_chunks += static_cast<unsigned long long>(n_tasks);
                    for (int f = 0; f < nb; ++f) {
                        exact_rows += fb_full[f] ? 1ull : 0ull;
                    }
                }
                __syncthreads();
            }
        };

        if (cs.cls == 1 && CountActive(cs) > 0) {
            encode_turn(0);
            encode_turn(1);
            encoded += tid == 0 ? 2ull * cs.active : 0ull;
        }
        for (int step = 0; step < kMaxTurns; ++step) {
            if (CountActive(cs) == 0 || ts.failed) {
                break;
            }
            const int t = cs.cls == 0 ? step : step + 2;
            if (step > 0) {
                encode_turn(t - 1);
                encoded += tid == 0 ? static_cast<unsigned long long>(cs.active) : 0ull;
            }
            trunk(t, step);
            score_tiles();
            if (ts.failed) {
                break;
            }
            decide(t);
            if (ts.n_fallback > 0) {
                exact_fallback(t, step);
                if (__syncthreads_or(failed_now())) {  // a ring wait gave up: no guess from this step
                    break;
                }
            }
            AppendGuesses(p, cs, step, decisions);
        }
        FinishChunk(p, cs, ind, episodes);
    }
    FlushCounters(p, decisions, encoded, episodes);
    if (tid == 0 && q.counters != nullptr) {
        atomicAdd(q.counters + 0, cand_chunks);
        atomicAdd(q.counters + 1, fallback_steps);
        atomicAdd(q.counters + 2, exact_chunks);
        atomicAdd(q.counters + 3, exact_rows);
    }
    __syncthreads();
    if (ts.failed) {  // read after the barrier: uniform
        if (tid == 0) {
            SetStatus(p.status, kTimeout);
        }
        // every warp's MMAs (a commit tracks all of its thread's earlier tensor-core operations; lane 0 of each warp
        // is the only issuer in it), then the last copy issued on each barrier (the n-th copy completes phase n - 1)
        if (lane == 0) {
            umma::Commit(&ts.bar_drain[warp]);
            (void)umma::MbarWait(&ts.bar_drain[warp], 0, kDrainLimit);
        }
        if (tid == 0) {
            for (int b = 0; b < kPages; ++b) {
                const unsigned int n = ts.loads_issued[b];
                if (n != 0) {
                    (void)umma::MbarWait(&ts.bar_load[b], (n - 1u) & 1u, kDrainLimit);
                }
            }
            for (int b = 0; b < kRing; ++b) {
                const unsigned int n = ts.ring_issued[b];
                if (n != 0) {
                    (void)umma::MbarWait(&ts.bar_ring[b], (n - 1u) & 1u, kDrainLimit);
                }
            }
        }
    }
    umma::FenceBeforeSync();
    __syncthreads();
    if (tid < 32) {
        umma::Dealloc(tmem, kTmemColumns);
    }
}

// Per individual: every trunk weight matrix as a 16-bit K-major canonical operand (kTblWe1 .. kTblW3).
// One thread writes one 16-byte segment (8 values of one row).
template <bool kFp16>
__global__ void BuildTrunkTablesKernel(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                       std::uint8_t *tables, std::size_t table_pitch) {
    const std::uint32_t ind = blockIdx.y;
    const int off = (blockIdx.x * blockDim.x + threadIdx.x) * 16;
    const __half *gh = reinterpret_cast<const __half *>(slab + static_cast<std::size_t>(slots[ind]) * pitch);
    int local, K, base, ld, col0, kvalid;
    if (off < kTblWe2) {
        local = off - kTblWe1, K = kKe1, base = kEncW1, ld = kTurnFeatures, col0 = 0, kvalid = kTurnFeatures;
    } else if (off < kTblW1) {
        local = off - kTblWe2, K = kEncoderHidden, base = kEncW2, ld = kEncoderHidden, col0 = 0, kvalid = K;
    } else if (off < kTblW2) {
        const int u = (off - kTblW1) / kW1SlotBytes;
        local = (off - kTblW1) - u * kW1SlotBytes, K = kEncoderOut, base = kTrW1, ld = kModelInput;
        col0 = 1 + kEncoderOut * u, kvalid = K;
    } else if (off < kTblW3) {
        const int kc = (off - kTblW2) / kW2ChunkBytes;
        local = (off - kTblW2) - kc * kW2ChunkBytes, K = 64, base = kTrW2, ld = kHidden0, col0 = 64 * kc, kvalid = K;
    } else {
        local = off - kTblW3, K = kHidden1, base = kTrW3, ld = kHidden1, col0 = 0, kvalid = K;
    }
    const int seg = local / 16;
    const int r = (seg / K) * 8 + (seg & 7);
    const int k0 = ((seg >> 3) % (K / 8)) * 8;
    std::uint16_t v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int k = k0 + i;
        const __half h = k < kvalid ? gh[base + r * ld + col0 + k] : __float2half_rn(0.0f);
        v[i] = kFp16 ? __half_as_ushort(h) : __bfloat16_as_ushort(__float2bfloat16_rn(__half2float(h)));
    }
    uint4 w;
    w.x = v[0] | (static_cast<std::uint32_t>(v[1]) << 16);
    w.y = v[2] | (static_cast<std::uint32_t>(v[3]) << 16);
    w.z = v[4] | (static_cast<std::uint32_t>(v[5]) << 16);
    w.w = v[6] | (static_cast<std::uint32_t>(v[7]) << 16);
    *reinterpret_cast<uint4 *>(tables + static_cast<std::size_t>(ind) * table_pitch + off) = w;
}

}  // namespace

std::size_t TrunkTablePitch() { return kTrunkTableBytes; }

cudaError_t LaunchBuildTrunkTables(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                   std::uint32_t population, std::uint8_t *tables, bool fp16, cudaStream_t stream) {
    const dim3 grid(kTrunkTableBytes / 16 / 256, population);
    if (fp16) {
        BuildTrunkTablesKernel<true><<<grid, 256, 0, stream>>>(slab, pitch, slots, tables, kTrunkTableBytes);
    } else {
        BuildTrunkTablesKernel<false><<<grid, 256, 0, stream>>>(slab, pitch, slots, tables, kTrunkTableBytes);
    }
    return cudaGetLastError();
}

cudaError_t LaunchEvalTct(const EvalParams &params, const std::uint8_t *embed_tables, std::size_t embed_pitch,
                          const std::uint8_t *trunk_tables, float tau, bool fp16, unsigned long long *counters,
                          int cta_count, cudaStream_t stream, std::uint32_t wait_limit) {
    static std::atomic<unsigned long long> configured[2]{{0}, {0}};
    if (const cudaError_t e = fp16 ? RaiseSharedLimit(EvalTctKernel<true>, kSmemBytes, configured[1])
                                   : RaiseSharedLimit(EvalTctKernel<false>, kSmemBytes, configured[0]);
        e != cudaSuccess) {
        return e;
    }
    if (cta_count <= 0) {
        return cudaSuccess;
    }
    TctParams q{};
    q.base = params;
    q.embed_tables = embed_tables;
    q.embed_pitch = embed_pitch;
    q.trunk_tables = trunk_tables;
    q.trunk_pitch = kTrunkTableBytes;
    q.tau = tau;
    q.counters = counters;
    q.wait_limit = wait_limit;
    if (fp16) {
        EvalTctKernel<true><<<cta_count, kEvalThreads, kSmemBytes, stream>>>(q);
    } else {
        EvalTctKernel<false><<<cta_count, kEvalThreads, kSmemBytes, stream>>>(q);
    }
    return cudaGetLastError();
}

}  // namespace nwg
