// Child assembly: hierarchical crossover plus Philox-driven mutation, one warp per child.
//
// Replaces AssembleChildBatchKernel (genotype_slab/device_runtime.cu:448-516), whose single thread per
// child walked BreedAndMutateGenome (genetic_algorithm/device/genome_ops.cuh:386-407) byte by byte.
// Here a warp assembles a child:
//   1. the crossover decisions are drawn from the child's stream (seed, uint32(child + g * 4099))
//      in the reference's order (genome_ops.cuh:264-299, :344-376);
//   2. the donor layers and tail rows are copied with coalesced 128-bit loads and stores, then the
//      single-neuron / single-row / splice overrides are applied;
//   3. the per-value mutation stream (genome_ops.cuh:153-167, :237-257): a fresh normal pair consumes two
//      more draw positions and leaves its second value cached for the next hit, as the generator's normal
//      does. Runs of at least 4,096 values take the window-parallel walk (MutateRunWindows: every lane owns
//      a 128-position window, 32 windows per step); shorter runs, mutation without normals and p >= 1 take
//      the serial walk (MutateRun: 128 positions at a time for the whole warp, the hit list resolved in
//      order, the normals applied 32 queued hits at a time).
// Every uniform, 32-bit draw and normal is produced by the toolkit generator itself (curand_init at the
// draw's position, then curand4 / curand_uniform / curand / curand_normal; a hit test compares the 32-bit
// draw with the threshold curand_uniform maps to p), so the child image is bit-identical to the
// reference's serial walk.
#include <cuda_fp16.h>
#include <curand_kernel.h>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kFlushAt = 32;
constexpr int kEventCapacity = kFlushAt + 128;  // queued hits: fewer than kFlushAt, plus at most 128 per window

struct LayerSpan {
    int weights;
    int biases;
    int fan_in;
    int outputs;
};

__constant__ LayerSpan kLayers[5] = {
    {kEncW1, kEncB1, kTurnFeatures, kEncoderHidden},
    {kEncW2, kEncB2, kEncoderHidden, kEncoderOut},
    {kTrW1, kTrB1, kModelInput, kHidden0},
    {kTrW2, kTrB2, kHidden0, kHidden1},
    {kTrW3, kTrB3, kHidden1, kPolicy},
};

struct Stream {
    unsigned long long seed;
    unsigned long long subsequence;
    unsigned long long position;     // next 32-bit output to be consumed
    unsigned long long cached_pair;  // position of the normal pair whose second value is cached
    bool cached;
};

__device__ __forceinline__ curandStatePhilox4_32_10_t StateAt(const Stream &s, unsigned long long position) {
    curandStatePhilox4_32_10_t state;
    curand_init(s.seed, s.subsequence, position, &state);
    return state;
}

// Sequential control draws (genome_ops.cuh:35-52); every lane computes the same values.
__device__ bool DrawBernoulli(Stream &s, float p) {
    if (p <= 0.0f) {
        return false;
    }
    if (p >= 1.0f) {
        return true;
    }
    curandStatePhilox4_32_10_t state = StateAt(s, s.position);
    s.position += 1;
    return curand_uniform(&state) < p;
}

__device__ std::uint32_t DrawIndex(Stream &s, std::uint32_t n) {
    if (n <= 1) {
        return 0;
    }
    curandStatePhilox4_32_10_t state = StateAt(s, s.position);
    s.position += 1;
    return curand(&state) % n;
}

// A queued hit in one word: the value index in the low 32 bits; in the high 32 bits the draw position of its
// normal pair, with bit 31 set when the hit takes the pair's second value. A child's draw positions stay below
// 2^31 (LaunchBreed checks the genome size), so a position fits in 31 bits.
struct EventList {
    unsigned long long packed[kEventCapacity];
};

__device__ __forceinline__ void ApplyNormal(__half *values, std::uint32_t v, const Stream &s, unsigned long long pair,
                                            bool second, float sigma) {
    const float old = __half2float(values[v]);
    curandStatePhilox4_32_10_t state = StateAt(s, pair);
    float n = curand_normal(&state);
    if (second) {
        n = curand_normal(&state);
    }
    values[v] = __float2half(__fmaf_rn(sigma, n, old));
}

// Applies the queued hits (each value is hit at most once per walk, so the order does not matter).
__device__ __forceinline__ void FlushEvents(__half *values, const Stream &s, float sigma, EventList &ev, int &n_events,
                                            int lane) {
    __syncwarp();
    for (int e = lane; e < n_events; e += 32) {
        const unsigned long long w = ev.packed[e];
        const std::uint32_t hi = static_cast<std::uint32_t>(w >> 32);
        ApplyNormal(values, static_cast<std::uint32_t>(w), s, hi & 0x7FFFFFFFu, (hi >> 31) != 0u, sigma);
    }
    __syncwarp();
    n_events = 0;
}

// Per-value Bernoulli(p) mutation with sigma * N(0, 1) on hits, over values[0, count).
// with_normals = false draws the Bernoulli uniforms but no normals (genome_ops.cuh:241-243 with sigma <= 0).
__device__ void MutateRun(__half *values, std::uint32_t count, Stream &s, float p, float sigma, bool with_normals,
                          EventList &ev, int lane) {
    if (count == 0 || p <= 0.0f) {
        return;
    }
    if (p >= 1.0f) {
        // every value is a hit and no uniform is drawn
        if (!with_normals) {
            return;
        }
        const bool c0 = s.cached;
        const unsigned long long base = s.position;
        for (std::uint32_t k0 = 0; k0 < count; k0 += 32) {
            const std::uint32_t k = k0 + lane;
            if (k < count) {
                if (c0 && k == 0) {
                    ApplyNormal(values, k, s, s.cached_pair, true, sigma);
                } else {
                    const std::uint32_t j = c0 ? k - 1 : k;
                    ApplyNormal(values, k, s, base + 2ull * (j / 2), (j & 1u) != 0, sigma);
                }
            }
        }
        const std::uint32_t fresh = c0 ? count - 1 : count;
        const unsigned long long pairs = (fresh + 1) / 2;
        s.position = base + 2ull * pairs;
        s.cached = (fresh & 1u) != 0;
        s.cached_pair = s.position - 2;
        __syncwarp();
        return;
    }
    std::uint32_t v = 0;
    int n_events = 0;
    // the cached pair's position with bit 31 set: the high word of the next cached hit's event
    std::uint32_t cached_word = static_cast<std::uint32_t>(s.cached_pair) | 0x80000000u;
    bool cached = s.cached;
    while (v < count) {
        const unsigned long long window = s.position & ~3ull;
        int r = static_cast<int>(s.position - window);
        curandStatePhilox4_32_10_t state = StateAt(s, window + 4ull * lane);
        const float u0 = curand_uniform(&state);
        const float u1 = curand_uniform(&state);
        const float u2 = curand_uniform(&state);
        const float u3 = curand_uniform(&state);
        const std::uint32_t nibble = (u0 < p ? 1u : 0u) | (u1 < p ? 2u : 0u) | (u2 < p ? 4u : 0u) |
                                     (u3 < p ? 8u : 0u);
        const std::uint32_t shifted = nibble << (4 * (lane & 7));
        const std::uint32_t m0 = __reduce_or_sync(0xffffffffu, (lane >> 3) == 0 ? shifted : 0u);
        const std::uint32_t m1 = __reduce_or_sync(0xffffffffu, (lane >> 3) == 1 ? shifted : 0u);
        const std::uint32_t m2 = __reduce_or_sync(0xffffffffu, (lane >> 3) == 2 ? shifted : 0u);
        const std::uint32_t m3 = __reduce_or_sync(0xffffffffu, (lane >> 3) == 3 ? shifted : 0u);
        const unsigned long long lo = static_cast<unsigned long long>(m0) | (static_cast<unsigned long long>(m1) << 32);
        const unsigned long long hi = static_cast<unsigned long long>(m2) | (static_cast<unsigned long long>(m3) << 32);
        while (v < count && r < 128) {
            const unsigned long long xlo = r < 64 ? (lo & (~0ull << (r & 63))) : 0ull;
            const unsigned long long xhi = r < 64 ? hi : (hi & (~0ull << ((r - 64) & 63)));
            const int h = xlo != 0ull ? __ffsll(static_cast<long long>(xlo)) - 1
                                      : (xhi != 0ull ? 63 + __ffsll(static_cast<long long>(xhi)) : 128);
            const std::uint32_t misses = static_cast<std::uint32_t>(h - r);
            if (misses >= count - v) {
                r += static_cast<int>(count - v);
                v = count;
                break;
            }
            v += misses;
            r = h;
            if (r >= 128) {
                break;
            }
            // value v is hit at draw position window + r
            if (with_normals) {
                const std::uint32_t fresh = static_cast<std::uint32_t>(window) + static_cast<std::uint32_t>(r) + 1u;
                // every lane stores the same word
                ev.packed[n_events] = (static_cast<unsigned long long>(cached ? cached_word : fresh) << 32) | v;
                ++n_events;
                cached_word = cached ? cached_word : (fresh | 0x80000000u);
                cached = !cached;
                r += cached ? 3 : 1;  // (toggled) a fresh pair takes two more positions
            } else {
                r += 1;
            }
            ++v;
        }
        s.position = window + r;
        if (n_events >= kFlushAt) {
            FlushEvents(values, s, sigma, ev, n_events, lane);
        }
    }
    if (n_events > 0) {
        FlushEvents(values, s, sigma, ev, n_events, lane);
    }
    s.cached = cached;
    s.cached_pair = cached_word & 0x7FFFFFFFu;
}

// ---- window-parallel mutation walk ----
//
// The serial walk's only state between draw positions is (offset into the next positions, cached normal held), so
// a run is cut into 128-position windows, one per lane, 32 windows per step: each lane draws its window's
// uniforms, turns them into a 128-bit hit mask and walks it from the two entry states with no position taken
// (cached or not; a window whose first positions were taken by the previous window's last normal pair walks the
// same way unless one of those positions is a hit, which the chain then walks again). A serial chain of 32
// shuffles picks every window's true entry state, a prefix sum of the windows' value counts gives
// each window its first value index, and every lane then walks its own window once more, drawing the normal
// pairs of its hits and applying them. The draws, their order and their arithmetic are the serial walk's.

constexpr unsigned kFullMask = 0xffffffffu;
constexpr std::uint32_t kWindowRunMin = 4096;  // shorter runs take the serial walk

// curand_uniform is non-decreasing in the generator's 32-bit output x, so (curand_uniform < p) <=> (x < threshold).
// Valid for 0 < p < 1 when the largest output's uniform is not below p (ok reports that).
__device__ std::uint32_t UniformThreshold(float p, bool &ok) {
    ok = !(_curand_uniform(0xFFFFFFFFu) < p);
    if (!(_curand_uniform(0u) < p)) {
        return 0u;
    }
    std::uint32_t lo = 0u, hi = 0xFFFFFFFFu;  // uniform(lo) < p <= uniform(hi)
    while (hi - lo > 1u) {
        const std::uint32_t mid = lo + (hi - lo) / 2u;
        if (_curand_uniform(mid) < p) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return hi;
}

// First hit at or after window offset r (0 <= r < 128); 128 when none.
__device__ __forceinline__ int NextHit(unsigned long long lo, unsigned long long hi, int r) {
    const unsigned long long xlo = r < 64 ? (lo & (~0ull << (r & 63))) : 0ull;
    const unsigned long long xhi = r < 64 ? hi : (hi & (~0ull << ((r - 64) & 63)));
    return xlo != 0ull ? __ffsll(static_cast<long long>(xlo)) - 1
                       : (xhi != 0ull ? 63 + __ffsll(static_cast<long long>(xhi)) : 128);
}

// Walks one window from entry state (e positions taken, cached c): every miss and every hit takes one position
// and one value; a hit without a cached normal also takes the next two positions for a fresh pair. Returns the
// exit state (positions of the next window taken + 3 * cached), the values walked, and 1 + the window offset
// of the last fresh pair (0: none drawn).
__device__ __forceinline__ void WalkWindow(unsigned long long lo, unsigned long long hi, int e, bool c,
                                           std::uint32_t &exit_state, std::uint32_t &walked,
                                           std::uint32_t &last_fresh) {
    int r = e;
    int n = 0;
    int lf = 0;
    while (r < 128) {
        const int h = NextHit(lo, hi, r);
        if (h >= 128) {
            n += 128 - r;
            r = 128;
            break;
        }
        n += h - r + 1;
        if (c) {
            c = false;
            r = h + 1;
        } else {
            c = true;
            lf = h + 2;
            r = h + 3;
        }
    }
    exit_state = static_cast<std::uint32_t>(r - 128) + (c ? 3u : 0u);
    walked = static_cast<std::uint32_t>(n);
    last_fresh = static_cast<std::uint32_t>(lf);
}

// The normal pair drawn at `pair`: the generator's curand_normal twice from that position.
__device__ __forceinline__ float2 PairNormals(const Stream &s, unsigned long long pair) {
    curandStatePhilox4_32_10_t state = StateAt(s, pair);
    const float a = curand_normal(&state);
    const float b = curand_normal(&state);
    return make_float2(a, b);
}

__device__ void MutateRunWindows(__half *values, std::uint32_t count, Stream &s, std::uint32_t threshold, float sigma,
                                 int lane) {
    unsigned long long pos = s.position;      // lane 0's window starts here with no position taken
    bool cached = s.cached;
    unsigned long long pair = s.cached_pair;  // the pair whose second value is cached
    std::uint32_t v_base = 0;
    while (v_base < count) {
        // the step's values lie in [v_base, v_base + 4096): their lines reach L2 while the hits are found
        for (std::uint32_t line = v_base / 64u + static_cast<std::uint32_t>(lane); line <= (v_base + 4095u) / 64u;
             line += 32u) {
            if (line * 64u < count) {
                asm volatile("prefetch.L2 [%0];" ::"l"(values + line * 64u));
            }
        }
        const unsigned long long win = pos + 128ull * static_cast<unsigned>(lane);
        const std::uint32_t delta = static_cast<std::uint32_t>(pos & 3ull);
        // ---- pass 1: the window's hit mask, from 33 aligned four-output blocks ----
        std::uint32_t raw0 = 0, raw1 = 0, raw2 = 0, raw3 = 0, raw4 = 0;
        {
            // a block boundary (the mask keeps that visible), so curand4 returns whole blocks
            curandStatePhilox4_32_10_t state = StateAt(s, (win - delta) & ~3ull);
#pragma unroll
            for (int b = 0; b < 33; ++b) {
                const uint4 x = curand4(&state);
                const std::uint32_t nib = (x.x < threshold ? 1u : 0u) | (x.y < threshold ? 2u : 0u) |
                                          (x.z < threshold ? 4u : 0u) | (x.w < threshold ? 8u : 0u);
                const std::uint32_t bits = nib << (4 * (b & 7));
                if (b < 8) {
                    raw0 |= bits;
                } else if (b < 16) {
                    raw1 |= bits;
                } else if (b < 24) {
                    raw2 |= bits;
                } else if (b < 32) {
                    raw3 |= bits;
                } else {
                    raw4 |= bits;
                }
            }
        }
        const unsigned long long lo = static_cast<unsigned long long>(__funnelshift_r(raw0, raw1, delta)) |
                                      (static_cast<unsigned long long>(__funnelshift_r(raw1, raw2, delta)) << 32);
        const unsigned long long hi = static_cast<unsigned long long>(__funnelshift_r(raw2, raw3, delta)) |
                                      (static_cast<unsigned long long>(__funnelshift_r(raw3, raw4, delta)) << 32);
        // ---- the two entry states with no position taken: exits, values walked, last fresh pairs ----
        // A window entered with e > 0 positions taken walks exactly like one entered with none when its first e
        // positions are misses (then it only walks e values fewer); otherwise the chain walks it again.
        std::uint32_t summary = static_cast<std::uint32_t>(lo & 3ull) << 6;  // hits among the first two positions
        std::uint32_t walked01 = 0;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            std::uint32_t x, n, f;
            WalkWindow(lo, hi, 0, c != 0, x, n, f);
            summary |= (x << (3 * c)) | (f << (8 + 8 * c));
            walked01 |= n << (16 * c);
        }
        // ---- the chain: every window's entry state, values walked and the pair cached on entry ----
        std::uint32_t state = cached ? 3u : 0u;
        std::uint32_t my_state = 0, my_walked = 0;
        unsigned long long my_pair = 0;
        for (int l = 0; l < 32; ++l) {
            const std::uint32_t w = __shfl_sync(kFullMask, summary, l);
            const std::uint32_t e = state % 3u;
            const std::uint32_t c = state / 3u;
            std::uint32_t x, n, f;
            if (e != 0u && ((w >> 6) & ((1u << e) - 1u)) != 0u) {
                // a hit among the taken positions: walk window l from its own entry (rare; warp-uniform)
                const unsigned long long lo_l = __shfl_sync(kFullMask, lo, l);
                const unsigned long long hi_l = __shfl_sync(kFullMask, hi, l);
                WalkWindow(lo_l, hi_l, static_cast<int>(e), c != 0u, x, n, f);
            } else {
                x = (w >> (3u * c)) & 7u;
                f = (w >> (8u + 8u * c)) & 0xFFu;
                n = ((walked01 >> (16u * c)) & 0xFFFFu) - e;  // meaningful on lane l only
            }
            if (lane == l) {
                my_state = state;
                my_pair = pair;
                my_walked = n;
            }
            if (f != 0u) {
                pair = pos + 128ull * static_cast<unsigned>(l) + (f - 1u);
            }
            state = x;
        }
        std::uint32_t inclusive = my_walked;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const std::uint32_t t = __shfl_up_sync(kFullMask, inclusive, d);
            if (lane >= d) {
                inclusive += t;
            }
        }
        const std::uint32_t total = __shfl_sync(kFullMask, inclusive, 31);
        const std::uint32_t v0 = v_base + (inclusive - my_walked);
        // ---- pass 2: this window's hits get their normals, one fresh pair and its cached second per trip ----
        const std::uint32_t limit = min(count, v0 + my_walked);
        int r = static_cast<int>(my_state % 3u);
        bool c = my_state >= 3u;
        unsigned long long lane_pair = my_pair;
        std::uint32_t v = v0;
        // Advances over the misses before the next hit; false when the lane's values end first.
        auto to_next_hit = [&](int &h) {
            h = NextHit(lo, hi, r);
            const std::uint32_t misses = static_cast<std::uint32_t>((h < 128 ? h : 128) - r);
            if (misses >= limit - v) {
                r += static_cast<int>(limit - v);
                v = limit;
                return false;
            }
            v += misses;
            return true;
        };
        auto apply = [&](float n) {
            values[v] = __float2half(__fmaf_rn(sigma, n, __half2float(values[v])));
            ++v;
        };
        int h = 0;
        if (c && v < limit && to_next_hit(h)) {  // the window's first hit takes the pair cached on entry
            apply(PairNormals(s, lane_pair).y);
            c = false;
            r = h + 1;
        }
        while (!c && v < limit && to_next_hit(h)) {
            // both values of the pair are found and loaded before its normals are computed
            const std::uint32_t v1 = v;
            const float old1 = __half2float(values[v1]);
            ++v;
            lane_pair = win + static_cast<unsigned long long>(h + 1);
            c = true;
            r = h + 3;
            std::uint32_t v2 = 0xFFFFFFFFu;
            float old2 = 0.0f;
            if (v < limit && to_next_hit(h)) {
                v2 = v;
                old2 = __half2float(values[v2]);
                ++v;
                c = false;
                r = h + 1;
            }
            const float2 nn = PairNormals(s, lane_pair);
            values[v1] = __float2half(__fmaf_rn(sigma, nn.x, old1));
            if (v2 != 0xFFFFFFFFu) {
                values[v2] = __float2half(__fmaf_rn(sigma, nn.y, old2));
            }
        }
        // ---- the stream state after this step ----
        const unsigned end_lanes = __ballot_sync(kFullMask, v0 < count && count <= v0 + my_walked);
        if (end_lanes != 0u) {
            const int L = __ffs(static_cast<int>(end_lanes)) - 1;
            const unsigned long long end_pos = win + static_cast<unsigned long long>(r);
            s.position = __shfl_sync(kFullMask, end_pos, L);
            s.cached = __shfl_sync(kFullMask, c ? 1 : 0, L) != 0;
            s.cached_pair = __shfl_sync(kFullMask, lane_pair, L);
            __syncwarp();
            return;
        }
        pos += 128ull * 32ull + state % 3u;
        cached = state >= 3u;
        v_base += total;
    }
    // count == 0 never reaches here with work done; the stream is unchanged
    s.position = pos;
    s.cached = cached;
    s.cached_pair = pair;
}

__device__ void CopyRegion(std::uint8_t *__restrict__ dst, const std::uint8_t *__restrict__ src, std::size_t bytes,
                           int lane) {

    const std::size_t n16 = bytes / 16;
    uint4 *d = reinterpret_cast<uint4 *>(dst);
    const uint4 *s = reinterpret_cast<const uint4 *>(src);
    std::size_t i = lane;
    for (; i + 96 < n16; i += 128) {
        const uint4 a = s[i];
        const uint4 b = s[i + 32];
        const uint4 c = s[i + 64];
        const uint4 e = s[i + 96];
        d[i] = a;
        d[i + 32] = b;
        d[i + 64] = c;
        d[i + 96] = e;
    }
    for (; i < n16; i += 32) {
        d[i] = s[i];
    }
    const std::size_t halfs = bytes / 2;
    std::uint16_t *d16 = reinterpret_cast<std::uint16_t *>(dst);
    const std::uint16_t *s16 = reinterpret_cast<const std::uint16_t *>(src);
    for (std::size_t k = n16 * 8 + lane; k < halfs; k += 32) {
        d16[k] = s16[k];
    }
}

// kWarps children per CTA (one warp each); the child images do not depend on it. Four-warp CTAs hold 28 children
// per SM at 72 registers, so 4,096 children fit in one wave of 148 SMs.
template <int kWarps>
__global__ void __launch_bounds__(kWarps * 32, kWarps == 4 ? 7 : 32 / kWarps) BreedKernel(const BreedParams p) {
    __shared__ EventList events[kWarps];
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const std::uint32_t child = blockIdx.x * kWarps + warp;
    if (child >= p.child_count) {
        return;
    }
    EventList &ev = events[warp];
    const std::uint32_t first_index = p.pairs[2 * child];
    const std::uint32_t second_index = p.pairs[2 * child + 1];
    const std::uint8_t *parent1 = p.parent_slab + static_cast<std::size_t>(p.parent_slots[first_index]) * p.parent_pitch;
    const std::uint8_t *parent2 =
        p.parent_slab + static_cast<std::size_t>(p.parent_slots[second_index]) * p.parent_pitch;
    const std::uint32_t child_slot = p.child_slots != nullptr ? p.child_slots[child] : child;
    std::uint8_t *out = p.child_slab + static_cast<std::size_t>(child_slot) * p.child_pitch;

    Stream s;
    s.seed = p.generation_seed;
    s.subsequence = static_cast<std::uint32_t>(p.child_first + child + p.generation_index * 4099u);
    s.position = 0;
    s.cached = false;
    s.cached_pair = 0;

    // ---- policy recombination decisions (genome_ops.cuh:264-299, :210-221, :259-262) ----
    bool from_first[5];
    int neuron[5];
    for (int group = 0; group < 2; ++group) {
        const bool base_first = !DrawBernoulli(s, p.crossover_l1);
        const int begin = group == 0 ? 0 : 2;
        const int end = group == 0 ? 2 : 5;
        for (int l = begin; l < end; ++l) {
            from_first[l] = DrawBernoulli(s, p.crossover_l2) ? !base_first : base_first;
            neuron[l] = DrawBernoulli(s, p.crossover_l3) ? static_cast<int>(DrawIndex(s, kLayers[l].outputs)) : -1;
        }
    }
    for (int l = 0; l < 5; ++l) {
        const LayerSpan layer = kLayers[l];
        const std::size_t begin = static_cast<std::size_t>(layer.weights) * 2;
        const std::size_t end = static_cast<std::size_t>(layer.biases + layer.outputs) * 2;
        CopyRegion(out + begin, (from_first[l] ? parent1 : parent2) + begin, end - begin, lane);
    }
    __syncwarp();
    for (int l = 0; l < 5; ++l) {
        if (neuron[l] < 0) {
            continue;
        }
        const LayerSpan layer = kLayers[l];
        const __half *other = reinterpret_cast<const __half *>(from_first[l] ? parent2 : parent1);
        __half *dst = reinterpret_cast<__half *>(out);
        const int row = layer.weights + neuron[l] * layer.fan_in;
        for (int k = lane; k < layer.fan_in; k += 32) {
            dst[row + k] = other[row + k];
        }
        if (lane == 0) {
            dst[layer.biases + neuron[l]] = other[layer.biases + neuron[l]];
        }
    }
    __syncwarp();

    // ---- policy mutation (genome_ops.cuh:153-167, :301-309): skipped entirely when p <= 0 or sigma <= 0 ----
    __half *values = reinterpret_cast<__half *>(out);
    bool windows_ok = false;
    const std::uint32_t threshold = p.mutation_probability > 0.0f && p.mutation_probability < 1.0f
                                        ? UniformThreshold(p.mutation_probability, windows_ok)
                                        : 0u;
    if (p.mutation_probability > 0.0f && p.mutation_sigma > 0.0f) {
        if (windows_ok && kPolicyHalfs >= kWindowRunMin) {
            MutateRunWindows(values, kPolicyHalfs, s, threshold, p.mutation_sigma, lane);
        } else {
            MutateRun(values, kPolicyHalfs, s, p.mutation_probability, p.mutation_sigma, true, ev, lane);
        }
    }

    // ---- tail rows (genome_ops.cuh:344-376) ----
    const std::uint32_t a_count = p.action_count;
    const bool rows_first = !DrawBernoulli(s, p.crossover_l1);
    CopyRegion(out + kTailOffsetBytes, (rows_first ? parent1 : parent2) + kTailOffsetBytes, a_count * kTailRowBytes,
               lane);
    __syncwarp();
    const __half *t1 = reinterpret_cast<const __half *>(parent1 + kTailOffsetBytes);
    const __half *t2 = reinterpret_cast<const __half *>(parent2 + kTailOffsetBytes);
    __half *tc = reinterpret_cast<__half *>(out + kTailOffsetBytes);
    bool has_swap = false;
    std::uint32_t swap_index = 0;
    if (a_count > 0 && DrawBernoulli(s, p.crossover_l2)) {
        has_swap = true;
        swap_index = DrawIndex(s, a_count);
        const __half *src = rows_first ? t2 : t1;
        for (int k = lane; k < kTailDim; k += 32) {
            tc[swap_index * kTailDim + k] = src[swap_index * kTailDim + k];
        }
    }
    __syncwarp();
    if (a_count > 0 && DrawBernoulli(s, p.crossover_l3)) {
        const std::uint32_t splice = DrawIndex(s, a_count);
        const bool row_first = (has_swap && splice == swap_index) ? !rows_first : rows_first;
        const std::uint32_t point = 1 + DrawIndex(s, kTailDim - 1);  // genome_ops.cuh:335-342
        for (int k = lane; k < kTailDim; k += 32) {
            const bool take_first = (static_cast<std::uint32_t>(k) < point) ? row_first : !row_first;
            tc[splice * kTailDim + k] = take_first ? t1[splice * kTailDim + k] : t2[splice * kTailDim + k];
        }
    }
    __syncwarp();

    // ---- tail mutation (genome_ops.cuh:237-257, :378-384) ----
    const bool with_normals = p.mutation_sigma > 0.0f;
    if (p.row_scale_probability <= 0.0f) {
        if (windows_ok && with_normals && a_count * kTailDim >= kWindowRunMin) {
            MutateRunWindows(tc, a_count * kTailDim, s, threshold, p.mutation_sigma, lane);
        } else {
            MutateRun(tc, a_count * kTailDim, s, p.mutation_probability, p.mutation_sigma, with_normals, ev, lane);
        }
    } else {
        for (std::uint32_t row = 0; row < a_count; ++row) {
            MutateRun(tc + row * kTailDim, kTailDim, s, p.mutation_probability, p.mutation_sigma, with_normals, ev,
                      lane);
            if (DrawBernoulli(s, p.row_scale_probability)) {
                const float scale = DrawBernoulli(s, 0.5f) ? 1.02f : 0.98f;  // output_tail_ops.hpp:7-12
                for (int k = lane; k < kTailDim; k += 32) {
                    tc[row * kTailDim + k] = __float2half(__half2float(tc[row * kTailDim + k]) * scale);
                }
            }
            __syncwarp();
        }
    }
}

}  // namespace

cudaError_t LaunchBreed(const BreedParams &params, cudaStream_t stream, int warps_per_cta) {
    if (params.child_count == 0) {
        return cudaSuccess;
    }
    // a child's draw positions: at most three per genome value plus the crossover draws, below 2^31
    const unsigned long long values =
        static_cast<unsigned long long>(kPolicyHalfs) + static_cast<unsigned long long>(kTailDim) * params.action_count;
    if (3ull * values + 64ull >= (1ull << 31)) {
        return cudaErrorInvalidValue;
    }
    switch (warps_per_cta) {
        case 8:
            BreedKernel<8><<<(params.child_count + 7) / 8, 8 * 32, 0, stream>>>(params);
            break;
        case 16:
            BreedKernel<16><<<(params.child_count + 15) / 16, 16 * 32, 0, stream>>>(params);
            break;
        default:
            BreedKernel<4><<<(params.child_count + 3) / 4, 4 * 32, 0, stream>>>(params);
            break;
    }
    return cudaGetLastError();
}

}  // namespace nwg
