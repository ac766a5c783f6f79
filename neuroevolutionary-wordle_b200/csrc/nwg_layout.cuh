// Genome byte image, catalog and shard formats shared by every kernel.
//
// The genome image is the reference's frozen layout (genetic_algorithm/genome/dynamic_layout.hpp:26-71,
// model/policy_model/policy_model.hpp:9-12): FP16 encoder, trunk and tail parameters in struct
// declaration order, weights row-major by output neuron. Slots in the device slab are placed at a
// 256-byte pitch so every parameter block starts 16-byte aligned; the image inside a slot is
// byte-identical to the reference's `slot_stride_bytes` image.
#pragma once

#include <cstddef>
#include <cstdint>

namespace nwg {

constexpr int kWordLength = 5;
constexpr int kAlphabet = 26;
constexpr int kTurnFeatures = 145;   // 5x26 letter one-hot + 5x3 tile one-hot
constexpr int kEncoderHidden = 128;
constexpr int kEncoderOut = 64;
constexpr int kModelInput = 321;     // virgin flag + 5 turn slots of 64
constexpr int kHidden0 = 256;
constexpr int kHidden1 = 128;
constexpr int kPolicy = 64;
constexpr int kFixedDim = 26;
constexpr int kTailDim = 38;
constexpr int kMaxTurns = 6;

// Offsets in halfs inside the genome image.
constexpr int kEncW1 = 0;
constexpr int kEncB1 = 18560;
constexpr int kEncW2 = 18688;
constexpr int kEncB2 = 26880;
constexpr int kTrW1 = 26944;
constexpr int kTrB1 = 109120;
constexpr int kTrW2 = 109376;
constexpr int kTrB2 = 142144;
constexpr int kTrW3 = 142272;
constexpr int kTrB3 = 150464;
constexpr int kPolicyHalfs = 150528;
constexpr std::size_t kTailOffsetBytes = 301056;
constexpr std::size_t kTailRowBytes = 76;
constexpr std::size_t kSlotPitchAlign = 256;

// dynamic_layout.hpp:30-36
__host__ __device__ constexpr std::size_t GenomeStrideBytes(std::size_t action_count) {
    return action_count == 0 ? 0 : ((kTailOffsetBytes + action_count * kTailRowBytes + 1) / 2) * 2;
}

__host__ __device__ constexpr std::size_t SlotPitchBytes(std::size_t action_count) {
    return ((GenomeStrideBytes(action_count) + kSlotPitchAlign - 1) / kSlotPitchAlign) * kSlotPitchAlign;
}

// Packed 5-letter word code: letter p (0..25) in bits [5p, 5p+5).
__host__ __device__ constexpr std::uint32_t PackWord(const std::uint8_t *letters) {
    return static_cast<std::uint32_t>(letters[0]) | (static_cast<std::uint32_t>(letters[1]) << 5) |
           (static_cast<std::uint32_t>(letters[2]) << 10) | (static_cast<std::uint32_t>(letters[3]) << 15) |
           (static_cast<std::uint32_t>(letters[4]) << 20);
}

__host__ __device__ constexpr std::uint32_t WordLetter(std::uint32_t code, int position) {
    return (code >> (5 * position)) & 31u;
}

// Training-data shard record, byte-compatible with the reference's TrainingDataShardRuntime
// (training_folder/training_data.hpp:35-42).
struct ShardRecord {
    std::uint64_t first_catalog_word_index;
    std::uint64_t word_count;
    std::uint64_t center_row;
    std::uint64_t center_column;
    std::uint64_t radius;
    std::uint8_t global_from_outset;
};
static_assert(sizeof(ShardRecord) == 48, "shard record must match the reference layout");

constexpr std::uint64_t kCatalogCapacity = 4739;  // training_data.hpp:22

// Wordle tile states (wordle/feedback.hpp:13-17).
constexpr std::uint32_t kGreen = 0;
constexpr std::uint32_t kYellow = 1;
constexpr std::uint32_t kGrey = 2;

// Feedback of `guess` against `secret` (wordle/feedback.hpp:103-136): greens first, then yellows
// consumed left to right from the secret's unmatched letters. Two bits per position.
__host__ __device__ inline std::uint32_t FeedbackPacked(std::uint32_t guess, std::uint32_t secret) {
    std::uint32_t green = 0;
    for (int p = 0; p < kWordLength; ++p) {
        green |= (WordLetter(guess, p) == WordLetter(secret, p)) ? (1u << p) : 0u;
    }
    std::uint32_t out = 0;
    for (int p = 0; p < kWordLength; ++p) {
        std::uint32_t tile = kGrey;
        if (green & (1u << p)) {
            tile = kGreen;
        } else {
            const std::uint32_t letter = WordLetter(guess, p);
            int available = 0;
            int earlier = 0;
            for (int q = 0; q < kWordLength; ++q) {
                if (!(green & (1u << q))) {
                    available += WordLetter(secret, q) == letter;
                    earlier += (q < p) && (WordLetter(guess, q) == letter);
                }
            }
            tile = earlier < available ? kYellow : kGrey;
        }
        out |= tile << (2 * p);
    }
    return out;
}

}  // namespace nwg
