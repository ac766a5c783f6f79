// Generation-0 genomes: He-normal FP16 weights, zero biases, N(0, 0.05) tail rows.
//
// Replaces BootstrapRandomGenerationKernel (genotype_slab/device_runtime.cu:258-314) with
// InitializeRandomGenome (genetic_algorithm/device/genome_ops.cuh:100-143). The random-stream map is
// the reference's: virtual thread t of organism o draws from (seed, (g * P + o) * 256 + t) and fills
// elements t, t + 256, ... of each buffer in struct order, so the images are bit-identical. Organism o
// is written to its planned slot; no slot allocation happens on the device.
#include <cuda_fp16.h>
#include <curand_kernel.h>

#include "nwg_internal.cuh"

namespace nwg {
namespace {

constexpr int kBootstrapThreads = 256;

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

// Organism i of this launch is organism organism_first + i of a population of stream_population (a row band of a
// larger grid draws the streams of its own rows).
__global__ void __launch_bounds__(kBootstrapThreads) BootstrapKernel(std::uint8_t *slab, std::size_t pitch,
                                                                     const std::uint32_t *slots,
                                                                     std::uint32_t population,
                                                                     std::uint64_t generation_index,
                                                                     std::uint32_t seed, std::uint32_t action_count,
                                                                     std::uint32_t organism_first,
                                                                     std::uint32_t stream_population) {
    const std::uint32_t organism = blockIdx.x;
    if (organism >= population) {
        return;
    }
    const std::uint32_t slot = slots != nullptr ? slots[organism] : organism;
    __half *genome = reinterpret_cast<__half *>(slab + static_cast<std::size_t>(slot) * pitch);
    const std::uint64_t stream =
        ((generation_index * static_cast<std::uint64_t>(stream_population) + organism_first + organism) *
         kBootstrapThreads) +
        threadIdx.x;
    curandStatePhilox4_32_10_t state;
    curand_init(static_cast<unsigned long long>(seed), stream, 0ULL, &state);
    for (int l = 0; l < 5; ++l) {
        const LayerSpan layer = kLayers[l];
        // genome_ops.cuh:61-63: gain * sqrt(2 / fan_in), gain 1
        const float stddev = 1.0f * sqrtf(2.0f / static_cast<float>(layer.fan_in));
        const int size = layer.fan_in * layer.outputs;
        for (int i = threadIdx.x; i < size; i += kBootstrapThreads) {
            genome[layer.weights + i] = __float2half(stddev * curand_normal(&state));
        }
        for (int i = threadIdx.x; i < layer.outputs; i += kBootstrapThreads) {
            genome[layer.biases + i] = __float2half(0.0f);
        }
    }
    const std::uint32_t tail_values = action_count * kTailDim;
    for (std::uint32_t i = threadIdx.x; i < tail_values; i += kBootstrapThreads) {
        genome[kPolicyHalfs + i] = __float2half(0.05f * curand_normal(&state));
    }
}

}  // namespace

cudaError_t LaunchBootstrap(std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                            std::uint32_t population, std::uint64_t generation_index, std::uint32_t seed,
                            std::uint32_t action_count, cudaStream_t stream, std::uint32_t organism_first,
                            std::uint32_t stream_population) {
    if (population == 0) {
        return cudaSuccess;
    }
    if (stream_population == 0) {
        stream_population = population;
    }
    BootstrapKernel<<<population, kBootstrapThreads, 0, stream>>>(slab, pitch, slots, population, generation_index,
                                                                   seed, action_count, organism_first,
                                                                   stream_population);
    return cudaGetLastError();
}

}  // namespace nwg
