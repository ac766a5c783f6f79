// Random-draw tapes for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (built into oracle/_lib/libnwg_tape.so). The oracle
// restates the reference's breeding, selection and bootstrap control flow on the
// CPU but never recomputes the toolkit generator's output transforms; instead it
// replays the values recorded here, where the generator itself is called on the GPU
// exactly as the reference calls it (genetic_algorithm/device/genome_ops.cuh:17-56).
#include <cuda_runtime.h>
#include <curand_kernel.h>

#include <cstddef>
#include <cstdint>

namespace {

// Position j of stream (seed, subsequence): the raw 32-bit output, the uniform made
// from it, and the two normals made from outputs j and j+1.
__global__ void PositionTapeKernel(std::uint32_t seed, unsigned long long subsequence, std::size_t length,
                                   std::uint32_t *raw, float *uniform, float *normal_pair) {
    const std::size_t j = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= length) {
        return;
    }
    curandStatePhilox4_32_10_t base;
    curand_init(static_cast<unsigned long long>(seed), subsequence, static_cast<unsigned long long>(j), &base);
    curandStatePhilox4_32_10_t state = base;
    raw[j] = curand(&state);
    state = base;
    uniform[j] = curand_uniform(&state);
    state = base;
    normal_pair[2 * j] = curand_normal(&state);
    normal_pair[2 * j + 1] = curand_normal(&state);
}

// Sequential normals of streams (seed, first_subsequence + t), t = 0..stream_count-1.
__global__ void NormalStreamKernel(std::uint32_t seed, unsigned long long first_subsequence, std::size_t stream_count,
                                   std::size_t per_stream, float *out) {
    const std::size_t t = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= stream_count) {
        return;
    }
    curandStatePhilox4_32_10_t state;
    curand_init(static_cast<unsigned long long>(seed), first_subsequence + t, 0ULL, &state);
    for (std::size_t k = 0; k < per_stream; ++k) {
        out[t * per_stream + k] = curand_normal(&state);
    }
}

// The six draws of one child's parent selection (selection_ops.cuh:63-66,120,142):
// u32, u32, uniform, u32, u32, uniform on stream (seed, (uint32)(child + g * 8191)).
__global__ void SelectionDrawsKernel(std::uint32_t seed, std::size_t generation_index, std::size_t child_count,
                                     std::uint32_t *draws) {
    const std::size_t child = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (child >= child_count) {
        return;
    }
    curandStatePhilox4_32_10_t state;
    curand_init(static_cast<unsigned long long>(seed),
                static_cast<unsigned long long>(static_cast<std::uint32_t>(child + generation_index * 8191U)), 0ULL,
                &state);
    std::uint32_t *d = draws + 6 * child;
    d[0] = curand(&state);
    d[1] = curand(&state);
    d[2] = __float_as_uint(curand_uniform(&state));
    d[3] = curand(&state);
    d[4] = curand(&state);
    d[5] = __float_as_uint(curand_uniform(&state));
}

__global__ void PowTableKernel(float exponent, std::size_t count, float *out) {
    const std::size_t r = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (r < count) {
        out[r] = powf(static_cast<float>(r), exponent);
    }
}

} // namespace

extern "C" {

int tape_positions(std::uint32_t seed, unsigned long long subsequence, std::size_t length, std::uint32_t *raw,
                   float *uniform, float *normal_pair) {
    PositionTapeKernel<<<static_cast<unsigned>((length + 255) / 256), 256>>>(seed, subsequence, length, raw, uniform,
                                                                           normal_pair);
    return (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess) ? 1 : 0;
}

int tape_normal_streams(std::uint32_t seed, unsigned long long first_subsequence, std::size_t stream_count,
                        std::size_t per_stream, float *out) {
    NormalStreamKernel<<<static_cast<unsigned>((stream_count + 127) / 128), 128>>>(seed, first_subsequence,
                                                                                  stream_count, per_stream, out);
    return (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess) ? 1 : 0;
}

int tape_selection_draws(std::uint32_t seed, std::size_t generation_index, std::size_t child_count,
                         std::uint32_t *draws) {
    SelectionDrawsKernel<<<static_cast<unsigned>((child_count + 127) / 128), 128>>>(seed, generation_index,
                                                                                   child_count, draws);
    return (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess) ? 1 : 0;
}

int tape_pow_table(float exponent, std::size_t count, float *out) {
    PowTableKernel<<<static_cast<unsigned>((count + 127) / 128), 128>>>(exponent, count, out);
    return (cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess) ? 1 : 0;
}

} // extern "C"
