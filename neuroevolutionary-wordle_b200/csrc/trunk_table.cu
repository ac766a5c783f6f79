// Per-individual exact trunk tables: the genome's encoder and trunk weights re-laid out for the streamed FP32 path
// (trunk_fp32.cuh), built once per evaluation from the current slab.
//
// Every weight matrix is stored as [input][output] (the order the register-tiled FP32 micro-kernel reads B in), the
// trunk's layer-1 weights split into its five 64-input turn slots (inputs 1 + 64u .. 64 + 64u; input 0, the virgin
// flag, stays in the genome). The values are the genome's FP16 values converted to FP32 exactly (W_e1 stays FP16:
// the encoder only gathers from it). Each CTA transposes 32 x 32 blocks through shared memory: rows of the genome
// are read contiguously, rows of the table written contiguously.
#include <cuda_fp16.h>

#include "trunk_fp32.cuh"

namespace nwg {
namespace {

using namespace evalx;

struct XtJob {
    int src;   // genome half offset of W[0][first input]
    int ld;    // the genome matrix's row length (its inputs)
    int K;     // inputs copied
    int N;     // outputs
    int dst;   // byte offset in the table
    int fp16;  // 1: the table keeps FP16
};

__device__ __forceinline__ XtJob JobOf(int j) {
    if (j == 0) {
        return {kEncW1, kTurnFeatures, kTurnFeatures, kEncoderHidden, kXtWe1, 1};
    }
    if (j == 1) {
        return {kEncW2, kEncoderHidden, kEncoderHidden, kEncoderOut, kXtWe2, 0};
    }
    if (j < 7) {
        const int u = j - 2;
        return {kTrW1 + 1 + kEncoderOut * u, kModelInput, kEncoderOut, kHidden0, kXtW1 + u * kXtW1Turn, 0};
    }
    if (j == 7) {
        return {kTrW2, kHidden0, kHidden0, kHidden1, kXtW2, 0};
    }
    return {kTrW3, kHidden1, kHidden1, kPolicy, kXtW3, 0};
}

// 32 x 32 blocks of each job in job order: W_e1 5 x 4, W_e2 4 x 2, five W1 slots 2 x 8 each, W2 8 x 4, W3 4 x 2.
constexpr int kXtJobs = 9;
constexpr int kXtBlocks = 20 + 8 + 5 * 16 + 32 + 8;

__global__ void __launch_bounds__(256) BuildExactTrunkTablesKernel(const std::uint8_t *slab, std::size_t pitch,
                                                                   const std::uint32_t *slots, std::uint8_t *tables,
                                                                   std::size_t table_pitch) {
    __shared__ float tile[32][33];
    const std::uint32_t ind = blockIdx.y;
    const __half *gh = reinterpret_cast<const __half *>(slab + static_cast<std::size_t>(slots[ind]) * pitch);
    std::uint8_t *table = tables + static_cast<std::size_t>(ind) * table_pitch;
    int b = static_cast<int>(blockIdx.x);
    int j = 0;
    XtJob job = JobOf(0);
    for (; j < kXtJobs; ++j) {
        job = JobOf(j);
        const int blocks = ((job.K + 31) / 32) * (job.N / 32);
        if (b < blocks) {
            break;
        }
        b -= blocks;
    }
    const int kb = (b / (job.N / 32)) * 32;
    const int nb = (b % (job.N / 32)) * 32;
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int n = e >> 5;
        const int k = e & 31;
        tile[n][k] = kb + k < job.K ? __half2float(gh[job.src + (nb + n) * job.ld + kb + k]) : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int k = e >> 5;
        const int n = e & 31;
        if (kb + k < job.K) {
            const std::size_t idx = static_cast<std::size_t>(kb + k) * job.N + nb + n;
            if (job.fp16) {
                reinterpret_cast<__half *>(table + job.dst)[idx] = __float2half_rn(tile[n][k]);
            } else {
                reinterpret_cast<float *>(table + job.dst)[idx] = tile[n][k];
            }
        }
    }
}

}  // namespace

std::size_t ExactTrunkTablePitch() { return kXtBytes; }

cudaError_t LaunchBuildExactTrunkTables(const std::uint8_t *slab, std::size_t pitch, const std::uint32_t *slots,
                                        std::uint32_t population, std::uint8_t *tables, cudaStream_t stream) {
    if (population == 0) {
        return cudaSuccess;
    }
    BuildExactTrunkTablesKernel<<<dim3(kXtBlocks, population), 256, 0, stream>>>(slab, pitch, slots, tables,
                                                                                   kXtBytes);
    return cudaGetLastError();
}

}  // namespace nwg
