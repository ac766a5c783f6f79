// Per-individual exact trunk tables: the genome's encoder and trunk weights re-laid out for the streamed FP32 path
// (trunk_fp32.cuh), built once per evaluation from the current slab.
//
// Every weight matrix is stored as [input][output] (the order the register-tiled FP32 micro-kernel reads B in), the
// trunk's layer-1 weights split into its five 64-input turn slots (inputs 1 + 64u .. 64 + 64u; input 0, the virgin
// flag, stays in the genome). The values are the genome's FP16 values converted to FP32 exactly (W_e1 stays FP16:
// the encoder only gathers from it). Each CTA transposes one 64 x 64 block through shared memory: rows of the
// genome are read contiguously (the genome's rows have odd lengths, so two bytes at a time), rows of the table
// written contiguously, 16 bytes per thread for the FP32 matrices.
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

// 64 x 64 blocks of each job in job order: W_e1 3 x 2, W_e2 2 x 1, five W1 slots 1 x 4 each, W2 4 x 2, W3 2 x 1.
constexpr int kXtJobs = 9;
constexpr int kXtBlock = 64;
constexpr int kXtBlocks = 6 + 2 + 5 * 4 + 8 + 2;

__global__ void __launch_bounds__(256) BuildExactTrunkTablesKernel(const std::uint8_t *slab, std::size_t pitch,
                                                                   const std::uint32_t *slots, std::uint8_t *tables,
                                                                   std::size_t table_pitch) {
    constexpr int kTileLd = kXtBlock + 1;
    __shared__ float tile[kXtBlock * kTileLd];  // [output n][input k]
    const std::uint32_t ind = blockIdx.y;
    const __half *gh = reinterpret_cast<const __half *>(slab + static_cast<std::size_t>(slots[ind]) * pitch);
    std::uint8_t *table = tables + static_cast<std::size_t>(ind) * table_pitch;
    int b = static_cast<int>(blockIdx.x);
    int j = 0;
    XtJob job = JobOf(0);
    for (; j < kXtJobs; ++j) {
        job = JobOf(j);
        const int blocks = ((job.K + kXtBlock - 1) / kXtBlock) * (job.N / kXtBlock);
        if (b < blocks) {
            break;
        }
        b -= blocks;
    }
    const int kb = (b / (job.N / kXtBlock)) * kXtBlock;
    const int nb = (b % (job.N / kXtBlock)) * kXtBlock;
    const int rows = job.K - kb < kXtBlock ? job.K - kb : kXtBlock;  // inputs of this block
    // every load of the block is issued before the first shared-memory store
    float v[kXtBlock * kXtBlock / 256];
#pragma unroll
    for (int i = 0; i < kXtBlock * kXtBlock / 256; ++i) {
        const int e = static_cast<int>(threadIdx.x) + i * 256;
        const int n = e >> 6;
        const int k = e & (kXtBlock - 1);
        v[i] = k < rows ? __half2float(gh[job.src + (nb + n) * job.ld + kb + k]) : 0.0f;
    }
#pragma unroll
    for (int i = 0; i < kXtBlock * kXtBlock / 256; ++i) {
        const int e = static_cast<int>(threadIdx.x) + i * 256;
        tile[(e >> 6) * kTileLd + (e & (kXtBlock - 1))] = v[i];
    }
    __syncthreads();
    if (job.fp16) {
        __half *out = reinterpret_cast<__half *>(table + job.dst);
        for (int e = static_cast<int>(threadIdx.x); e < rows * kXtBlock; e += 256) {
            const int k = e >> 6;
            const int n = e & (kXtBlock - 1);
            out[static_cast<std::size_t>(kb + k) * job.N + nb + n] = __float2half_rn(tile[n * kTileLd + k]);
        }
    } else {
        float *out = reinterpret_cast<float *>(table + job.dst);
        for (int e = static_cast<int>(threadIdx.x); e < rows * (kXtBlock / 4); e += 256) {
            const int k = e >> 4;
            const int n = (e & 15) * 4;
            const float4 w = make_float4(tile[n * kTileLd + k], tile[(n + 1) * kTileLd + k],
                                         tile[(n + 2) * kTileLd + k], tile[(n + 3) * kTileLd + k]);
            *reinterpret_cast<float4 *>(out + static_cast<std::size_t>(kb + k) * job.N + nb + n) = w;
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
