// The learned surrogate's network: an MLP 8,192 -> 512 -> 128 -> 1 with GELU, BF16 weights for the products,
// FP32 master weights, FP32 accumulation and Adam; forward, backward and update are this file's own kernels.
//
// The two large products run on the 5th-generation tensor cores: the first layer over a brood of descriptors,
// Z1[rows][512] = X[rows][8192] . W1[512][8192]^T, and its weight gradient, dW1[512][8192] = dZ1^T[512][B] .
// X^T[8192][B]^T. Both are "NT" products of K-major BF16 operands (GemmNtKernel): a CTA owns a 128 x 256 FP32
// accumulator in tensor memory, 64-deep K stages are copied with 16-byte cp.async straight into the canonical
// no-swizzle core-matrix layout (three stages in flight), one thread issues four tcgen05.mma per stage and
// commits to the stage's mbarrier, and every mbarrier wait is bounded (a timeout sets an error flag, the kernel
// drains its MMAs and frees its tensor memory). The small layers (512 -> 128 -> 1), GELU, the loss and the
// column sums of the gradients are FP32 CUDA-core kernels with a fixed summation order (no atomics), so a training
// step is deterministic.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/nwg_capi.h"
#include "nwg_internal.cuh"
#include "umma.cuh"

using namespace nwg;

namespace {

constexpr int kGemmThreads = 128;
constexpr int kBM = 128;
constexpr int kBN = 256;
constexpr int kBK = 64;
constexpr int kStages = 3;
constexpr int kStageABytes = kBM * kBK * 2;  // 16 KB
constexpr int kStageBBytes = kBN * kBK * 2;  // 32 KB
constexpr int kGemmSmem = kStages * (kStageABytes + kStageBBytes) + 1024;
constexpr std::uint32_t kWaitLimit = 1u << 26;

__device__ __forceinline__ void CpAsync16(std::uint32_t smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem), "l"(gmem) : "memory");
}
__device__ __forceinline__ void CpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void CpAsyncWait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// C[M][N] (FP32, row stride ldc) = A[M][K] . B[N][K]^T, A and B BF16 row-major (K contiguous).
// M % 128 == 0, N % 256 == 0, K % 64 == 0; lda, ldb multiples of 8 elements; 16-byte aligned bases.
__global__ void __launch_bounds__(kGemmThreads, 1)
    GemmNtKernel(const __nv_bfloat16 *A, std::size_t lda, const __nv_bfloat16 *B, std::size_t ldb, float *C,
                 std::size_t ldc, int K, int *error) {
    extern __shared__ __align__(1024) std::uint8_t gemm_smem[];
    __shared__ std::uint64_t mbar[kStages];
    __shared__ std::uint32_t tmem_base;
    __shared__ int failed;
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    const std::size_t m0 = static_cast<std::size_t>(blockIdx.y) * kBM;
    const std::size_t n0 = static_cast<std::size_t>(blockIdx.x) * kBN;
    std::uint8_t *base = reinterpret_cast<std::uint8_t *>(
        (reinterpret_cast<std::uintptr_t>(gemm_smem) + 1023u) & ~static_cast<std::uintptr_t>(1023u));
    const std::uint32_t sbase = umma::SmemAddress(base);
    if (tid == 0) {
        failed = 0;
        for (int s = 0; s < kStages; ++s) {
            umma::MbarInit(&mbar[s], 1);
        }
    }
    if (warp == 0) {
        umma::Alloc(&tmem_base, kBN);
    }
    umma::FenceBeforeSync();
    __syncthreads();
    umma::FenceAfterSync();
    const std::uint32_t tmem = tmem_base;
    const int k_tiles = K / kBK;

    // stage s: A tile at sbase + s * (A + B bytes), B tile right after it
    auto load_stage = [&](int kt, int s) {
        const std::uint32_t a_s = sbase + s * (kStageABytes + kStageBBytes);
        const std::uint32_t b_s = a_s + kStageABytes;
        const std::size_t k0 = static_cast<std::size_t>(kt) * kBK;
        for (int c = tid; c < kBM * (kBK / 8); c += kGemmThreads) {
            const int r = c >> 3;
            const int kc = c & 7;
            CpAsync16(a_s + umma::TileOffset(r, kc * 8, kBK), A + (m0 + r) * lda + k0 + kc * 8);
        }
        for (int c = tid; c < kBN * (kBK / 8); c += kGemmThreads) {
            const int r = c >> 3;
            const int kc = c & 7;
            CpAsync16(b_s + umma::TileOffset(r, kc * 8, kBK), B + (n0 + r) * ldb + k0 + kc * 8);
        }
    };
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < k_tiles) {
            load_stage(s, s);
        }
        CpAsyncCommit();
    }
    constexpr std::uint32_t idesc = umma::InstrDescBf16(kBM, kBN);
    std::uint32_t phase[kStages] = {0, 0, 0};
    for (int kt = 0; kt < k_tiles; ++kt) {
        const int s = kt % kStages;
        CpAsyncWait<kStages - 2>();
        umma::FenceProxyAsyncShared();
        __syncthreads();
        if (tid == 0 && failed == 0) {
            umma::FenceAfterSync();
            const std::uint32_t a_s = sbase + s * (kStageABytes + kStageBBytes);
            const std::uint32_t b_s = a_s + kStageABytes;
#pragma unroll
            for (int kk = 0; kk < kBK / 16; ++kk) {
                const std::uint64_t ad = umma::SmemDescriptor(a_s + kk * 256, 128, (kBK / 8) * 128);
                const std::uint64_t bd = umma::SmemDescriptor(b_s + kk * 256, 128, (kBK / 8) * 128);
                umma::Mma(tmem, ad, bd, idesc, kt > 0 || kk > 0);
            }
            umma::Commit(&mbar[s]);
        }
        // refill the stage the previous k-tile used, once its MMAs are done
        const int next = kt + kStages - 1;
        if (kt >= 1) {
            const int sp = (kt - 1) % kStages;
            if (tid == 0 && failed == 0 && !umma::MbarWait(&mbar[sp], phase[sp], kWaitLimit)) {
                failed = 1;
            }
            phase[sp] ^= 1u;
        }
        __syncthreads();
        if (next < k_tiles && failed == 0) {
            load_stage(next, next % kStages);
        }
        CpAsyncCommit();
    }
    // the last k-tile's commit covers every MMA before it
    if (k_tiles > 0) {
        const int sl = (k_tiles - 1) % kStages;
        if (tid == 0 && failed == 0 && !umma::MbarWait(&mbar[sl], phase[sl], kWaitLimit)) {
            failed = 1;
        }
    }
    CpAsyncWait<0>();
    __syncthreads();
    umma::FenceAfterSync();
    if (failed == 0) {
        const std::size_t row = m0 + warp * 32 + (tid & 31);
        float *out = C + row * ldc + n0;
        for (int c0 = 0; c0 < kBN; c0 += 64) {
            float v[64];
            umma::Load64(tmem + (static_cast<std::uint32_t>(warp * 32) << 16) + c0, v);
#pragma unroll
            for (int i = 0; i < 64; i += 4) {
                *reinterpret_cast<float4 *>(out + c0 + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
            }
        }
    } else if (tid == 0) {
        atomicExch(error, 1);
    }
    umma::FenceBeforeSync();
    __syncthreads();
    if (warp == 0) {
        umma::Dealloc(tmem, kBN);
    }
}

__device__ __forceinline__ float Gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float GeluGrad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

constexpr int kH1 = 512;
constexpr int kH2 = 128;
constexpr int kRowsPerBlock = 8;

// Layers 2 and 3 for kRowsPerBlock rows: z1 = Z1 + b1 (in place), a1 = gelu(z1), z2 = b2 + W2 a1, a2 = gelu(z2),
// y = b3 + w3 . a2. Each of the 128 threads owns one z2 output; sums run over inputs in ascending order.
__global__ void __launch_bounds__(kH2) MlpTailForwardKernel(float *Z1, std::size_t rows, const float *b1,
                                                            const float *W2, const float *b2, const float *w3,
                                                            const float *b3, float *A1, float *Z2, float *A2,
                                                            float *y) {
    __shared__ float a1s[kRowsPerBlock][kH1];
    __shared__ float a2s[kRowsPerBlock][kH2];
    const int tid = threadIdx.x;
    const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * kRowsPerBlock;
    for (int idx = tid; idx < kRowsPerBlock * kH1; idx += kH2) {
        const int rr = idx / kH1;
        const int i = idx - rr * kH1;
        const std::size_t r = r0 + rr;
        float a = 0.0f;
        if (r < rows) {
            const float z = Z1[r * kH1 + i] + b1[i];
            Z1[r * kH1 + i] = z;
            a = Gelu(z);
            if (A1 != nullptr) {
                A1[r * kH1 + i] = a;
            }
        }
        a1s[rr][i] = a;
    }
    __syncthreads();
    float acc[kRowsPerBlock];
    for (int rr = 0; rr < kRowsPerBlock; ++rr) {
        acc[rr] = b2[tid];
    }
    const float *w = W2 + static_cast<std::size_t>(tid) * kH1;
    for (int i = 0; i < kH1; ++i) {
        const float wi = w[i];
#pragma unroll
        for (int rr = 0; rr < kRowsPerBlock; ++rr) {
            acc[rr] = fmaf(wi, a1s[rr][i], acc[rr]);
        }
    }
    for (int rr = 0; rr < kRowsPerBlock; ++rr) {
        const std::size_t r = r0 + rr;
        const float a2 = Gelu(acc[rr]);
        a2s[rr][tid] = a2;
        if (r < rows && Z2 != nullptr) {
            Z2[r * kH2 + tid] = acc[rr];
            A2[r * kH2 + tid] = a2;
        }
    }
    __syncthreads();
    if (tid < kRowsPerBlock && r0 + tid < rows) {
        float out = b3[0];
        for (int j = 0; j < kH2; ++j) {
            out = fmaf(w3[j], a2s[tid][j], out);
        }
        y[r0 + tid] = out;
    }
}

// Backward through layers 3 and 2 and the first GELU, for kRowsPerBlock rows of a minibatch of B rows, with the
// loss mean((y - t)^2): dy, dZ2 = (dy w3) * gelu'(z2), dZ1 = (W2^T dZ2) * gelu'(z1); dZ1 also transposed to BF16
// ([512][ldt]) for the tensor-core weight gradient.
__global__ void __launch_bounds__(kH2) MlpTailBackwardKernel(const float *y, const float *t, std::size_t rows,
                                                             float inv_rows, const float *Z1, const float *Z2,
                                                             const float *W2, const float *w3, float *dy,
                                                             float *dZ2, float *dZ1, __nv_bfloat16 *dZ1T,
                                                             std::size_t ldt) {
    __shared__ float dz2s[kRowsPerBlock][kH2];
    const int tid = threadIdx.x;
    const std::size_t r0 = static_cast<std::size_t>(blockIdx.x) * kRowsPerBlock;
    for (int rr = 0; rr < kRowsPerBlock; ++rr) {
        const std::size_t r = r0 + rr;
        float g = 0.0f;
        if (r < rows) {
            const float d = 2.0f * (y[r] - t[r]) * inv_rows;
            if (tid == 0) {
                dy[r] = d;
            }
            g = d * w3[tid] * GeluGrad(Z2[r * kH2 + tid]);
            dZ2[r * kH2 + tid] = g;
        }
        dz2s[rr][tid] = g;
    }
    __syncthreads();
    for (int i = tid; i < kH1; i += kH2) {
        float acc[kRowsPerBlock];
#pragma unroll
        for (int rr = 0; rr < kRowsPerBlock; ++rr) {
            acc[rr] = 0.0f;
        }
        for (int j = 0; j < kH2; ++j) {
            const float w = W2[static_cast<std::size_t>(j) * kH1 + i];
#pragma unroll
            for (int rr = 0; rr < kRowsPerBlock; ++rr) {
                acc[rr] = fmaf(w, dz2s[rr][j], acc[rr]);
            }
        }
        for (int rr = 0; rr < kRowsPerBlock; ++rr) {
            const std::size_t r = r0 + rr;
            if (r < rows) {
                const float g = acc[rr] * GeluGrad(Z1[r * kH1 + i]);
                dZ1[r * kH1 + i] = g;
                dZ1T[static_cast<std::size_t>(i) * ldt + r] = __float2bfloat16_rn(g);
            }
        }
    }
}

// out[j * stride_out] = sum_r a[r * lda + j] * (b ? b[r * ldb + i] : 1), over r ascending: the column sums and the
// small weight gradients (dW2[j][i] = sum_r dZ2[r][j] A1[r][i], db2, dW3, db3, db1).
__global__ void ColumnProductSumKernel(const float *a, std::size_t lda, int a_cols, const float *b, std::size_t ldb,
                                       int b_cols, std::size_t rows, float *out) {
    const std::size_t total = static_cast<std::size_t>(a_cols) * b_cols;
    for (std::size_t o = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; o < total;
         o += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const int j = static_cast<int>(o / b_cols);
        const int i = static_cast<int>(o - static_cast<std::size_t>(j) * b_cols);
        float s = 0.0f;
        for (std::size_t r = 0; r < rows; ++r) {
            s = fmaf(a[r * lda + j], b != nullptr ? b[r * ldb + i] : 1.0f, s);
        }
        out[o] = s;
    }
}

// Adam (bias-corrected) over the flat parameter vector; refreshes the BF16 copy of W1 (the first n_bf16 values).
__global__ void AdamKernel(float *params, const float *grads, float *m, float *v, std::size_t n, float lr,
                           float beta1, float beta2, float eps, float correction1, float correction2,
                           __nv_bfloat16 *w1_bf16, std::size_t n_bf16) {
    for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        const float g = grads[i];
        const float mi = beta1 * m[i] + (1.0f - beta1) * g;
        const float vi = beta2 * v[i] + (1.0f - beta2) * g * g;
        m[i] = mi;
        v[i] = vi;
        const float p = params[i] - lr * (mi / correction1) / (sqrtf(vi / correction2) + eps);
        params[i] = p;
        if (i < n_bf16) {
            w1_bf16[i] = __float2bfloat16_rn(p);
        }
    }
}

__global__ void ToBf16Kernel(const float *in, __nv_bfloat16 *out, std::size_t n) {
    for (std::size_t i = blockIdx.x * static_cast<std::size_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<std::size_t>(gridDim.x) * blockDim.x) {
        out[i] = __float2bfloat16_rn(in[i]);
    }
}

// Transposes rows x cols BF16 (row stride ld_in) into cols x rows (row stride ld_out) through 32 x 32 tiles.
__global__ void TransposeBf16Kernel(const __nv_bfloat16 *in, std::size_t ld_in, std::size_t rows, std::size_t cols,
                                    __nv_bfloat16 *out, std::size_t ld_out) {
    __shared__ __nv_bfloat16 tile[32][33];
    const std::size_t c0 = static_cast<std::size_t>(blockIdx.x) * 32;
    const std::size_t r0 = static_cast<std::size_t>(blockIdx.y) * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const std::size_t r = r0 + k, c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < rows && c < cols) ? in[r * ld_in + c] : __float2bfloat16_rn(0.0f);
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const std::size_t c = c0 + k, r = r0 + threadIdx.x;
        if (c < cols && r < rows) {
            out[c * ld_out + r] = tile[threadIdx.x][k];
        }
    }
}

}  // namespace

namespace nwg {

cudaError_t LaunchGemmNt(const void *a, std::size_t lda, const void *b, std::size_t ldb, float *c, std::size_t ldc,
                         std::size_t m, std::size_t n, std::size_t k, int *error, cudaStream_t stream) {
    static std::atomic<unsigned long long> configured{0};
    if (const cudaError_t e = RaiseSharedLimit(GemmNtKernel, kGemmSmem, configured);
        e != cudaSuccess) {
        return e;
    }
    if (m % kBM != 0 || n % kBN != 0 || k % kBK != 0 || lda % 8 != 0 || ldb % 8 != 0 || ldc % 4 != 0 ||
        (reinterpret_cast<std::uintptr_t>(a) & 15u) != 0 || (reinterpret_cast<std::uintptr_t>(b) & 15u) != 0 ||
        (reinterpret_cast<std::uintptr_t>(c) & 15u) != 0) {
        return cudaErrorInvalidValue;
    }
    if (m == 0 || n == 0) {
        return cudaSuccess;
    }
    const dim3 grid(static_cast<unsigned>(n / kBN), static_cast<unsigned>(m / kBM));
    GemmNtKernel<<<grid, kGemmThreads, kGemmSmem, stream>>>(static_cast<const __nv_bfloat16 *>(a), lda,
                                                            static_cast<const __nv_bfloat16 *>(b), ldb, c, ldc,
                                                            static_cast<int>(k), error);
    return cudaGetLastError();
}

}  // namespace nwg

// ---- the network object ----

struct nwg_mlp {
    cudaStream_t stream = nullptr;
    std::size_t capacity = 0;  // rows a forward or a training step may take (multiple of 128)
    float *params = nullptr;   // flat FP32 masters: W1, b1, W2, b2, w3, b3
    float *grads = nullptr;
    float *adam_m = nullptr;
    float *adam_v = nullptr;
    __nv_bfloat16 *w1_bf16 = nullptr;
    std::uint64_t step = 0;
    float lr = 1.0e-3f, beta1 = 0.9f, beta2 = 0.999f, eps = 1.0e-8f;
    // activations of the last forward, [capacity] rows
    float *Z1 = nullptr, *A1 = nullptr, *Z2 = nullptr, *A2 = nullptr, *y = nullptr;
    float *dy = nullptr, *dZ2 = nullptr, *dZ1 = nullptr;
    __nv_bfloat16 *dZ1T = nullptr, *XT = nullptr;
    int *error = nullptr;
};

namespace {

constexpr std::size_t kW1 = static_cast<std::size_t>(kH1) * kDescriptorWidth;
constexpr std::size_t kOffB1 = kW1;
constexpr std::size_t kOffW2 = kOffB1 + kH1;
constexpr std::size_t kOffB2 = kOffW2 + static_cast<std::size_t>(kH2) * kH1;
constexpr std::size_t kOffW3 = kOffB2 + kH2;
constexpr std::size_t kOffB3 = kOffW3 + kH2;
constexpr std::size_t kParams = kOffB3 + 1;

int GemmStatus(nwg_mlp *m) {
    int e = 0;
    if (cudaMemcpyAsync(&e, m->error, sizeof(int), cudaMemcpyDeviceToHost, m->stream) != cudaSuccess ||
        cudaStreamSynchronize(m->stream) != cudaSuccess) {
        return kCudaFailure;
    }
    return e != 0 ? kTimeout : kOk;
}

// rows is a multiple of 128 (the product reads whole 128-row tiles of x).
int Forward(nwg_mlp *m, const std::uint16_t *x, std::size_t rows, bool keep) {
    const std::size_t padded = rows;
    if (rows % kBM != 0 || padded > m->capacity) {
        return kUnsupported;
    }
    if (LaunchGemmNt(x, kDescriptorWidth, m->w1_bf16, kDescriptorWidth, m->Z1, kH1, padded, kH1, kDescriptorWidth,
                     m->error, m->stream) != cudaSuccess) {
        return kCudaFailure;
    }
    const float *p = m->params;
    const unsigned blocks = static_cast<unsigned>((rows + kRowsPerBlock - 1) / kRowsPerBlock);
    MlpTailForwardKernel<<<blocks, kH2, 0, m->stream>>>(m->Z1, rows, p + kOffB1, p + kOffW2, p + kOffB2, p + kOffW3,
                                                        p + kOffB3, keep ? m->A1 : nullptr, keep ? m->Z2 : nullptr,
                                                        keep ? m->A2 : nullptr, m->y);
    return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

// Gradients of mean((y - t)^2) over rows into m->grads (the rows of the last kept forward).
int Backward(nwg_mlp *m, const std::uint16_t *x, const float *t, std::size_t rows) {
    const std::size_t padded = rows;  // a multiple of 128, checked by Forward
    const float *p = m->params;
    float *g = m->grads;
    cudaStream_t s = m->stream;
    const unsigned blocks = static_cast<unsigned>((rows + kRowsPerBlock - 1) / kRowsPerBlock);
    MlpTailBackwardKernel<<<blocks, kH2, 0, s>>>(m->y, t, rows, 1.0f / static_cast<float>(rows), m->Z1, m->Z2,
                                                 p + kOffW2, p + kOffW3, m->dy, m->dZ2, m->dZ1, m->dZ1T,
                                                 m->capacity);
    const dim3 tb(32, 8);
    const dim3 tg(kDescriptorWidth / 32, static_cast<unsigned>((rows + 31) / 32));
    TransposeBf16Kernel<<<tg, tb, 0, s>>>(reinterpret_cast<const __nv_bfloat16 *>(x), kDescriptorWidth, rows,
                                          kDescriptorWidth, m->XT, m->capacity);
    if (cudaGetLastError() != cudaSuccess ||
        LaunchGemmNt(m->dZ1T, m->capacity, m->XT, m->capacity, g, kDescriptorWidth, kH1, kDescriptorWidth, padded,
                     m->error, s) != cudaSuccess) {
        return kCudaFailure;
    }
    ColumnProductSumKernel<<<256, 256, 0, s>>>(m->dZ1, kH1, kH1, nullptr, 0, 1, rows, g + kOffB1);
    ColumnProductSumKernel<<<256, 256, 0, s>>>(m->dZ2, kH2, kH2, m->A1, kH1, kH1, rows, g + kOffW2);
    ColumnProductSumKernel<<<1, 128, 0, s>>>(m->dZ2, kH2, kH2, nullptr, 0, 1, rows, g + kOffB2);
    ColumnProductSumKernel<<<1, 128, 0, s>>>(m->dy, 1, 1, m->A2, kH2, kH2, rows, g + kOffW3);
    ColumnProductSumKernel<<<1, 32, 0, s>>>(m->dy, 1, 1, nullptr, 0, 1, rows, g + kOffB3);
    return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

void FreeMlp(nwg_mlp *m) {
    if (m == nullptr) {
        return;
    }
    void *ptrs[] = {m->params, m->grads, m->adam_m, m->adam_v, m->w1_bf16, m->Z1,  m->A1,  m->Z2,
                    m->A2,     m->y,     m->dy,     m->dZ2,    m->dZ1,     m->dZ1T, m->XT, m->error};
    for (void *p : ptrs) {
        cudaFree(p);
    }
    delete m;
}

// splitmix64 + Box-Muller: He-style initial weights N(0, 2 / fan_in), zero biases.
std::vector<float> InitialParameters(std::uint32_t seed) {
    std::vector<float> p(kParams, 0.0f);
    std::uint64_t state = 0x6a09e667f3bcc909ULL ^ seed;
    auto next = [&]() {
        std::uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
        return z ^ (z >> 31);
    };
    auto normal = [&]() {
        const double u1 = (static_cast<double>(next() >> 11) + 0.5) / 9007199254740992.0;
        const double u2 = static_cast<double>(next() >> 11) / 9007199254740992.0;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    };
    const auto fill = [&](std::size_t off, std::size_t n, double fan_in) {
        const double s = std::sqrt(2.0 / fan_in);
        for (std::size_t i = 0; i < n; ++i) {
            p[off + i] = static_cast<float>(normal() * s);
        }
    };
    fill(0, kW1, kDescriptorWidth);
    fill(kOffW2, static_cast<std::size_t>(kH2) * kH1, kH1);
    fill(kOffW3, kH2, kH2);
    return p;
}

}  // namespace

extern "C" {

int nwg_mlp_create(size_t capacity_rows, uint32_t seed, float learning_rate, nwg_mlp **out) {
    if (out == nullptr || capacity_rows == 0) {
        return kInvalidRuntimeConfig;
    }
    *out = nullptr;
    nwg_mlp *m = new (std::nothrow) nwg_mlp();
    if (m == nullptr) {
        return kCudaFailure;
    }
    m->capacity = (capacity_rows + kBM - 1) / kBM * kBM;
    m->lr = learning_rate;
    const std::size_t c = m->capacity;
    bool ok = cudaMalloc(&m->params, kParams * 4) == cudaSuccess && cudaMalloc(&m->grads, kParams * 4) == cudaSuccess &&
              cudaMalloc(&m->adam_m, kParams * 4) == cudaSuccess && cudaMalloc(&m->adam_v, kParams * 4) == cudaSuccess &&
              cudaMalloc(&m->w1_bf16, kW1 * 2) == cudaSuccess && cudaMalloc(&m->Z1, c * kH1 * 4) == cudaSuccess &&
              cudaMalloc(&m->A1, c * kH1 * 4) == cudaSuccess && cudaMalloc(&m->Z2, c * kH2 * 4) == cudaSuccess &&
              cudaMalloc(&m->A2, c * kH2 * 4) == cudaSuccess && cudaMalloc(&m->y, c * 4) == cudaSuccess &&
              cudaMalloc(&m->dy, c * 4) == cudaSuccess && cudaMalloc(&m->dZ2, c * kH2 * 4) == cudaSuccess &&
              cudaMalloc(&m->dZ1, c * kH1 * 4) == cudaSuccess && cudaMalloc(&m->dZ1T, c * kH1 * 2) == cudaSuccess &&
              cudaMalloc(&m->XT, c * kDescriptorWidth * 2) == cudaSuccess &&
              cudaMalloc(&m->error, sizeof(int)) == cudaSuccess;
    const std::vector<float> init = InitialParameters(seed);
    ok = ok && cudaMemcpy(m->params, init.data(), kParams * 4, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(m->adam_m, 0, kParams * 4) == cudaSuccess && cudaMemset(m->adam_v, 0, kParams * 4) == cudaSuccess &&
         cudaMemset(m->error, 0, sizeof(int)) == cudaSuccess;
    if (ok) {
        ToBf16Kernel<<<1024, 256>>>(m->params, m->w1_bf16, kW1);
        ok = cudaGetLastError() == cudaSuccess && cudaDeviceSynchronize() == cudaSuccess;
    }
    if (!ok) {
        FreeMlp(m);
        return kCudaFailure;
    }
    *out = m;
    return kOk;
}

void nwg_mlp_destroy(nwg_mlp *m) { FreeMlp(m); }

int nwg_mlp_set_stream(nwg_mlp *m, void *cuda_stream) {
    if (m == nullptr) {
        return kInvalidRuntimeConfig;
    }
    m->stream = static_cast<cudaStream_t>(cuda_stream);
    return kOk;
}

size_t nwg_mlp_parameter_count(void) { return kParams; }

int nwg_mlp_parameters(nwg_mlp *m, float *host_out, const float *host_in) {
    if (m == nullptr) {
        return kInvalidRuntimeConfig;
    }
    if (cudaStreamSynchronize(m->stream) != cudaSuccess ||
        (host_out != nullptr && cudaMemcpy(host_out, m->params, kParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess)) {
        return kCudaFailure;
    }
    if (host_in != nullptr) {
        if (cudaMemcpy(m->params, host_in, kParams * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
            return kCudaFailure;
        }
        ToBf16Kernel<<<1024, 256, 0, m->stream>>>(m->params, m->w1_bf16, kW1);
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(m->stream) != cudaSuccess) {
            return kCudaFailure;
        }
    }
    return kOk;
}

int nwg_mlp_forward(nwg_mlp *m, const uint16_t *x, size_t rows, float *y_out) {
    if (m == nullptr || x == nullptr || y_out == nullptr || rows == 0) {
        return kInvalidRuntimeConfig;
    }
    int st = Forward(m, x, rows, false);
    if (st == kOk && cudaMemcpyAsync(y_out, m->y, rows * 4, cudaMemcpyDeviceToDevice, m->stream) != cudaSuccess) {
        st = kCudaFailure;
    }
    return st == kOk ? GemmStatus(m) : st;
}

int nwg_mlp_gradients(nwg_mlp *m, const uint16_t *x, const float *targets, size_t rows, float *grads_out,
                      float *loss_out) {
    if (m == nullptr || x == nullptr || targets == nullptr || rows == 0) {
        return kInvalidRuntimeConfig;
    }
    int st = Forward(m, x, rows, true);
    if (st == kOk) {
        st = Backward(m, x, targets, rows);
    }
    if (st == kOk) {
        st = GemmStatus(m);
    }
    if (st != kOk) {
        return st;
    }
    if (grads_out != nullptr && cudaMemcpy(grads_out, m->grads, kParams * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
        return kCudaFailure;
    }
    if (loss_out != nullptr) {
        std::vector<float> y(rows), t(rows);
        if (cudaMemcpy(y.data(), m->y, rows * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
            cudaMemcpy(t.data(), targets, rows * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
            return kCudaFailure;
        }
        double loss = 0.0;
        for (std::size_t r = 0; r < rows; ++r) {
            loss += (static_cast<double>(y[r]) - t[r]) * (static_cast<double>(y[r]) - t[r]);
        }
        *loss_out = static_cast<float>(loss / static_cast<double>(rows));
    }
    return kOk;
}

int nwg_mlp_train_step(nwg_mlp *m, const uint16_t *x, const float *targets, size_t rows) {
    if (m == nullptr || x == nullptr || targets == nullptr || rows == 0) {
        return kInvalidRuntimeConfig;
    }
    int st = Forward(m, x, rows, true);
    if (st == kOk) {
        st = Backward(m, x, targets, rows);
    }
    if (st != kOk) {
        return st;
    }
    ++m->step;
    const float c1 = 1.0f - std::pow(m->beta1, static_cast<float>(m->step));
    const float c2 = 1.0f - std::pow(m->beta2, static_cast<float>(m->step));
    AdamKernel<<<2048, 256, 0, m->stream>>>(m->params, m->grads, m->adam_m, m->adam_v, kParams, m->lr, m->beta1,
                                            m->beta2, m->eps, c1, c2, m->w1_bf16, kW1);
    return cudaGetLastError() == cudaSuccess ? kOk : kCudaFailure;
}

int nwg_descriptors(const void *slab, size_t pitch, const uint32_t *slots, size_t count, const uint8_t *probe_letters,
                    const uint8_t *probe_feedback, const uint8_t *probe_turns, float scale, uint16_t *out,
                    void *cuda_stream) {
    if (slab == nullptr || slots == nullptr || out == nullptr || probe_letters == nullptr ||
        probe_feedback == nullptr || probe_turns == nullptr) {
        return kInvalidRuntimeConfig;
    }
    std::vector<std::uint32_t> codes(kProbeStates * kProbeMaxTurns, 0);
    std::vector<std::uint16_t> tiles(kProbeStates * kProbeMaxTurns, 0);
    for (int p = 0; p < kProbeStates; ++p) {
        if (probe_turns[p] > kProbeMaxTurns) {
            return kPolicyForwardFailed;
        }
        for (int u = 0; u < probe_turns[p]; ++u) {
            const std::uint8_t *w = probe_letters + (p * kProbeMaxTurns + u) * kWordLength;
            const std::uint8_t *f = probe_feedback + (p * kProbeMaxTurns + u) * kWordLength;
            std::uint32_t packed = 0;
            for (int k = 0; k < kWordLength; ++k) {
                if (w[k] >= kAlphabet || f[k] > kGrey) {
                    return kPolicyForwardFailed;
                }
                packed |= static_cast<std::uint32_t>(f[k]) << (2 * k);
            }
            codes[p * kProbeMaxTurns + u] = PackWord(w);
            tiles[p * kProbeMaxTurns + u] = static_cast<std::uint16_t>(packed);
        }
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    const int ctas = EvalCtaCount(static_cast<std::uint32_t>(count));
    std::uint32_t *d_codes = nullptr;
    std::uint16_t *d_tiles = nullptr;
    std::uint8_t *d_turns = nullptr;
    float *scratch = nullptr;
    bool ok = cudaMalloc(&d_codes, codes.size() * 4) == cudaSuccess &&
              cudaMalloc(&d_tiles, tiles.size() * 2) == cudaSuccess && cudaMalloc(&d_turns, kProbeStates) == cudaSuccess &&
              cudaMalloc(&scratch, static_cast<std::size_t>(ctas) * EvalScratchFloatsPerCta() * 4) == cudaSuccess &&
              cudaMemcpyAsync(d_codes, codes.data(), codes.size() * 4, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(d_tiles, tiles.data(), tiles.size() * 2, cudaMemcpyHostToDevice, s) == cudaSuccess &&
              cudaMemcpyAsync(d_turns, probe_turns, kProbeStates, cudaMemcpyHostToDevice, s) == cudaSuccess;
    if (ok) {
        DescriptorParams q{};
        q.slab = static_cast<const std::uint8_t *>(slab);
        q.pitch = pitch;
        q.slots = slots;
        q.count = static_cast<std::uint32_t>(count);
        q.probe_codes = d_codes;
        q.probe_tiles = d_tiles;
        q.probe_turns = d_turns;
        q.scale = scale;
        q.scratch = scratch;
        q.out = out;
        q.out_ld = kDescriptorWidth;
        ok = LaunchDescriptors(q, ctas, s) == cudaSuccess && cudaStreamSynchronize(s) == cudaSuccess;
    }
    cudaFree(d_codes);
    cudaFree(d_tiles);
    cudaFree(d_turns);
    cudaFree(scratch);
    return ok ? kOk : kCudaFailure;
}

int nwg_bf16_gemm_nt(const void *a, size_t lda, const void *b, size_t ldb, float *c, size_t ldc, size_t m, size_t n,
                     size_t k, void *cuda_stream) {
    int *error = nullptr;
    if (cudaMalloc(&error, sizeof(int)) != cudaSuccess) {
        return kCudaFailure;
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    int st = cudaMemsetAsync(error, 0, sizeof(int), s) == cudaSuccess ? kOk : kCudaFailure;
    if (st == kOk) {
        const cudaError_t e = LaunchGemmNt(a, lda, b, ldb, c, ldc, m, n, k, error, s);
        st = e == cudaSuccess ? kOk : (e == cudaErrorInvalidValue ? kUnsupported : kCudaFailure);
    }
    int flag = 0;
    if (st == kOk && (cudaMemcpyAsync(&flag, error, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                      cudaStreamSynchronize(s) != cudaSuccess)) {
        st = kCudaFailure;
    }
    cudaFree(error);
    return st == kOk && flag != 0 ? kTimeout : st;
}

}  // extern "C"
