// The learned warm start of the stage systems: a 4 -> 128 -> 128 -> 12 MLP (GELU, BF16 weights
// and activations, FP32 accumulation) that maps a Hénon–Heiles state to the stage increments Z.
// The 128 x 128 and 128 x 16 products of inference and training run on the fifth-generation
// tensor cores (tcgen05, gsb_umma.cuh) from operand tiles in shared memory, accumulating in
// tensor memory; the 4-input first layer and the elementwise work run on the CUDA cores.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/gsb.h"
#include "gsb_umma.cuh"

namespace gsb {
namespace mlp {

constexpr uint32_t kWaitLimit = 1u << 26;  // mbarrier polls before a tile gives up

__device__ __forceinline__ uint16_t bf16_bits(float v) {
    return __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// ─── self-test of the tile product ─────────────────────────────────────────────────────────
// D (128 x N, FP32) = A B^T for a 128 x K A and an N x K B (mode 0, both K-major), or with A
// given as its K x 128 transpose and B as its K x N transpose (mode 1, both read MN-major).
__global__ void __launch_bounds__(128) umma_selftest(const uint16_t* A, const uint16_t* B, float* D,
                                                     int K, int N, int mode, int* err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    uint16_t* sa = reinterpret_cast<uint16_t*>(sm);
    uint16_t* sb = reinterpret_cast<uint16_t*>(sm + 128 * K * 2);
    __shared__ uint64_t mbar;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x;
    if (mode == 0) {
        for (int q = t; q < 128 * K; q += 128) {
            const int r = q / K, k = q % K;
            sa[umma::tile_offset(128, r, k) / 2] = A[q];
        }
        for (int q = t; q < N * K; q += 128) {
            const int r = q / K, k = q % K;
            sb[umma::tile_offset(N, r, k) / 2] = B[q];
        }
    } else {
        for (int q = t; q < K * 128; q += 128) {
            const int r = q / 128, c = q % 128;
            sa[umma::tile_offset(K, r, c) / 2] = A[q];
        }
        for (int q = t; q < K * N; q += 128) {
            const int r = q / N, c = q % N;
            sb[umma::tile_offset(K, r, c) / 2] = B[q];
        }
    }
    uint32_t ncols = 32;
    while (ncols < (uint32_t)N) ncols <<= 1;
    if (t < 32) umma::tmem_alloc(&tslot, ncols);
    if (t == 0) umma::mbar_init(&mbar, 1);
    umma::fence_async_shared();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = tslot;
    if (t == 0) {
        const uint32_t id = umma::idesc_bf16(128, N, mode, mode);
        const uint32_t a0 = umma::smem_u32(sa), b0 = umma::smem_u32(sb);
        for (int s = 0; s < K / 16; ++s) {
            const uint64_t da = mode == 0 ? umma::desc_kmajor(a0, 128, s) : umma::desc_mnmajor(a0, K, s);
            const uint64_t db = mode == 0 ? umma::desc_kmajor(b0, N, s) : umma::desc_mnmajor(b0, K, s);
            umma::mma(tmem, da, db, id, s > 0);
        }
        umma::commit(&mbar);
    }
    const bool ok = umma::mbar_wait(&mbar, 0, kWaitLimit);
    umma::fence_after_sync();
    if (!ok) {
        if (t == 0) atomicExch(err, 1);
    } else {
        for (int c = 0; c < N; c += 16) {
            float v[16];
            umma::ld16(umma::lane_base(tmem) + (uint32_t)c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) D[t * N + c + i] = v[i];
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    if (t < 32) umma::tmem_free(tmem, ncols);
}

}  // namespace mlp
}  // namespace gsb

extern "C" {

GSB_API int gsb_umma_selftest(const uint16_t* A, const uint16_t* B, float* D, int32_t K, int32_t N,
                              int32_t mode, void* stream) {
    if (K < 16 || K > 128 || K % 16 || N < 16 || N > 256 || N % 16 || (mode != 0 && mode != 1))
        return GSB_ERR_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    int* err = nullptr;
    if (cudaMalloc(&err, sizeof(int)) != cudaSuccess) return GSB_ERR_CUDA;
    cudaMemsetAsync(err, 0, sizeof(int), st);
    const size_t smem = (size_t)(128 * K + N * K) * 2;
    cudaFuncSetAttribute(gsb::mlp::umma_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    gsb::mlp::umma_selftest<<<1, 128, smem, st>>>(A, B, D, K, N, mode, err);
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(err);
    if (e != cudaSuccess) return GSB_ERR_CUDA;
    return h ? GSB_ERR_CUDA : 0;
}

}  // extern "C"
