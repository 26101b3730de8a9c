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
// Two values rounded to BF16 (nearest even), the first in the low half.
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    return (uint32_t)bf16_bits(lo) | ((uint32_t)bf16_bits(hi) << 16);
}
// 16 bytes into a tile at byte offset `off` (a multiple of 16).
__device__ __forceinline__ void store16(uint16_t* tile, uint32_t off, const uint32_t (&w)[4]) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(umma::smem_u32(tile) + off),
                 "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3])
                 : "memory");
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

// ─── the network ────────────────────────────────────────────────────────────────────────────
//
// theta (FP32 master parameters): W1 [128][4] (out, in), b1 [128], W2 [128][128] (in, out),
// b2 [128], W3 [128][16] (in, out; outputs 12..15 stay zero), b3 [16]. norm: the input's mean
// (4) and inverse deviation (4), then the output scale (12). pack (BF16): W2 transposed
// [out][in], W2 [in][out], W3 transposed [16][128], W3 [128][16].
constexpr int kW1 = 0, kB1 = 512, kW2 = 640, kB2 = 17024, kW3 = 17152, kB3 = 19200, kTheta = 19216;
constexpr int kPW2T = 0, kPW2 = 16384, kPW3T = 32768, kPW3 = 34816, kPack = 36864;
constexpr int kOut = 12;

__device__ __forceinline__ float gelu(float z) {
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float z) {
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) +
           z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__global__ void pack_weights(const float* theta, uint16_t* pack) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < 16384) {
        const int in = q / 128, out = q % 128;
        const uint16_t v = bf16_bits(theta[kW2 + q]);
        pack[kPW2 + q] = v;
        pack[kPW2T + out * 128 + in] = v;
    }
    if (q < 2048) {
        const int in = q / 16, o = q % 16;
        const uint16_t v = bf16_bits(theta[kW3 + q]);
        pack[kPW3 + q] = v;
        pack[kPW3T + o * 128 + in] = v;
    }
}

// Shared memory of a network CTA: the operand tiles (BF16, K-chunked layout), the small FP32
// parameters, the row-reduced gradients, and the barrier state.
struct NetSmem {
    uint16_t w2t[128 * 128];  // B of layer 2: N = out, K = in
    uint16_t w3t[16 * 128];   // B of layer 3: N = 16, K = in
    uint16_t h1[128 * 128];   // A of layer 2; MN-major A of dW2
    uint16_t h2[128 * 128];   // A of layer 3; MN-major A of dW3
    uint16_t w2[128 * 128];   // B of dH1: N = in, K = out (training)
    uint16_t w3[128 * 16];    // B of dH2: N = in, K = 16 (training)
    uint16_t g3[128 * 16];    // dout: A of dH2; MN-major B of dW3 (training)
    uint16_t g2[128 * 128];   // dZ2: A of dH1; MN-major B of dW2 (training)
    float w1[512], b1[128], b2[128], b3[16];
    float gw1[512], gb1[128], gb2[128], gb3[16];
    float loss;
    uint64_t mbar;
    uint32_t tmem;
    int failed;
};

// Stage a row-major BF16 matrix (rows x cols) into the K-chunked layout of a tile with `rows`
// rows (the M or N side) and `cols` reduction columns.
__device__ __forceinline__ void stage_tile(uint16_t* dst, const uint16_t* src, int rows, int cols) {
    for (int q = threadIdx.x; q < rows * cols; q += blockDim.x) {
        const int r = q / cols, c = q % cols;
        dst[umma::tile_offset(rows, r, c) / 2] = src[q];
    }
}

__device__ __forceinline__ void net_setup(NetSmem& S, const float* theta, const uint16_t* pack,
                                          bool training, uint32_t ncols) {
    stage_tile(S.w2t, pack + kPW2T, 128, 128);
    stage_tile(S.w3t, pack + kPW3T, 16, 128);
    if (training) {
        stage_tile(S.w2, pack + kPW2, 128, 128);
        stage_tile(S.w3, pack + kPW3, 128, 16);
    }
    for (int q = threadIdx.x; q < 512; q += blockDim.x) {
        S.w1[q] = theta[kW1 + q];
        S.gw1[q] = 0.0f;
    }
    for (int q = threadIdx.x; q < 128; q += blockDim.x) {
        S.b1[q] = theta[kB1 + q];
        S.b2[q] = theta[kB2 + q];
        S.gb1[q] = 0.0f;
        S.gb2[q] = 0.0f;
    }
    if (threadIdx.x < 16) {
        S.b3[threadIdx.x] = theta[kB3 + threadIdx.x];
        S.gb3[threadIdx.x] = 0.0f;
    }
    if (threadIdx.x == 0) {
        S.loss = 0.0f;
        S.failed = 0;
        umma::mbar_init(&S.mbar, 1);
    }
    if (threadIdx.x < 32) umma::tmem_alloc(&S.tmem, ncols);
    umma::fence_async_shared();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
}

// Make the tiles this thread wrote visible to the tensor cores, and let thread 0 issue.
__device__ __forceinline__ void tiles_ready() {
    umma::fence_async_shared();
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
}

// Wait for the MMAs committed so far; false (and the CTA's failure flag) on a timeout.
template <class Smem> __device__ __forceinline__ bool mma_done(Smem& S, uint32_t& phase) {
    const bool ok = umma::mbar_wait(&S.mbar, phase & 1u, kWaitLimit);
    phase += 1;
    umma::fence_after_sync();
    if (!ok) S.failed = 1;
    __syncthreads();
    return S.failed == 0;
}

// Sum over the CTA's 128 rows of one value per thread into a shared accumulator.
__device__ __forceinline__ void row_sum(float* acc, float v) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(acc, v);
}

// TMEM column bases
constexpr uint32_t kD2 = 0, kD3 = 128, kDW3 = 144, kDH = 160, kDW2 = 288;

// The forward pass of the tile: the layer-1 row, then layers 2 and 3 on the tensor cores.
// Leaves Z2 - b2 in TMEM column kD2, the output in kD3 (both in this thread's lane), H1 and H2
// in shared memory, and the normalised input in xh.
__device__ __forceinline__ bool net_forward(NetSmem& S, const float (&xh)[4], bool active,
                                            uint32_t& phase, float (&out)[16]) {
    const int t = threadIdx.x;
    for (int j = 0; j < 128; ++j) {
        float z = S.b1[j];
#pragma unroll
        for (int i = 0; i < 4; ++i) z = fmaf(S.w1[j * 4 + i], xh[i], z);
        S.h1[umma::tile_offset(128, t, j) / 2] = active ? bf16_bits(gelu(z)) : (uint16_t)0;
    }
    tiles_ready();
    const uint32_t tm = S.tmem;
    if (t == 0) {
        const uint32_t a0 = umma::smem_u32(S.h1), b0 = umma::smem_u32(S.w2t);
        const uint32_t id = umma::idesc_bf16(128, 128, 0, 0);
        for (int s = 0; s < 8; ++s)
            umma::mma(tm + kD2, umma::desc_kmajor(a0, 128, s), umma::desc_kmajor(b0, 128, s), id, s > 0);
        umma::commit(&S.mbar);
    }
    if (!mma_done(S, phase)) return false;
    const uint32_t lb = umma::lane_base(tm);
    for (int c = 0; c < 128; c += 16) {
        float v[16];
        umma::ld16(lb + kD2 + (uint32_t)c, v);
#pragma unroll
        for (int i = 0; i < 16; ++i)
            S.h2[umma::tile_offset(128, t, c + i) / 2] =
                active ? bf16_bits(gelu(v[i] + S.b2[c + i])) : (uint16_t)0;
    }
    tiles_ready();
    if (t == 0) {
        const uint32_t a0 = umma::smem_u32(S.h2), b0 = umma::smem_u32(S.w3t);
        const uint32_t id = umma::idesc_bf16(128, 16, 0, 0);
        for (int s = 0; s < 8; ++s)
            umma::mma(tm + kD3, umma::desc_kmajor(a0, 128, s), umma::desc_kmajor(b0, 16, s), id, s > 0);
        umma::commit(&S.mbar);
    }
    if (!mma_done(S, phase)) return false;
    umma::ld16(lb + kD3, out);
#pragma unroll
    for (int o = 0; o < 16; ++o) out[o] += S.b3[o];
    return true;
}

__device__ __forceinline__ void normalise(const double* state, const float* norm, bool active,
                                          float (&xh)[4]) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
        xh[i] = active ? ((float)state[i] - norm[i]) * norm[4 + i] : 0.0f;
}

// The explicit stage guess Z_j = h c_j f(y), c_j the row sums of the tableau (shared = h, A
// column-major), in double.
__device__ __forceinline__ void stage_guess(const double* y, const double* shared, double (&z)[12]) {
    const double h = shared[0];
    const double f[4] = {y[2], y[3], -y[0] - 2.0 * y[0] * y[1], -y[1] - y[0] * y[0] + y[1] * y[1]};
#pragma unroll
    for (int j = 0; j < 3; ++j) {
        const double c = shared[1 + j] + shared[1 + j + 3] + shared[1 + j + 6];
#pragma unroll
        for (int k = 0; k < 4; ++k) z[4 * j + k] = h * c * f[k];
    }
}

// Shared memory of an inference CTA: the two weight tiles, one activation tile (H1, then H2 once
// the layer-2 product has read H1), the small FP32 parameters and the barrier state — about
// 72 KB, so that three CTAs share an SM where the training layout (182 KB) fits one. Layer 3's
// accumulator reuses TMEM columns 0..15 once layer 2's have been read, so a CTA holds 128 columns.
struct InferSmem {
    uint16_t w2t[128 * 128];  // B of layer 2: N = out, K = in
    uint16_t w3t[16 * 128];   // B of layer 3: N = 16, K = in
    uint16_t h[128 * 128];    // A of layer 2 (H1), then A of layer 3 (H2)
    float w1[512], b1[128], b2[128], b3[16];
    uint64_t mbar;
    uint32_t tmem;
    int failed;
};

// Inference: Z0 = guess + scale * net(y), persistent over 128-system tiles.
__global__ void __launch_bounds__(128) net_predict(const float* theta, const uint16_t* pack,
                                                   const float* norm, const double* shared,
                                                   const double* states, double* Z0, int64_t n,
                                                   int* err) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smraw);
    const int t = threadIdx.x;
    stage_tile(S.w2t, pack + kPW2T, 128, 128);
    stage_tile(S.w3t, pack + kPW3T, 16, 128);
    for (int q = t; q < 512; q += blockDim.x) S.w1[q] = theta[kW1 + q];
    for (int q = t; q < 128; q += blockDim.x) {
        S.b1[q] = theta[kB1 + q];
        S.b2[q] = theta[kB2 + q];
    }
    if (t < 16) S.b3[t] = theta[kB3 + t];
    if (t == 0) {
        S.failed = 0;
        umma::mbar_init(&S.mbar, 1);
    }
    if (t < 32) umma::tmem_alloc(&S.tmem, 128);
    tiles_ready();
    const uint32_t tm = S.tmem;
    const uint32_t lb = umma::lane_base(tm);
    uint32_t phase = 0;
    for (int64_t tile = blockIdx.x; tile * 128 < n; tile += gridDim.x) {
        const int64_t row = tile * 128 + t;
        const bool active = row < n;
        float xh[4];
        normalise(states + (active ? row : 0) * 4, norm, active, xh);
        // layer 1 on the CUDA cores, H1 into the activation tile: the eight columns of a
        // core-matrix row are 16 contiguous bytes, one store (a warp's 32 rows fill 512
        // contiguous bytes, no bank conflict)
        for (int jc = 0; jc < 16; ++jc) {
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float g[2];
#pragma unroll
                for (int u = 0; u < 2; ++u) {
                    const int j = jc * 8 + 2 * q + u;
                    float z = S.b1[j];
#pragma unroll
                    for (int i = 0; i < 4; ++i) z = fmaf(S.w1[j * 4 + i], xh[i], z);
                    g[u] = active ? gelu(z) : 0.0f;
                }
                w[q] = pack_bf16x2(g[0], g[1]);
            }
            store16(S.h, umma::tile_offset(128, t, jc * 8), w);
        }
        tiles_ready();
        if (t == 0) {
            const uint32_t a0 = umma::smem_u32(S.h), b0 = umma::smem_u32(S.w2t);
            const uint32_t id = umma::idesc_bf16(128, 128, 0, 0);
            for (int s = 0; s < 8; ++s)
                umma::mma(tm, umma::desc_kmajor(a0, 128, s), umma::desc_kmajor(b0, 128, s), id, s > 0);
            umma::commit(&S.mbar);
        }
        if (!mma_done(S, phase)) break;
        // H2 over H1 (the product that read H1 has completed)
        for (int c = 0; c < 128; c += 16) {
            float v[16];
            umma::ld16(lb + (uint32_t)c, v);
#pragma unroll
            for (int h8 = 0; h8 < 2; ++h8) {
                uint32_t w[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int i0 = h8 * 8 + 2 * q;
                    const float g0 = active ? gelu(v[i0] + S.b2[c + i0]) : 0.0f;
                    const float g1 = active ? gelu(v[i0 + 1] + S.b2[c + i0 + 1]) : 0.0f;
                    w[q] = pack_bf16x2(g0, g1);
                }
                store16(S.h, umma::tile_offset(128, t, c + h8 * 8), w);
            }
        }
        tiles_ready();
        if (t == 0) {
            const uint32_t a0 = umma::smem_u32(S.h), b0 = umma::smem_u32(S.w3t);
            const uint32_t id = umma::idesc_bf16(128, 16, 0, 0);
            for (int s = 0; s < 8; ++s)
                umma::mma(tm, umma::desc_kmajor(a0, 128, s), umma::desc_kmajor(b0, 16, s), id, s > 0);
            umma::commit(&S.mbar);
        }
        if (!mma_done(S, phase)) break;
        float out[16];
        umma::ld16(lb, out);
        if (active) {
            double z[12];
            stage_guess(states + row * 4, shared, z);
#pragma unroll
            for (int o = 0; o < kOut; ++o)
                Z0[row * 12 + o] = z[o] + (double)norm[8 + o] * (double)(out[o] + S.b3[o]);
        }
        // every lane has read its output before the next tile's products overwrite the columns
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
    }
    if (S.failed && t == 0) atomicExch(err, 1);
    umma::fence_before_sync();
    __syncthreads();
    if (t < 32) umma::tmem_free(S.tmem, 128);
}

// Training: the mean squared error of the scaled outputs against `targets` (B x 12) and its
// gradient with respect to theta, accumulated into grad (kTheta floats, zeroed by the caller)
// and loss. Each CTA takes tiles of 128 samples; dW2 and dW3 accumulate in tensor memory across
// the CTA's tiles and reach grad once.
__global__ void __launch_bounds__(128) net_grad(const float* theta, const uint16_t* pack,
                                                const float* norm, const double* states,
                                                const float* targets, int64_t n, float* grad,
                                                float* loss, int* err) {
    extern __shared__ __align__(1024) unsigned char smraw[];
    NetSmem& S = *reinterpret_cast<NetSmem*>(smraw);
    net_setup(S, theta, pack, true, 512);
    uint32_t phase = 0;
    const int t = threadIdx.x;
    const uint32_t tm = S.tmem;
    const uint32_t lb = umma::lane_base(tm);
    const float inv = 2.0f / (float)(n * kOut);
    int tiles = 0;
    for (int64_t tile = blockIdx.x; tile * 128 < n; tile += gridDim.x, ++tiles) {
        const int64_t row = tile * 128 + t;
        const bool active = row < n;
        float xh[4];
        normalise(states + (active ? row : 0) * 4, norm, active, xh);
        float out[16];
        if (!net_forward(S, xh, active, phase, out)) break;
        // dL/dout, the loss, db3
        float l = 0.0f;
#pragma unroll
        for (int o = 0; o < 16; ++o) {
            float g = 0.0f;
            if (active && o < kOut) {
                const float d = out[o] - targets[row * kOut + o];
                l = fmaf(d, d, l);
                g = inv * d;
            }
            S.g3[umma::tile_offset(128, t, o) / 2] = bf16_bits(g);
            row_sum(&S.gb3[o], g);
        }
        row_sum(&S.loss, l);
        tiles_ready();
        if (t == 0) {
            // dH2 = dout W3^T; dW3 += H2^T dout
            umma::mma(tm + kDH, umma::desc_kmajor(umma::smem_u32(S.g3), 128, 0),
                      umma::desc_kmajor(umma::smem_u32(S.w3), 128, 0), umma::idesc_bf16(128, 128, 0, 0),
                      false);
            const uint32_t id = umma::idesc_bf16(128, 16, 1, 1);
            for (int s = 0; s < 8; ++s)
                umma::mma(tm + kDW3, umma::desc_mnmajor(umma::smem_u32(S.h2), 128, s),
                          umma::desc_mnmajor(umma::smem_u32(S.g3), 128, s), id, tiles > 0 || s > 0);
            umma::commit(&S.mbar);
        }
        if (!mma_done(S, phase)) break;
        // dZ2 = dH2 * gelu'(Z2), db2
        for (int c = 0; c < 128; c += 16) {
            float dh[16], z2[16];
            umma::ld16(lb + kDH + (uint32_t)c, dh);
            umma::ld16(lb + kD2 + (uint32_t)c, z2);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float g = active ? dh[i] * gelu_grad(z2[i] + S.b2[c + i]) : 0.0f;
                S.g2[umma::tile_offset(128, t, c + i) / 2] = bf16_bits(g);
                row_sum(&S.gb2[c + i], g);
            }
        }
        tiles_ready();
        if (t == 0) {
            // dH1 = dZ2 W2^T; dW2 += H1^T dZ2
            const uint32_t idk = umma::idesc_bf16(128, 128, 0, 0);
            for (int s = 0; s < 8; ++s)
                umma::mma(tm + kDH, umma::desc_kmajor(umma::smem_u32(S.g2), 128, s),
                          umma::desc_kmajor(umma::smem_u32(S.w2), 128, s), idk, s > 0);
            const uint32_t idm = umma::idesc_bf16(128, 128, 1, 1);
            for (int s = 0; s < 8; ++s)
                umma::mma(tm + kDW2, umma::desc_mnmajor(umma::smem_u32(S.h1), 128, s),
                          umma::desc_mnmajor(umma::smem_u32(S.g2), 128, s), idm, tiles > 0 || s > 0);
            umma::commit(&S.mbar);
        }
        if (!mma_done(S, phase)) break;
        // dZ1 = dH1 * gelu'(Z1); dW1, db1
        for (int c = 0; c < 128; c += 16) {
            float dh[16];
            umma::ld16(lb + kDH + (uint32_t)c, dh);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int j = c + i;
                float z = S.b1[j];
#pragma unroll
                for (int q = 0; q < 4; ++q) z = fmaf(S.w1[j * 4 + q], xh[q], z);
                const float g = active ? dh[i] * gelu_grad(z) : 0.0f;
                row_sum(&S.gb1[j], g);
#pragma unroll
                for (int q = 0; q < 4; ++q) row_sum(&S.gw1[j * 4 + q], g * xh[q]);
            }
        }
        __syncthreads();
    }
    __syncthreads();
    if (!S.failed && tiles > 0) {
        // dW2 [in = this lane][out], dW3 [in = this lane][o] from tensor memory
        for (int c = 0; c < 128; c += 16) {
            float v[16];
            umma::ld16(lb + kDW2 + (uint32_t)c, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) atomicAdd(&grad[kW2 + t * 128 + c + i], v[i]);
        }
        float v[16];
        umma::ld16(lb + kDW3, v);
#pragma unroll
        for (int o = 0; o < kOut; ++o) atomicAdd(&grad[kW3 + t * 16 + o], v[o]);
        for (int q = t; q < 512; q += 128) atomicAdd(&grad[kW1 + q], S.gw1[q]);
        atomicAdd(&grad[kB1 + t], S.gb1[t]);
        atomicAdd(&grad[kB2 + t], S.gb2[t]);
        if (t < kOut) atomicAdd(&grad[kB3 + t], S.gb3[t]);
        if (t == 0) atomicAdd(loss, S.loss);
    }
    if (S.failed && t == 0) atomicExch(err, 1);
    umma::fence_before_sync();
    __syncthreads();
    if (t < 32) umma::tmem_free(tm, 512);
}

// Adam (bias-corrected) on the FP32 master parameters; the outputs 12..15 of W3 and b3 stay zero.
__global__ void adam_step(float* theta, float* m, float* v, const float* grad, float lr, float b1,
                          float b2, float eps, int step) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kTheta) return;
    if ((q >= kW3 && q < kB3 && (q - kW3) % 16 >= kOut) || (q >= kB3 + kOut)) return;
    const float g = grad[q];
    const float mq = b1 * m[q] + (1.0f - b1) * g;
    const float vq = b2 * v[q] + (1.0f - b2) * g * g;
    m[q] = mq;
    v[q] = vq;
    const float mh = mq / (1.0f - powf(b1, (float)step));
    const float vh = vq / (1.0f - powf(b2, (float)step));
    theta[q] -= lr * mh / (sqrtf(vh) + eps);
}

// The accept-if-better gate: per system, the FP64 residual norm of the stage equations at the
// network's start and at the default start; the better start goes into X (the default wins
// ties and non-finite predictions), and `accepted` records the choice.
__global__ void warm_select(const double* shared, const double* states, const double* Z0,
                            const double* Xdef, double* X, uint8_t* accepted, int64_t n) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const double h = shared[0];
    const double* A = shared + 1;
    const double* y = states + s * 4;
    double nrm[2];
    for (int w = 0; w < 2; ++w) {
        const double* Z = w == 0 ? Z0 + s * 12 : Xdef + s * 12;
        double G[12];
        for (int k = 0; k < 12; ++k) G[k] = Z[k];
        for (int j = 0; j < 3; ++j) {
            double Y[4];
            for (int k = 0; k < 4; ++k) Y[k] = __dadd_rn(y[k], Z[4 * j + k]);
            const double f[4] = {Y[2], Y[3], __dsub_rn(-Y[0], __dmul_rn(2.0, __dmul_rn(Y[0], Y[1]))),
                                 __dadd_rn(__dsub_rn(-Y[1], __dmul_rn(Y[0], Y[0])), __dmul_rn(Y[1], Y[1]))};
            for (int i = 0; i < 3; ++i) {
                const double a = __dmul_rn(h, A[i + 3 * j]);
                for (int k = 0; k < 4; ++k) G[4 * i + k] = __dsub_rn(G[4 * i + k], __dmul_rn(a, f[k]));
            }
        }
        double q = 0.0;
        for (int k = 0; k < 12; ++k) q = fma(G[k], G[k], q);
        nrm[w] = q;
    }
    const bool take = isfinite(nrm[0]) && nrm[0] < nrm[1];
    for (int k = 0; k < 12; ++k) X[s * 12 + k] = take ? Z0[s * 12 + k] : Xdef[s * 12 + k];
    accepted[s] = take ? 1 : 0;
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

namespace {

// A persistent grid: the CTAs that are resident at once, by shared memory (the device's per-SM
// capacity and per-block reservation) and by tensor memory (512 columns per SM, `tmem_cols` per
// CTA), at most one per 128-row tile.
int net_grid(const void* fn, size_t smem, int64_t n, int tmem_cols, int* grid) {
    int dev = 0, sms = 0, smem_sm = 0, reserved = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return GSB_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return GSB_ERR_CUDA;
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess)
        return GSB_ERR_CUDA;
    if (cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess)
        return GSB_ERR_CUDA;
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return GSB_ERR_CUDA;
    // the largest shared-memory carveout, so that the CTAs that fit by shared memory are resident
    if (cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared) != cudaSuccess)
        return GSB_ERR_CUDA;
    int occ = (int)((size_t)smem_sm / (smem + (size_t)reserved));
    const int by_tmem = 512 / tmem_cols;
    if (occ > by_tmem) occ = by_tmem;
    if (occ > 16) occ = 16;  // 2048 threads per SM
    if (occ < 1) occ = 1;
    const int64_t tiles = (n + 127) / 128;
    const int64_t g = (int64_t)sms * occ;
    *grid = (int)(tiles < g ? tiles : g);
    return 0;
}

int finish(int* err, cudaStream_t st) {
    int h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return GSB_ERR_CUDA;
    return h ? GSB_ERR_CUDA : 0;
}

}  // namespace

extern "C" {

int gsb_mlp_sizes(int64_t* theta_floats, int64_t* pack_halves) {
    if (theta_floats) *theta_floats = gsb::mlp::kTheta;
    if (pack_halves) *pack_halves = gsb::mlp::kPack;
    return 0;
}

int gsb_mlp_pack(const float* theta, uint16_t* pack, void* stream) {
    if (!theta || !pack) return GSB_ERR_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    gsb::mlp::pack_weights<<<64, 256, 0, st>>>(theta, pack);
    return cudaGetLastError() == cudaSuccess ? 0 : GSB_ERR_CUDA;
}

int gsb_mlp_predict(const float* theta, const uint16_t* pack, const float* norm,
                    const double* shared, const double* states, double* Z0, int64_t n,
                    int* err_scratch, void* stream) {
    if (n < 0 || !theta || !pack || !norm || !shared || !states || !Z0 || !err_scratch)
        return GSB_ERR_ARGUMENT;
    if (n == 0) return 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const size_t smem = sizeof(gsb::mlp::InferSmem);
    int grid = 0;
    if (int rc = net_grid((const void*)gsb::mlp::net_predict, smem, n, 128, &grid)) return rc;
    cudaMemsetAsync(err_scratch, 0, sizeof(int), st);
    gsb::mlp::net_predict<<<grid, 128, smem, st>>>(theta, pack, norm, shared, states, Z0, n, err_scratch);
    if (cudaGetLastError() != cudaSuccess) return GSB_ERR_CUDA;
    return finish(err_scratch, st);
}

int gsb_mlp_grad(const float* theta, const uint16_t* pack, const float* norm, const double* states,
                 const float* targets, int64_t n, float* grad, float* loss, int* err_scratch,
                 void* stream) {
    if (n <= 0 || !theta || !pack || !norm || !states || !targets || !grad || !loss || !err_scratch)
        return GSB_ERR_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const size_t smem = sizeof(gsb::mlp::NetSmem);
    int grid = 0;
    if (int rc = net_grid((const void*)gsb::mlp::net_grad, smem, n, 512, &grid)) return rc;
    cudaMemsetAsync(grad, 0, gsb::mlp::kTheta * sizeof(float), st);
    cudaMemsetAsync(loss, 0, sizeof(float), st);
    cudaMemsetAsync(err_scratch, 0, sizeof(int), st);
    gsb::mlp::net_grad<<<grid, 128, smem, st>>>(theta, pack, norm, states, targets, n, grad, loss,
                                                 err_scratch);
    if (cudaGetLastError() != cudaSuccess) return GSB_ERR_CUDA;
    return 0;
}

int gsb_mlp_adam(float* theta, float* m, float* v, const float* grad, uint16_t* pack, float lr,
                 float beta1, float beta2, float eps, int32_t step, void* stream) {
    if (!theta || !m || !v || !grad || !pack || step < 1) return GSB_ERR_ARGUMENT;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    gsb::mlp::adam_step<<<(gsb::mlp::kTheta + 255) / 256, 256, 0, st>>>(theta, m, v, grad, lr, beta1,
                                                                         beta2, eps, step);
    gsb::mlp::pack_weights<<<64, 256, 0, st>>>(theta, pack);
    return cudaGetLastError() == cudaSuccess ? 0 : GSB_ERR_CUDA;
}

int gsb_warm_start_select(const double* shared, const double* states, const double* Z0,
                          const double* Xdefault, double* X, uint8_t* accepted, int64_t n,
                          void* stream) {
    if (n < 0 || !shared || !states || !Z0 || !Xdefault || !X || !accepted) return GSB_ERR_ARGUMENT;
    if (n == 0) return 0;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    gsb::mlp::warm_select<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(shared, states, Z0, Xdefault,
                                                                       X, accepted, n);
    return cudaGetLastError() == cudaSuccess ? 0 : GSB_ERR_CUDA;
}

}  // extern "C"
