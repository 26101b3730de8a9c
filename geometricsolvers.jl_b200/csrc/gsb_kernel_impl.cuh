// The batch kernel template: parameter staging, one Newton solve per thread, the stores of the
// iterate and the 72-byte status, and the tally of the count form. Instantiated per family and
// size in the gsb_inst_*.cu translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/gsb.h"
#include "gsb_families.cuh"
#include "gsb_newton.cuh"
#include "gsb_numerics.cuh"

namespace gsb {

constexpr int kThreads = 128;

struct Launch {
    double* X;
    int x_layout;
    void* S;
    int s_kind;
    const double* P;
    int p_layout;
    const int64_t* order;
    int order_base;
    int64_t nsys;
    const double* shared;
    unsigned long long* tally;  // 6 counters or nullptr
};

// Row of a thread's shared memory: its parameter block (np doubles), then 2n doubles where the
// iterate and the residual wait while a factor holds the registers; the stride is odd, so that
// thread t's entry k (address t*RS + k) falls in a distinct 8-byte bank slot for the 16 threads
// of each half-warp access.
__host__ __device__ constexpr int row_stride(int np, int n) {
    return ((np + 2 * n) % 2 == 1) ? np + 2 * n : np + 2 * n + 1;
}

__device__ __forceinline__ void store_status(void* S, int64_t idx, const DevStatus& s, double gr) {
    unsigned long long* w = reinterpret_cast<unsigned long long*>(
        reinterpret_cast<unsigned char*>(S) + idx * 72);
    unsigned long long w0 = (unsigned long long)(unsigned char)s.code |
                            ((unsigned long long)(unsigned int)s.iterations << 32);
    unsigned long long w3 = (unsigned long long)(unsigned int)s.step_failures |
                            ((unsigned long long)(s.promoted ? 1u : 0u) << 32) |
                            ((unsigned long long)(s.stationary ? 1u : 0u) << 40);
    unsigned long long w4 = (unsigned long long)(unsigned int)(-1);
    w[0] = w0;
    w[1] = (unsigned long long)__double_as_longlong(s.fnorm);
    w[2] = (unsigned long long)__double_as_longlong(s.stepnorm);
    w[3] = w3;
    w[4] = w4;
    w[5] = (unsigned long long)__double_as_longlong(kNaN);
    w[6] = (unsigned long long)__double_as_longlong(gr);
    w[7] = (unsigned long long)__double_as_longlong(s.rate);
    w[8] = (unsigned long long)(s.contracted ? 1u : 0u);
}

__device__ __forceinline__ void tally_code(unsigned long long* tally, int code) {
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        unsigned b = __ballot_sync(mask, code == c);
        if (lane == leader && b) atomicAdd(tally + c, (unsigned long long)__popc(b));
    }
}

template <class Fam, bool F, bool Mixed>
__global__ void __launch_bounds__(kThreads) newton_kernel(GsbMethod m, GsbOptions o, Launch L) {
    extern __shared__ double smem[];
    constexpr int N = Fam::N, NP = Fam::NP, RS = row_stride(NP, N);
    const int tid = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x * blockDim.x;
    const int64_t i = base + tid;
    double* prow = smem + tid * RS;
    if (L.order == nullptr && L.p_layout == GSB_AOS) {
        int64_t rem = L.nsys - base;
        int nloc = rem < (int64_t)blockDim.x ? (int)rem : (int)blockDim.x;
        const double* src = L.P + base * NP;
        for (int q = tid; q < nloc * NP; q += blockDim.x) {
            int s = q / NP;
            int k = q - s * NP;
            smem[s * RS + k] = __ldg(src + q);
        }
    } else if (i < L.nsys) {
        int64_t idx = L.order ? L.order[i] - L.order_base : i;
        if (L.p_layout == GSB_SOA) {
#pragma unroll 4
            for (int k = 0; k < NP; ++k) prow[k] = __ldg(L.P + (int64_t)k * L.nsys + idx);
        } else {
#pragma unroll 4
            for (int k = 0; k < NP; ++k) prow[k] = __ldg(L.P + idx * NP + k);
        }
    }
    __syncthreads();
    if (i >= L.nsys) return;
    const int64_t idx = L.order ? L.order[i] - L.order_base : i;
    Fam fam{prow};
    double x[N];
#pragma unroll
    for (int k = 0; k < N; ++k)
        x[k] = L.x_layout == GSB_SOA ? L.X[(int64_t)k * L.nsys + idx] : L.X[idx * N + k];
    Solver<Fam, F, Mixed> sv(fam, m, o, N >= 6 ? prow + NP : nullptr);
    double gr;
    DevStatus s = sv.solve(x, gr);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (L.x_layout == GSB_SOA) L.X[(int64_t)k * L.nsys + idx] = x[k];
        else L.X[idx * N + k] = x[k];
    }
    if (L.s_kind == GSB_STATUS64) store_status(L.S, idx, s, gr);
    else reinterpret_cast<unsigned char*>(L.S)[idx] = (unsigned char)s.code;
    if (L.tally) tally_code(L.tally, s.code);
}

using KernelFn = void (*)(GsbMethod, GsbOptions, Launch);

struct KernelEntry {
    KernelFn fn;
    int row;  // doubles of shared memory per thread
    bool attr_set[64];
};

template <class Fam, bool F, bool Mixed> KernelEntry* entry() {
    static KernelEntry e{newton_kernel<Fam, F, Mixed>, row_stride(Fam::NP, Fam::N), {}};
    return &e;
}

// The four kernels of a family: arithmetic fused or unfused, factor Float64 or Float32.
template <class Fam> KernelEntry* pick(bool fused, bool mixed) {
    if (fused) return mixed ? entry<Fam, true, true>() : entry<Fam, true, false>();
    return mixed ? entry<Fam, false, true>() : entry<Fam, false, false>();
}

#define GSB_DECLARE_ENTRY(NAME) KernelEntry* entry_##NAME(bool fused, bool mixed)
#define GSB_DEFINE_ENTRY(NAME, ...) \
    KernelEntry* entry_##NAME(bool fused, bool mixed) { return pick<__VA_ARGS__>(fused, mixed); }

}  // namespace gsb
