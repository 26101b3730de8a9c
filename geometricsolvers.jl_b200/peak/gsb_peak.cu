// libgsbpeak: measures the FP64 and FP32 FMA-pipe throughput of the current device, the
// denominators of the batch kernel's roofline (the driver's peak file holds HBM and tensor
// peaks only). Each thread runs 8 independent FMA chains, so the pipe, not latency, bounds it.
#include <cuda_runtime.h>

#include <cstdint>

template <class T>
__global__ void __launch_bounds__(256) fma_chains(T* out, int iters, T a, T b) {
    T x0 = T(threadIdx.x) * T(1e-3), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int u = 0; u < 16; ++u) {
            x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
            x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
        }
    }
    T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == T(-12345.678)) out[0] = s;  // keeps the chains live
}

template <class T> static int run(int iters, double* tflops, void* buf) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_chains<T><<<blocks, threads>>>((T*)buf, 2, T(0.999999), T(1e-7));
    cudaEventRecord(e0);
    fma_chains<T><<<blocks, threads>>>((T*)buf, iters, T(0.999999), T(1e-7));
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" __attribute__((visibility("default"))) int gsb_peak_fma(int fp64, int iters,
                                                                   double* tflops) {
    void* buf = nullptr;
    if (cudaMalloc(&buf, 16) != cudaSuccess) return -4;
    int rc = fp64 ? run<double>(iters, tflops, buf) : run<float>(iters, tflops, buf);
    cudaFree(buf);
    return rc;
}
