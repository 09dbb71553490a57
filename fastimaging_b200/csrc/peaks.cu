// Floating-point FMA throughput of the device, the compute roof of the
// imager's roofline (the gridder's complex taps run on the FP32 / FP64 FMA
// pipes, not on tensor cores).  Built as libstpgpu_peaks.so, a measurement
// helper beside the imaging library; bench.py records its figures next to the
// measured HBM bandwidth.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kChains = 8;  // independent FMA chains per thread
constexpr int kUnroll = 16; // FMAs per chain per loop iteration

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chains(T* sink, int iters, T a, T b)
{
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; c++)
        x[c] = T(threadIdx.x + c) * T(1e-3);
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
#pragma unroll
            for (int c = 0; c < kChains; c++)
                x[c] = fma(x[c], a, b);
        }
    }
    T s = T(0);
#pragma unroll
    for (int c = 0; c < kChains; c++)
        s += x[c];
    if (s == T(-1)) // never true: keeps the chains live
        sink[blockIdx.x] = s;
}

template <typename T>
int measure(int device, double* tflops)
{
    if (cudaSetDevice(device) != cudaSuccess)
        return 1;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return 1;
    const int blocks = sms * 8, threads = 256, iters = 4096;
    T* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T) * size_t(blocks)) != cudaSuccess)
        return 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const T a = T(0.999), b = T(1e-4); // the chains converge to 0.1: values stay normal
    k_fma_chains<T><<<blocks, threads>>>(sink, iters / 8, a, b); // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        k_fma_chains<T><<<blocks, threads>>>(sink, iters, a, b);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        best = ms < best ? ms : best;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess)
        return 1;
    const double flops = 2.0 * double(blocks) * threads * double(iters) * kUnroll * kChains;
    *tflops = flops / (double(best) * 1e-3) / 1e12;
    return 0;
}

} // namespace

// FMA throughput (TFLOP/s, 2 flops per FMA) of `device` in single
// (fp64 = 0) or double precision, best of five timed launches of
// independent FMA chains over every SM.  Returns 0 on success.
extern "C" __attribute__((visibility("default"))) int stpgpu_peaks_fma_tflops(int device, int fp64, double* tflops)
{
    return fp64 ? measure<double>(device, tflops) : measure<float>(device, tflops);
}
