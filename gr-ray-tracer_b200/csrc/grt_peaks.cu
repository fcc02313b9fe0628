// FP64 / FP32 fused-multiply-add throughput of the current device, measured
// with CUDA events over long independent FMA chains.  The trace kernels are
// CUDA-core FP64/FP32 bound, and the driver-measured peaks cover only HBM and
// bf16 tensor throughput, so this supplies the roofline denominators.
#include <cuda_runtime.h>

#include "grt.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

template <class T>
__global__ void fma_chain(T* out, T a, T b) {
    T acc[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) acc[c] = static_cast<T>(threadIdx.x + c);
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) acc[c] = fma(acc[c], a, b);
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += acc[c];
    if (s == static_cast<T>(-1.2345)) out[threadIdx.x] = s;  // keep the chains alive
}

template <class T>
double measure(int sm_count) {
    T* out = nullptr;
    if (cudaMalloc(&out, 1024 * sizeof(T)) != cudaSuccess) return -1.0;
    const int blocks = sm_count * 8, threads = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 5; ++rep) {
        cudaEventRecord(e0);
        fma_chain<T><<<blocks, threads>>>(out, static_cast<T>(0.999999), static_cast<T>(1e-7));
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    const double flops = 2.0 * kChains * static_cast<double>(kIters) * blocks * threads;
    return flops / (best * 1e-3) / 1e12;
}

}  // namespace

extern "C" grt_status grt_measure_fma_peaks(double* fp64_tflops, double* fp32_tflops) {
    int dev = 0;
    cudaDeviceProp prop;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return GRT_ENODEV;
    const double d = measure<double>(prop.multiProcessorCount);
    const double f = measure<float>(prop.multiProcessorCount);
    if (d < 0 || f < 0) return GRT_ECUDA;
    if (fp64_tflops) *fp64_tflops = d;
    if (fp32_tflops) *fp32_tflops = f;
    return cudaGetLastError() == cudaSuccess ? GRT_OK : GRT_ECUDA;
}
