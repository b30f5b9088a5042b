// FP64 FMA-pipe probe: the denominator of the integrator's roofline.
// Independent FMA chains per thread, grid = resident blocks on every SM,
// timed with CUDA events on the caller's stream.
#include <cuda_runtime.h>

#include "../../include/hurchem_b200.h"

namespace {

constexpr int kChains = 8;

__global__ void fma_probe(double *sink, int iters, double a, double b) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-9 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.678) sink[threadIdx.x] = s;   // keeps the chains live
}

}  // namespace

extern "C" int hc_probe_fp64_peak(int iters, double *tflops, void *stream) {
    if (!tflops || iters <= 0) return HC_E_INVALID;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fma_probe, threads, 0) != cudaSuccess)
        return HC_E_CUDA;
    double *sink = nullptr;
    if (cudaMallocAsync(&sink, threads * sizeof(double), st) != cudaSuccess) return HC_E_CUDA;
    const int blocks = sms * per_sm;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe<<<blocks, threads, 0, st>>>(sink, iters / 8, 0.999999, 1e-7);  // warm-up
    cudaEventRecord(e0, st);
    fma_probe<<<blocks, threads, 0, st>>>(sink, iters, 0.999999, 1e-7);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(sink, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return HC_E_CUDA;
    const double flops = 2.0 * kChains * (double)iters * blocks * threads;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return HC_OK;
}
