// Compute-peak microbenchmarks for the roofline of the spectrum kernels:
// FP64 FMA, FP32 FMA and SFU (MUFU sin/cos) throughput of the device, each
// from independent dependency chains in every thread of a grid of
// 8 blocks per SM.  Timed with CUDA events; results in operations/s.

#include <cuda_runtime.h>

#include "bgw_internal.h"
#include "device_common.cuh"

namespace bgw {
namespace {

constexpr int kChains = 8;

template <class T>
__global__ void __launch_bounds__(256) k_fma_peak(T* out, int iters, T a, T b) {
    T x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = (T)(threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = x[c] * a + b;
    }
    T s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == (T)-12345.678) out[threadIdx.x] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) k_sfu_peak(float* out, int iters) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = 0.001f * (threadIdx.x + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = __sinf(x[c]) + __cosf(x[c]);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == -12345.678f) out[threadIdx.x] = s;
}

template <class F>
double time_ms(F&& launch) {
    cudaEvent_t a, b;
    CUDA_OK(cudaEventCreate(&a));
    CUDA_OK(cudaEventCreate(&b));
    launch();  // warm-up
    CUDA_OK(cudaEventRecord(a));
    launch();
    CUDA_OK(cudaEventRecord(b));
    CUDA_OK(cudaEventSynchronize(b));
    float ms = 0;
    CUDA_OK(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    CUDA_OK(cudaGetLastError());
    return ms;
}

}  // namespace
}  // namespace bgw

extern "C" BgwStatus bgwx_measure_compute_peaks(double* fp64_flops, double* fp32_flops, double* sfu_ops) {
    using namespace bgw;
    try {
        if (device_count() < 1) throw Error{"no CUDA device is available"};
        int dev = 0, sms = 0;
        CUDA_OK(cudaGetDevice(&dev));
        CUDA_OK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int blocks = sms * 8, threads = 256;
        void* out = nullptr;
        CUDA_OK(cudaMalloc(&out, 4096));
        const double nthr = (double)blocks * threads;
        const int it64 = 4096, it32 = 16384, itsfu = 2048;
        double ms64 = time_ms([&] { k_fma_peak<double><<<blocks, threads>>>((double*)out, it64, 0.999, 1e-3); });
        double ms32 = time_ms([&] { k_fma_peak<float><<<blocks, threads>>>((float*)out, it32, 0.999f, 1e-3f); });
        double mssfu = time_ms([&] { k_sfu_peak<<<blocks, threads>>>((float*)out, itsfu); });
        cudaFree(out);
        if (fp64_flops) *fp64_flops = 2.0 * kChains * it64 * nthr / (ms64 * 1e-3);
        if (fp32_flops) *fp32_flops = 2.0 * kChains * it32 * nthr / (ms32 * 1e-3);
        if (sfu_ops) *sfu_ops = 2.0 * kChains * itsfu * nthr / (mssfu * 1e-3);
        return BGW_STATUS_OK;
    } catch (const Error&) {
        return BGW_STATUS_CALCULATION_ERROR;
    }
}
