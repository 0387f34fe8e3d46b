// Throughput probes for the roofline denominators this path needs and
// MEASURED_PEAKS.json does not hold: FP32 FMA, FP64 FMA and the FP32
// reciprocal (MUFU) rate of the device.  Each thread runs 8 independent
// dependency chains so the pipes, not latency, bound the rate.
#include <cuda_runtime.h>

#include "xs_engine.h"
#include "xsec_b200.h"

namespace {

constexpr int kChains = 8;
constexpr int kIters = 4096;

__global__ void k_fma32(float* sink, float seed) {
    float a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = seed + float(threadIdx.x + c);
    const float m = 0.9999999f, k = 1e-7f;
    for (int i = 0; i < kIters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) a[c] = fmaf(a[c], m, k);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == 1234.5678f) sink[threadIdx.x] = s;
}

__global__ void k_fma64(double* sink, double seed) {
    double a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = seed + double(threadIdx.x + c);
    const double m = 0.9999999, k = 1e-7;
    for (int i = 0; i < kIters / 4; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) a[c] = fma(a[c], m, k);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == 1234.5678) sink[threadIdx.x] = s;
}

__global__ void k_rcp32(float* sink, float seed) {
    float a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = seed + float(threadIdx.x + c);
    for (int i = 0; i < kIters / 4; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) {
            // a <- 1/a + 1 (converges to the golden ratio): the add keeps
            // consecutive reciprocals from cancelling
            float r;
            asm volatile("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(a[c]));
            a[c] = r + 1.0f;
        }
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == 1234.5678f) sink[threadIdx.x] = s;
}

template <class K, class... Args>
float time_kernel(K kernel, int blocks, int threads, Args... args) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    kernel<<<blocks, threads>>>(args...);  // warm-up
    cudaEventRecord(a);
    for (int r = 0; r < 5; ++r) kernel<<<blocks, threads>>>(args...);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms / 5.0f;
}

}  // namespace

extern "C" int xs_measure_peaks(int device, double* fp32_tflops, double* fp64_tflops,
                                double* rcp32_tops) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return xs::set_error(XS_ERR_NODEVICE, "bad device");
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    void* sink = nullptr;
    if (cudaMalloc(&sink, 1024 * sizeof(double)) != cudaSuccess) {
        cudaSetDevice(prev);
        return xs::set_error(XS_ERR_NOMEM, "probe sink");
    }
    const int threads = 256, blocks = sms * 8;
    const double n = double(blocks) * threads * kChains;
    const float t32 = time_kernel(k_fma32, blocks, threads, static_cast<float*>(sink), 1.0f);
    const float t64 = time_kernel(k_fma64, blocks, threads, static_cast<double*>(sink), 1.0);
    const float tr = time_kernel(k_rcp32, blocks, threads, static_cast<float*>(sink), 1.5f);
    const cudaError_t err = cudaGetLastError();
    cudaFree(sink);
    cudaSetDevice(prev);
    if (err != cudaSuccess) return xs::set_error(XS_ERR_CUDA, cudaGetErrorString(err));
    if (fp32_tflops) *fp32_tflops = 2.0 * n * kIters / (double(t32) * 1e-3) / 1e12;
    if (fp64_tflops) *fp64_tflops = 2.0 * n * (kIters / 4) / (double(t64) * 1e-3) / 1e12;
    if (rcp32_tops) *rcp32_tops = n * (kIters / 4) / (double(tr) * 1e-3) / 1e12;
    return XS_OK;
}
