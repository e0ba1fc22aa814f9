// Compute-throughput denominators for the blend's roofline: the measured rate of MUFU ex2
// (ex2.approx.ftz.f32, one per pixel-splat evaluation in the blend) and of FP32 FMA on this GPU,
// at whatever clock it runs. Built as its own small library (libaniso_b200_peaks.so); the
// renderer does not link it.
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__device__ __forceinline__ float ex2(float x) {
    float y;
    asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// kChains independent chains per thread; each step is one ex2 and one add that keeps the
// argument in [-1, 0] so the chain neither overflows nor denormalises.
__global__ void ex2_kernel(float* out, int iters) {
    float a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = -0.01f * (threadIdx.x % 32 + c);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) a[c] = ex2(a[c]) - 1.5f;
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == 12345.f) out[blockIdx.x] = s;  // keeps the loop alive
}

__global__ void fma_kernel(float* out, int iters) {
    float a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) a[c] = 0.001f * (threadIdx.x + c);
    const float m = 0.999f, k = 0.0001f;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) a[c] = fmaf(a[c], m, k);
    }
    float s = 0.f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += a[c];
    if (s == 12345.f) out[blockIdx.x] = s;
}

template <class K>
double rate(K kernel, int blocks, int threads, int iters, float* out) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    kernel<<<blocks, threads>>>(out, iters / 10);  // warm-up
    cudaEventRecord(e0);
    kernel<<<blocks, threads>>>(out, iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return static_cast<double>(blocks) * threads * iters * kChains / (ms * 1e-3);
}

}  // namespace

extern "C" int ab2_measure_peaks(double* ex2_per_s, double* fma_per_s) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
    float* out = nullptr;
    if (cudaMalloc(&out, 1 << 16) != cudaSuccess) return 1;
    const int blocks = sms * 8, threads = 256;  // 64 warps per SM
    if (ex2_per_s) *ex2_per_s = rate(ex2_kernel, blocks, threads, 4096, out);
    if (fma_per_s) *fma_per_s = rate(fma_kernel, blocks, threads, 16384, out);
    const cudaError_t e = cudaGetLastError();
    cudaFree(out);
    return e == cudaSuccess ? 0 : 1;
}
