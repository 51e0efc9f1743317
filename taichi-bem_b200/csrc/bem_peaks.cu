// Pipe-throughput probes of the device (FP32 FMA, FP64 FMA, MUFU), used as the
// roofline denominators of the assembly kernels (which are bound by the FP32 /
// FP64 FMA pipes and the special-function unit, not by HBM or tensor cores).
#include <cuda_runtime.h>

#include "bem_internal.cuh"

namespace {

constexpr int PROBE_ITERS = 2048;

template <typename T>
__global__ void __launch_bounds__(256) fma_probe(T* out, T b, T c) {
    T a0 = T(threadIdx.x), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
    T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
#pragma unroll 16
    for (int i = 0; i < PROBE_ITERS; ++i) {
        a0 = a0 * b + c; a1 = a1 * b + c; a2 = a2 * b + c; a3 = a3 * b + c;
        a4 = a4 * b + c; a5 = a5 * b + c; a6 = a6 * b + c; a7 = a7 * b + c;
    }
    T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == T(-12345.678)) out[blockIdx.x] = s;  // keeps the chains live
}

__global__ void __launch_bounds__(256) mufu_probe(float* out, float c) {
    float a0 = 1.0f + threadIdx.x, a1 = a0 + 1.f, a2 = a0 + 2.f, a3 = a0 + 3.f;
    float a4 = a0 + 4.f, a5 = a0 + 5.f, a6 = a0 + 6.f, a7 = a0 + 7.f;
#pragma unroll 16
    for (int i = 0; i < PROBE_ITERS; ++i) {
        a0 = rsqrtf(a0 + c); a1 = rsqrtf(a1 + c); a2 = rsqrtf(a2 + c); a3 = rsqrtf(a3 + c);
        a4 = rsqrtf(a4 + c); a5 = rsqrtf(a5 + c); a6 = rsqrtf(a6 + c); a7 = rsqrtf(a7 + c);
    }
    float s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == -12345.678f) out[blockIdx.x] = s;
}

template <typename K>
double time_ms(K launch, cudaStream_t s) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    launch();  // warm-up
    cudaEventRecord(e0, s);
    for (int r = 0; r < 5; ++r) launch();
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / 5.0;
}

}  // namespace

extern "C" int bem_measure_peaks(bem_ctx* ctx, double* out, void* stream) {
    if (!ctx || !out) return BEM_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const int blocks = ctx->num_sms * 8, threads = 256;
    void* buf = nullptr;
    if (int rc = bem_check_cuda(ctx, cudaMalloc(&buf, sizeof(double) * blocks), "probe buffer")) return rc;
    const double nthreads = double(blocks) * threads;
    double ms32 = time_ms([&] { fma_probe<float><<<blocks, threads, 0, s>>>((float*)buf, 0.999f, 0.001f); }, s);
    double ms64 = time_ms([&] { fma_probe<double><<<blocks, threads, 0, s>>>((double*)buf, 0.999, 0.001); }, s);
    double msmu = time_ms([&] { mufu_probe<<<blocks, threads, 0, s>>>((float*)buf, 0.5f); }, s);
    ctx->launches += 18;
    cudaFree(buf);
    if (int rc = bem_check_cuda(ctx, cudaGetLastError(), "probe kernels")) return rc;
    const double fmas = nthreads * PROBE_ITERS * 8.0;
    out[0] = 2.0 * fmas / (ms32 * 1e-3) / 1e12;  // FP32 TFLOP/s (FMA = 2 flops)
    out[1] = 2.0 * fmas / (ms64 * 1e-3) / 1e12;  // FP64 TFLOP/s
    out[2] = fmas / (msmu * 1e-3) / 1e9;         // MUFU (rsqrt) Gop/s
    return BEM_OK;
}

// Architecture of the device code this library runs on the current device:
// the binaryVersion (major*10 + minor) of one of its kernels, as the runtime
// reports it after loading the module.  100 for the sm_100a build.
extern "C" int bem_binary_version(int* version) {
    if (!version) return BEM_ERR_INVALID;
    cudaFuncAttributes attr;
    cudaError_t e = cudaFuncGetAttributes(&attr, mufu_probe);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return BEM_ERR_CUDA;
    }
    *version = attr.binaryVersion;
    return BEM_OK;
}
