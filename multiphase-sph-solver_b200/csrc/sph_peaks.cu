// sph_peaks.cu -- the FP64 and FP32 arithmetic rates of the device, measured
// (the denominators of the compute side of the step's roofline: the copy
// bandwidth and the BF16 tensor rate the driver measures say nothing about
// the FP64 pipe the drop-in form's pair arithmetic runs on).
//
// Each thread runs eight independent fused multiply-add chains (explicit
// __fma_rn / __fmaf_rn, which this file's -fmad=false build leaves as
// written), so the pipe, not a dependency, sets the rate; a grid of 32 blocks
// of 256 threads per SM keeps every SM's schedulers issuing.  The rate is the
// multiply-adds' flops (two per instruction) over the kernel's device time.
#include <cuda_runtime.h>

#include "../../include/sphgpu.h"

namespace {

constexpr int kChains = 8;

template <typename T>
__device__ __forceinline__ T fma_rn(T a, T b, T c);
template <>
__device__ __forceinline__ double fma_rn<double>(double a, double b, double c) { return __fma_rn(a, b, c); }
template <>
__device__ __forceinline__ float fma_rn<float>(float a, float b, float c) { return __fmaf_rn(a, b, c); }

template <typename T>
__global__ void __launch_bounds__(256) k_fma_rate(T* sink, int iters)
{
    T a[kChains];
    const T m = T(0.9999999), c = T(1.0e-7);
    for (int k = 0; k < kChains; k++) a[k] = T(threadIdx.x + k) * T(1.0e-3);
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < kChains; k++) a[k] = fma_rn<T>(a[k], m, c);
    }
    T s = T(0);
    for (int k = 0; k < kChains; k++) s = s + a[k];
    // never true for these inputs: keeps the chains live without a store
    if (s == T(-1)) sink[blockIdx.x] = s;
}

template <typename T>
int rate(int sms, cudaStream_t st, T* sink, double* tflops)
{
    const int blocks = 32 * sms, threads = 256, iters = 2048;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) return SPHGPU_E_CUDA;
    float best = 0.f;
    for (int rep = 0; rep < 4; rep++) {      // the first launch warms the clocks up
        cudaEventRecord(e0, st);
        k_fma_rate<T><<<blocks, threads, 0, st>>>(sink, iters);
        cudaEventRecord(e1, st);
        if (cudaEventSynchronize(e1) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && (best == 0.f || ms < best)) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess || best <= 0.f) return SPHGPU_E_CUDA;
    const double flops = 2.0 * kChains * (double)iters * threads * blocks;
    *tflops = flops / (best * 1.0e-3) / 1.0e12;
    return 0;
}

}  // namespace

extern "C" int sphgpu_pipe_peaks(int device, double* fp64_tflops, double* fp32_tflops)
{
    if (!fp64_tflops || !fp32_tflops) return SPHGPU_E_ARG;
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();      // this call's own error: not left for the caller's next check
        return SPHGPU_E_NODEVICE;
    }
    cudaGetLastError();          // an earlier call's last error is not this measurement's
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || sms <= 0)
        return SPHGPU_E_CUDA;
    cudaStream_t st;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return SPHGPU_E_CUDA;
    void* sink = nullptr;
    int r = cudaMalloc(&sink, sizeof(double) * 32 * (size_t)sms) == cudaSuccess ? 0 : SPHGPU_E_CUDA;
    if (!r) r = rate<double>(sms, st, (double*)sink, fp64_tflops);
    if (!r) r = rate<float>(sms, st, (float*)sink, fp32_tflops);
    if (sink) cudaFree(sink);
    cudaStreamDestroy(st);
    return r;
}
