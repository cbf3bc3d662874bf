// FP64 FMA throughput of the current GPU, measured: the denominator of the
// narrow phase's FP64 roofline (the ACCD runs on the FP64 pipe, and no other
// measured FP64 figure exists for the device).  Every thread runs eight
// independent fused multiply-add chains in registers, so the FP64 pipe, not
// latency, sets the rate; one wave of 8 blocks of 256 threads per SM.
#include "mclccd_b200.h"

#include <cuda_runtime.h>

namespace mclccd {

__global__ void __launch_bounds__(256) k_fp64_fma(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = 1e-3 * threadIdx.x + j;
    for (int i = 0; i < iters; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) x[j] = fma(x[j], a, b);
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += x[j];
    if (s == -1.0) out[0] = s;   // never true: keeps the chains live
}

} // namespace mclccd

extern "C" int mclccd_fp64_fma_rate(int device, double *tflops)
{
    using namespace mclccd;
    if (!tflops) return MCLCCD_ERR_INVALID;
    *tflops = 0.0;
    int prev = 0, sms = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return MCLCCD_ERR_CUDA;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    double *out = nullptr;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaStream_t st = nullptr;
    if (e == cudaSuccess) e = cudaMalloc(&out, sizeof(double));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&t0);
    if (e == cudaSuccess) e = cudaEventCreate(&t1);
    const int blocks = 8 * sms, iters = 1 << 14;
    float ms = 0.f;
    if (e == cudaSuccess) {
        k_fp64_fma<<<blocks, 256, 0, st>>>(out, iters / 16, 0.999999, 1e-3);   // warm-up
        cudaEventRecord(t0, st);
        k_fp64_fma<<<blocks, 256, 0, st>>>(out, iters, 0.999999, 1e-3);
        cudaEventRecord(t1, st);
        e = cudaEventSynchronize(t1);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
    }
    if (e == cudaSuccess && ms > 0.f)
        *tflops = 2.0 * 8.0 * (double)iters * (double)blocks * 256.0 / (ms * 1e-3) / 1e12;
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    if (st) cudaStreamDestroy(st);
    if (out) cudaFree(out);
    cudaSetDevice(prev);
    return e == cudaSuccess ? MCLCCD_OK : MCLCCD_ERR_CUDA;
}
