// peak.cu -- measures the device's FP64 / FP32 FMA throughput, the
// denominator of the flash kernels' compute roofline (the driver's measured
// peaks cover HBM bandwidth and bf16 tensor throughput only).
#include <cuda_runtime.h>

#include "ocp_flash.h"

namespace {

template <typename R>
__global__ void __launch_bounds__(256) k_fma_peak(R* sink, int iters, R b, R c)
{
    R a[8];
#pragma unroll
    for (int j = 0; j < 8; j++) a[j] = (R)(threadIdx.x + j) * (R)1e-3;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int j = 0; j < 8; j++) a[j] = fma(a[j], b, c);
    }
    R s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += a[j];
    if (s == (R)-12345.0) sink[0] = s;  // keeps the chains live
}

template <typename R>
int run(int device, double* tflops)
{
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return OCPF_ECUDA;
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, device);
    R* sink = nullptr;
    if (cudaMalloc(&sink, sizeof(R)) != cudaSuccess) return OCPF_ENOMEM;
    const int    blocks = prop.multiProcessorCount * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t  e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0);
        k_fma_peak<R><<<blocks, threads>>>(sink, iters, (R)0.999999, (R)1e-7);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    const cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    cudaSetDevice(prev);
    if (err != cudaSuccess) return OCPF_ECUDA;
    const double fl = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = fl / (best * 1e-3) / 1e12;
    return OCPF_OK;
}

}  // namespace

extern "C" int ocpf_measure_fma_peak(int device, int bits, double* tflops)
{
    if (!tflops) return OCPF_EINVAL;
    if (bits == 64) return run<double>(device, tflops);
    if (bits == 32) return run<float>(device, tflops);
    return OCPF_EINVAL;
}
