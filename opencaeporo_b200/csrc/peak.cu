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

namespace {

// One thread, clock64: the latency of the FP64 operations that bound a
// single cell's chain of dependent iterations (the restart path).
__global__ void k_fp64_latency(double* out, long long* cyc, double a, double b, int n)
{
    double    x = b, y[12];
    long long t0, t1;
#pragma unroll
    for (int i = 0; i < 12; i++) y[i] = b + i * 1e-3;
    t0 = clock64();  // dependent divisions
    for (int i = 0; i < n; i++) x = a / x;
    t1     = clock64();
    cyc[0] = t1 - t0;
    out[0] = x;
    t0     = clock64();  // twelve independent division chains (cycles per division)
    for (int i = 0; i < n; i++) {
#pragma unroll
        for (int j = 0; j < 12; j++) y[j] = a / y[j];
    }
    t1       = clock64();
    cyc[1]   = (t1 - t0) / 12;
    double s = 0;
#pragma unroll
    for (int j = 0; j < 12; j++) s += y[j];
    out[1] = s;
    x      = b;
    t0     = clock64();  // dependent FMA
    for (int i = 0; i < n; i++) x = fma(x, a, 1e-3);
    t1     = clock64();
    cyc[2] = t1 - t0;
    out[2] = x;
    x      = b;
    t0     = clock64();  // dependent exp
    for (int i = 0; i < n; i++) x = exp(x * 1e-3);
    t1     = clock64();
    cyc[3] = t1 - t0;
    out[3] = x;
    x      = b + 2;
    t0     = clock64();  // dependent log
    for (int i = 0; i < n; i++) x = log(x + 3.0);
    t1     = clock64();
    cyc[4] = t1 - t0;
    out[4] = x;
    x      = 0.3;
    t0     = clock64();  // dependent acos + cos
    for (int i = 0; i < n; i++) x = cos(acos(x) * 0.5);
    t1     = clock64();
    cyc[5] = t1 - t0;
    out[5] = x;
}

}  // namespace

extern "C" int ocpf_measure_fp64_latency(int device, double* cycles)
{
    if (!cycles) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return OCPF_ECUDA;
    double*    out = nullptr;
    long long* cyc = nullptr;
    int        rc  = OCPF_OK;
    if (cudaMalloc(&out, 8 * sizeof(double)) != cudaSuccess || cudaMalloc(&cyc, 8 * sizeof(long long)) != cudaSuccess)
        rc = OCPF_ENOMEM;
    const int n = 1000;
    long long h[8] = {};
    if (rc == OCPF_OK) {
        k_fp64_latency<<<1, 1>>>(out, cyc, 1.7, 1.3, n);  // warm-up (instruction cache)
        k_fp64_latency<<<1, 1>>>(out, cyc, 1.7, 1.3, n);
        if (cudaMemcpy(h, cyc, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) rc = OCPF_ECUDA;
    }
    if (out) cudaFree(out);
    if (cyc) cudaFree(cyc);
    cudaSetDevice(prev);
    if (rc != OCPF_OK) return rc;
    for (int i = 0; i < 6; i++) cycles[i] = (double)h[i] / n;
    return OCPF_OK;
}
