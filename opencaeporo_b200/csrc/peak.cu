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

// ---------------------------------------------------------------- ddiv check
#include "flash_common.cuh"

namespace {

__device__ __forceinline__ unsigned long long xs_next(unsigned long long& s)
{
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return s;
}

// A double with a uniformly random significand and sign, and an exponent
// uniform in [emin, emax].
__device__ __forceinline__ double xs_double(unsigned long long& s, int emin, int emax)
{
    const unsigned long long m    = xs_next(s) & ((1ull << 52) - 1);
    const int                e    = emin + (int)(xs_next(s) % (unsigned long long)(emax - emin + 1));
    const unsigned long long sign = xs_next(s) & 1ull;
    return __longlong_as_double((long long)((sign << 63) | ((unsigned long long)(e + 1023) << 52) | m));
}

// Replaces the significand's low three bits (mode 1) or sets it within
// eight units of all ones (mode 2): operands next to a power of two.
__device__ __forceinline__ double xs_near_pow2(unsigned long long& s, double v)
{
    unsigned long long b = (unsigned long long)__double_as_longlong(v) & ~((1ull << 52) - 1);
    b |= (xs_next(s) & 1) ? (xs_next(s) & 7ull) : (((1ull << 52) - 1) - (xs_next(s) & 7ull));
    return __longlong_as_double((long long)b);
}

// ocpf::ddiv(a, b) against a / b on `per_thread` random pairs per thread:
// mode 0 exponents in [-20, 20]; 1 in [-500, 500]; 2 the divisor, 3 the
// dividend next to a power of two; 4 quotients next to one; 5 one operand
// outside the fast path's range (zeros, extremes, infinities).
__global__ void k_check_ddiv(unsigned long long* bad, int per_thread, unsigned long long seed, int mode)
{
    const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    unsigned long long       s   = seed ^ (tid * 0x9E3779B97F4A7C15ull) ^ 0x5DEECE66Dull;
    if (!s) s = 1;
    unsigned long long n = 0;
    for (int i = 0; i < per_thread; i++) {
        const int lo = mode == 1 ? -500 : -20, hi = mode == 1 ? 500 : 20;
        double    a = xs_double(s, lo, hi), b = xs_double(s, lo, hi);
        if (mode == 2) b = xs_near_pow2(s, b);
        if (mode == 3) a = xs_near_pow2(s, a);
        if (mode == 4) a = b * (1.0 + (double)(xs_next(s) % 1024) * 1.1102230246251565e-16);
        if (mode == 5) {
            const double ex[6] = {0.0, -0.0, 1e-300, 1e300, __longlong_as_double(0x7ff0000000000000ll), 3e-160};
            if (xs_next(s) & 1)
                a = ex[xs_next(s) % 6];
            else
                b = ex[xs_next(s) % 6];
        }
        const double q = a / b, d = ocpf::ddiv(a, b);
        const bool   both_nan = (q != q) && (d != d);
        if (!both_nan && __double_as_longlong(q) != __double_as_longlong(d)) n++;
    }
    if (n) atomicAdd(bad, n);
}

// Dependent-chain latency of ddiv (cycles per division), one thread.
__global__ void k_ddiv_latency(double* out, long long* cyc, double a, double b, int n)
{
    double          x  = b;
    const long long t0 = clock64();
    for (int i = 0; i < n; i++) x = ocpf::ddiv(a, x);
    const long long t1 = clock64();
    cyc[0]             = t1 - t0;
    out[0]             = x;
}

}  // namespace

extern "C" int ocpf_selfcheck_division(int device, int64_t pairs, uint64_t seed, int64_t* mismatches,
                                       double* cycles)
{
    if (!mismatches || pairs < 0) return OCPF_EINVAL;
    int prev = 0;
    cudaGetDevice(&prev);
    if (cudaSetDevice(device) != cudaSuccess) return OCPF_ECUDA;
    unsigned long long* bad = nullptr;
    double*             out = nullptr;
    long long*          cyc = nullptr;
    int                 rc  = OCPF_OK;
    if (cudaMalloc(&bad, sizeof(unsigned long long)) != cudaSuccess || cudaMalloc(&out, sizeof(double)) != cudaSuccess ||
        cudaMalloc(&cyc, sizeof(long long)) != cudaSuccess)
        rc = OCPF_ENOMEM;
    unsigned long long total = 0;
    if (rc == OCPF_OK) {
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, device);
        const int     blocks = prop.multiProcessorCount * 4, threads = 256;
        const int64_t per    = pairs / 6 / ((int64_t)blocks * threads);
        cudaMemset(bad, 0, sizeof(unsigned long long));
        for (int mode = 0; mode < 6; mode++)
            k_check_ddiv<<<blocks, threads>>>(bad, (int)(per > 0 ? per : 1), seed + 7919ull * mode, mode);
        if (cycles) {
            k_ddiv_latency<<<1, 1>>>(out, cyc, 1.7, 1.3, 1000);
            k_ddiv_latency<<<1, 1>>>(out, cyc, 1.7, 1.3, 1000);
        }
        long long c = 0;
        if (cudaMemcpy(&total, bad, sizeof(total), cudaMemcpyDeviceToHost) != cudaSuccess ||
            (cycles && cudaMemcpy(&c, cyc, sizeof(c), cudaMemcpyDeviceToHost) != cudaSuccess))
            rc = OCPF_ECUDA;
        if (cycles) *cycles = (double)c / 1000;
    }
    if (bad) cudaFree(bad);
    if (out) cudaFree(out);
    if (cyc) cudaFree(cyc);
    cudaSetDevice(prev);
    *mismatches = (int64_t)total;
    return rc;
}
