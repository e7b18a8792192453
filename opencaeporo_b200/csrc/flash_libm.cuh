// flash_libm.cuh -- the flash kernels' own FP64 exponential and logarithm:
// table-driven, short dependent chains, and within one unit in the last
// place of the exact result.
//
// The reference evaluates exp and log with the host C library; CUDA's
// device functions return different last bits for a few percent of
// arguments (measured on the B200: 6.2 % of exp results differ from glibc's
// on 4M arguments in [-80, 20]), and their dependent latency is ~147 (exp)
// and ~271 (log) cycles. These two follow the published table-driven
// methods -- P. T. P. Tang, "Table-driven implementation of the exponential
// function in IEEE floating-point arithmetic", ACM TOMS 15(2), 1989, and
// "Table-driven implementation of the logarithm function in IEEE
// floating-point arithmetic", ACM TOMS 16(4), 1990 -- with their reductions
// carried in fused multiply-adds, Taylor polynomials evaluated by Estrin's
// scheme, and tables computed to 60 digits (gen_libm_tables.py). Measured
// on the B200: ~130 and ~148 cycles of dependent latency; last bits equal
// to glibc's for 99.35 % (exp) and 99.97 % (log) of arguments, never more
// than one unit apart. Arguments outside the fast paths' ranges (exp:
// |x| >= 700 or NaN; log: x not a positive normal number in [2^-1000,
// 2^1000], infinities, NaN) take CUDA's functions, in one out-of-line copy
// each.
#pragma once

#include <cuda_runtime.h>

#include "flash_libm_tables.h"

namespace ocpf {

static __device__ __noinline__ double dexp_wide(double x) { return exp(x); }
static __device__ __noinline__ double dlog_wide(double x) { return log(x); }

// exp(x) = 2^k 2^(j/32) exp(r): N = 32 k + j = rint(32 x / ln 2) from the
// rounding constant 1.5 * 2^52 (N is the low word of t); r = x - N ln2/32 in
// two fused steps (|r| <= ln2/64); exp(r) - 1 by its Taylor series to r^6
// (truncation below 4e-18 relative); the table head and tail give
// 2^(j/32) to ~106 bits; the scale 2^k is an exponent-field product.
__device__ __forceinline__ double dexp(double x)
{
    if (!(fabs(x) < 700.0)) return dexp_wide(x);
    const double SH = 6755399441055744.0;  // 1.5 * 2^52
    const double t  = fma(x, k32ByLn2, SH);
    const double N  = t - SH;
    const int    n  = __double2loint(t);
    double       r  = fma(-N, kLn2By32Head, x);
    r               = fma(-N, kLn2By32Tail, r);
    const int    j  = n & 31;
    const double2 T = __ldg(reinterpret_cast<const double2*>(kExpTable) + j);
    const double r2 = r * r;
    const double A  = fma(1.0 / 6, r, 0.5);
    const double B  = fma(1.0 / 120, r, 1.0 / 24);
    const double r4 = r2 * r2;
    double       q  = fma(r2, B, A);
    q               = fma(r4, 1.0 / 720, q);
    const double p  = fma(r2, q, r);  // exp(r) - 1
    const double s  = fma(T.x, p, T.y) + T.x;
    return s * __hiloint2double(((n >> 5) + 1023) << 20, 0);
}

// ln(x) = k ln2 - ln(c_j) + ln(1 + r): x = 2^k m with m in [sqrt(2)/2,
// sqrt(2)); c_j a 10-bit reciprocal of m's interval midpoint (c = 1 on the
// intervals touching m = 1, so r = m - 1 exactly there and arguments near
// one keep their relative accuracy); r = m c_j - 1 in one fused
// multiply-add (|r| < 2^-6.9); ln(1 + r) by its Taylor series to r^9
// (truncation below 2e-22); k ln2_head - ln(c_j)_head exact (both heads are
// multiples of 2^-42), the tails added to the small part first.
__device__ __forceinline__ double dlog(double x)
{
    const int hi = __double2hiint(x);
    if ((unsigned)(hi - 0x01700000) >= (unsigned)(0x7e700000 - 0x01700000)) return dlog_wide(x);
    const int  lo  = __double2loint(x);
    const int  mh  = hi & 0x000fffff;
    const bool big = mh >= 0x6a09e;  // m >= sqrt(2): use m / 2 and k + 1
    const int  k   = (hi >> 20) - 1023 + (big ? 1 : 0);
    const double m = __hiloint2double(((big ? 1022 : 1023) << 20) | mh, lo);
    const int  j   = (big ? 0 : 64) + (mh >> 14);
    const double2 c0 = __ldg(reinterpret_cast<const double2*>(kLogTable) + 2 * j);
    const double2 c1 = __ldg(reinterpret_cast<const double2*>(kLogTable) + 2 * j + 1);
    const double r  = fma(m, c0.x, -1.0);
    const double r2 = r * r;
    const double a0 = fma(1.0 / 3, r, -0.5);
    const double a1 = fma(1.0 / 5, r, -0.25);
    const double a2 = fma(1.0 / 7, r, -1.0 / 6);
    const double a3 = fma(1.0 / 9, r, -0.125);
    const double r4 = r2 * r2;
    const double b0 = fma(r2, a1, a0);
    const double b1 = fma(r2, a3, a2);
    const double q  = fma(r4, b1, b0);  // (ln(1 + r) - r) / r^2
    const double kd = (double)k;
    const double sh = fma(kd, kLn2Head, c0.y);
    const double sl = fma(kd, kLn2Tail, c1.x);
    return sh + (fma(r2, q, sl) + r);
}

}  // namespace ocpf
