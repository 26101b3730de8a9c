// exp(x) in double precision by Tang's table-driven method (P. T. P. Tang, "Table-driven
// implementation of the exponential function in IEEE floating-point arithmetic", ACM TOMS 15(2),
// 1989), written once for the device and the host, so that the exponential-sum family gives the
// same bits in the batch kernel and in its CPU check.
//
//   x = (128 e + j) (ln 2 / 128) + r,   k = 128 e + j = x 128 / ln 2 rounded,  0 <= j < 128,
//   r = (x - k L1) - k L2 with L1 + L2 = ln 2 / 128 and k L1 exact (L1 has 35 significant
//   bits, |k| < 2^18), so |r| <= ln 2 / 256 + a few ulp;
//   exp(x) = 2^e 2^(j/128) e^r ~ 2^e (T[j] + (T[j] p(r) + T_lo[j])), p(r) = e^r - 1 by its
//   Taylor polynomial of degree 5 (the remainder r^6 / 720 < 6e-19 is far below 2^-53).
// The table T + T_lo holds 2^(j/128) to about 106 bits (csrc/gsb_exp_table.h, generated by
// make_exp_table.py). Each operation is a single IEEE operation or a fused multiply-add on
// both sides (device __fma_rn, host std::fma), so host and device agree bit for bit. The error is
// below 0.52 ulp over the normal range (the CPU tests measure it against long double).
#pragma once

#include <stdint.h>

#include <cmath>
#include <cstring>

#include "gsb_exp_table.h"

#if defined(__CUDACC__)
#define GSB_EXP_FN __host__ __device__ __forceinline__
#else
#define GSB_EXP_FN inline
#endif

namespace gsb_exp {

#if defined(__CUDACC__)
static __device__ const double kHiDev[128] = GSB_EXP_TABLE_HI;
static __device__ const double kLoDev[128] = GSB_EXP_TABLE_LO;
#endif
static const double kHiHost[128] = GSB_EXP_TABLE_HI;
static const double kLoHost[128] = GSB_EXP_TABLE_LO;

GSB_EXP_FN double fma_(double a, double b, double c) {
#if defined(__CUDA_ARCH__)
    return __fma_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
GSB_EXP_FN int lo32_(double v) {  // the low 32 bits of v's representation
#if defined(__CUDA_ARCH__)
    return __double2loint(v);
#else
    uint64_t b;
    std::memcpy(&b, &v, sizeof b);
    return (int)(uint32_t)b;
#endif
}
GSB_EXP_FN double pow2_(int e) {  // 2^e for e in [-1022, 1023], exactly
    const uint64_t b = (uint64_t)(e + 1023) << 52;
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)b);
#else
    double v;
    std::memcpy(&v, &b, sizeof v);
    return v;
#endif
}

// The largest x whose exp is finite, and the x below which exp rounds to 0.
constexpr double kOverflow = 0x1.62e42fefa39efp+9;    // 709.78271289338397
constexpr double kUnderflow = -0x1.74910d52d3052p+9;  // -745.13321910194122
constexpr double kShifter = 0x1.8p52;                 // 1.5 2^52

// exp(x) = y 2^e for |x| > 708 or x NaN: the results near and beyond the ends of the range.
#if defined(__CUDA_ARCH__)
__device__ __noinline__
#else
inline
#endif
double exp_edge(double x, double y, int e) {
    if (!(x == x)) return x;  // NaN
    if (x > kOverflow) return __builtin_inf();
    if (x < kUnderflow) return 0.0;
    if (e >= -1021) return e <= 1023 ? y * pow2_(e) : (y * pow2_(1023)) * pow2_(e - 1023);
    // a subnormal result: scale by 2^(e + 64) exactly, then by 2^-64 with the one rounding
    return (y * pow2_(e + 64)) * pow2_(-64);
}

GSB_EXP_FN double exp(double x) {
    // k = x 128 / ln 2 rounded to an integer: the fused product plus 1.5 2^52 rounds once, to a
    // double whose last bits hold k (|k| < 2^31 for every x that reaches the common path)
    const double t = fma_(x, GSB_EXP_INV_STEP, kShifter);
    const double kd = t - kShifter;
    const int k = lo32_(t);
    const double r1 = fma_(-kd, GSB_EXP_STEP_HI, x);  // exact: k L1 is exact and near x
    const double r = fma_(-kd, GSB_EXP_STEP_LO, r1);
    // p(r) = r + r^2 (1/2 + r (1/6 + r (1/24 + r / 120)))
    double q = fma_(r, 1.0 / 120.0, 1.0 / 24.0);
    q = fma_(r, q, 1.0 / 6.0);
    q = fma_(r, q, 0.5);
    const double p = fma_(r * r, q, r);
    const int j = k & 127;
    const int e = k >> 7;  // floor(k / 128)
#if defined(__CUDA_ARCH__)
    const double hi = __ldg(kHiDev + j), lo = __ldg(kLoDev + j);
#else
    const double hi = kHiHost[j], lo = kLoHost[j];
#endif
    const double y = hi + fma_(hi, p, lo);  // 2^(j/128) e^r, in [2^-1/256, 2^(1+1/256)]
    // |x| <= 708: e in [-1022, 1021] and y 2^e a normal number, one exact scaling
    if (fabs(x) <= 708.0) return y * pow2_(e);
    return exp_edge(x, y, e);
}

}  // namespace gsb_exp
