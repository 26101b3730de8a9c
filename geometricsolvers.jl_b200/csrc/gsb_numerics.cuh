// Device numerics of the batch solver: Julia's float semantics where the solver's decisions
// depend on them (NaN-propagating max/min, the exact power-of-two scaling `ldexp2`, the scaled
// 2-norm `rnorm`), and the arithmetic policy of the linear algebra.
//
// Policy `Fused` (the default) contracts each product-and-sum into one FMA; policy `Unfused`
// rounds every product and every sum on its own, as Julia evaluates `a * b + c`
// (src/linear/static/lu.jl:58 and the StaticArrays products), so that a run can be compared with
// a CPU restatement bit for bit.
#pragma once

#include <cstdint>

namespace gsb {

constexpr double kNaN = __builtin_nan("");
constexpr double kInf = __builtin_inf();
constexpr double kEps = 2.220446049250313e-16;
constexpr double kSqrtEps = 1.4901161193847656e-08;
constexpr double kFloatmin = 2.2250738585072014e-308;
constexpr double kFloatmax = 1.7976931348623157e308;

enum Code : int { SUCCESS = 0, STALLED = 1, MAXITERS = 2, SINGULAR = 3, NONFINITE = 4,
                  LINESEARCH_FAILED = 5 };

template <bool Fused> struct Arith {
    __device__ __forceinline__ static double mul(double a, double b) { return __dmul_rn(a, b); }
    __device__ __forceinline__ static double add(double a, double b) { return __dadd_rn(a, b); }
    __device__ __forceinline__ static double sub(double a, double b) { return __dsub_rn(a, b); }
    // c + a b
    __device__ __forceinline__ static double madd(double a, double b, double c) {
        return Fused ? __fma_rn(a, b, c) : __dadd_rn(__dmul_rn(a, b), c);
    }
    // c - a b
    __device__ __forceinline__ static double msub(double a, double b, double c) {
        return Fused ? __fma_rn(-a, b, c) : __dsub_rn(c, __dmul_rn(a, b));
    }
    __device__ __forceinline__ static float mul(float a, float b) { return __fmul_rn(a, b); }
    __device__ __forceinline__ static float add(float a, float b) { return __fadd_rn(a, b); }
    __device__ __forceinline__ static float sub(float a, float b) { return __fsub_rn(a, b); }
    __device__ __forceinline__ static float madd(float a, float b, float c) {
        return Fused ? __fmaf_rn(a, b, c) : __fadd_rn(__fmul_rn(a, b), c);
    }
    __device__ __forceinline__ static float msub(float a, float b, float c) {
        return Fused ? __fmaf_rn(-a, b, c) : __fsub_rn(c, __fmul_rn(a, b));
    }
};

__device__ __forceinline__ bool isfin(double x) { return isfinite(x); }
__device__ __forceinline__ bool isfin(float x) { return isfinite(x); }

// Julia's max/min on floats: NaN propagates, max(-0.0, 0.0) = 0.0, min(-0.0, 0.0) = -0.0.
template <class T> __device__ __forceinline__ T jmax(T a, T b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a == b) return signbit(a) ? b : a;
    return a > b ? a : b;
}
template <class T> __device__ __forceinline__ T jmin(T a, T b) {
    if (a != a) return a;
    if (b != b) return b;
    if (a == b) return signbit(a) ? a : b;
    return a < b ? a : b;
}

template <class T> struct FBits;
template <> struct FBits<double> {
    using U = unsigned long long;
    static constexpr int sig = 52, ebits = 11, raw_max = 2047, emax = 1023;
    static constexpr U sign_mask = 1ull << 63, exp_mask = 0x7ffull << 52,
                       sig_mask = (1ull << 52) - 1;
    __device__ __forceinline__ static U bits(double x) { return (U)__double_as_longlong(x); }
    __device__ __forceinline__ static double from(U u) { return __longlong_as_double((long long)u); }
    __device__ __forceinline__ static int clz(U x) { return __clzll((long long)x); }
};
template <> struct FBits<float> {
    using U = unsigned int;
    static constexpr int sig = 23, ebits = 8, raw_max = 255, emax = 127;
    static constexpr U sign_mask = 1u << 31, exp_mask = 0xffu << 23, sig_mask = (1u << 23) - 1;
    __device__ __forceinline__ static U bits(float x) { return (U)__float_as_int(x); }
    __device__ __forceinline__ static float from(U u) { return __int_as_float((int)u); }
    __device__ __forceinline__ static int clz(U x) { return __clz((int)x); }
};

// `x * 2^e`, exact unless the result leaves the range, rounded to nearest-even into the
// subnormals: the bit algorithm of the reference's ldexp2 (src/linear/factors.jl:726-758).
template <class T> __device__ __forceinline__ T ldexp2(T x, int e) {
    using B = FBits<T>;
    using U = typename B::U;
    U xu = B::bits(x);
    U sign = xu & B::sign_mask;
    U xs = xu & ~B::sign_mask;
    if (xs >= B::exp_mask || xs == 0) return x;
    int k = (int)(xs >> B::sig);
    if (k == 0) {
        int m = B::clz(xs) - B::ebits;
        xs <<= m;
        k = 1 - m;
    }
    U sig = (xs & B::sig_mask) | (U(1) << B::sig);
    k += e;
    if (k >= B::raw_max) return B::from(sign | B::exp_mask);
    if (k > 0) return B::from(sign | (U(k) << B::sig) | (sig & B::sig_mask));
    if (k <= -B::sig - 1) return B::from(sign);
    int shift = 1 - k;
    U lower = sig & ((U(1) << shift) - U(1));
    U half = U(1) << (shift - 1);
    U sub = sig >> shift;
    if (lower > half || (lower == half && (sub & 1))) sub += 1;
    return B::from(sign | sub);
}

static __device__ __noinline__ double ldexp2_slow(double x, int e);
static __device__ __noinline__ float ldexp2_slow(float x, int e);

// 2^e as a double for e in [-1074, 1023] (subnormal below -1022): exactly representable.
__device__ __forceinline__ double pow2d(int e) {
    return e >= -1022 ? __longlong_as_double((long long)(e + 1023) << 52)
                      : __longlong_as_double(1ll << (e + 1074));
}
__device__ __forceinline__ float pow2f(int e) {
    return e >= -126 ? __int_as_float((e + 127) << 23) : __int_as_float(1 << (e + 149));
}

// ldexp2(x, e) as one multiplication where 2^e is representable: the product x 2^e is exact
// before rounding, so the single IEEE round-to-nearest-even of the multiplication is the
// rounding of ldexp2 (exact in the normal range, nearest-even into the subnormals, Inf on
// overflow, NaN and Inf unchanged). Other exponents take the bitwise routine.
// For e in (1023, 2046] it is two multiplications: by 2^1023, exact unless it overflows (and
// then the result overflows too), and by 2^(e - 1023), the one rounding.
__device__ __forceinline__ double scale2(double x, int e) {
    if (e > 1023 && e <= 2046) return __dmul_rn(__dmul_rn(x, pow2d(1023)), pow2d(e - 1023));
    return (e >= -1074 && e <= 1023) ? __dmul_rn(x, pow2d(e)) : ldexp2_slow(x, e);
}
// scale2 for an exponent known to lie in [-1074, 2046], with no call.
__device__ __forceinline__ double scale2_in(double x, int e) {
    if (e > 1023) return __dmul_rn(__dmul_rn(x, pow2d(1023)), pow2d(e - 1023));
    return __dmul_rn(x, pow2d(e));
}
__device__ __forceinline__ float scale2(float x, int e) {
    if (e > 127 && e <= 254) return __fmul_rn(__fmul_rn(x, pow2f(127)), pow2f(e - 127));
    return (e >= -149 && e <= 127) ? __fmul_rn(x, pow2f(e)) : ldexp2_slow(x, e);
}
__device__ __forceinline__ float scale2_in(float x, int e) {
    if (e > 127) return __fmul_rn(__fmul_rn(x, pow2f(127)), pow2f(e - 127));
    return __fmul_rn(x, pow2f(e));
}

// Loads and stores of shared memory by its 32-bit shared-window address, as volatile PTX: the
// compiler keeps them where they stand (a parameter block is read at each use instead of being
// held in registers across the solve) and they issue as shared-memory instructions, not as
// generic loads through the L1 path.
__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ double lds(unsigned addr) {
    double v;
    asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
    return v;
}
__device__ __forceinline__ void sts(unsigned addr, double v) {
    asm volatile("st.shared.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}
// Two consecutive doubles at a 16-byte aligned shared address, as one 16-byte access.
__device__ __forceinline__ void lds2(unsigned addr, double& v0, double& v1) {
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v0), "=d"(v1) : "r"(addr));
}
__device__ __forceinline__ void sts2(unsigned addr, double v0, double v1) {
    asm volatile("st.shared.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v0), "d"(v1) : "memory");
}

// Julia's `exponent` of a finite nonzero value.
__device__ __forceinline__ int jexponent(double x) { return ilogb(x); }
__device__ __forceinline__ int jexponent(float x) { return ilogbf(x); }

// norm2 as a left fold (src/base/reductions.jl:19-22).
template <bool F, int L, class T> __device__ __forceinline__ T norm2(const T (&a)[L]) {
    T s = Arith<F>::mul(a[0], a[0]);
#pragma unroll
    for (int i = 1; i < L; ++i) s = Arith<F>::madd(a[i], a[i], s);
    return s;
}

// rnorm with the scaled fallback (src/base/reductions.jl:348-364).
template <bool F, int L, class T> __device__ __forceinline__ T rnorm_from(const T (&a)[L], T s) {
    const T tiny = sizeof(T) == 8 ? T(kFloatmin) : T(1.17549435e-38f);
    if (isfin(s) && s >= T(L) * tiny) return sqrt(s);
    T m = jmax(fabs(a[0]), T(0));
#pragma unroll
    for (int i = 1; i < L; ++i) m = jmax(m, jmax(fabs(a[i]), T(0)));
    if (m == T(0) || !isfin(m)) return m;
    int e = jexponent(m);
    T t = scale2_in(a[0], -e);
    T acc = Arith<F>::mul(t, t);
#pragma unroll
    for (int i = 1; i < L; ++i) {
        T u = scale2_in(a[i], -e);
        acc = Arith<F>::madd(u, u, acc);
    }
    return scale2_in(T(sqrt(acc)), e);
}
template <bool F, int L, class T> __device__ __forceinline__ T rnorm(const T (&a)[L]) {
    return rnorm_from<F, L, T>(a, norm2<F, L, T>(a));
}

template <int L, class T> __device__ __forceinline__ T rmaxnorm(const T (&a)[L]) {
    T m = fabs(a[0]);
#pragma unroll
    for (int i = 1; i < L; ++i) m = jmax(m, T(fabs(a[i])));
    return m;
}

// matrix_exponent over the bits of |a| (src/linear/factors.jl:833-843): the exponent of the
// largest |a_i| (0 when it is zero or not finite), clamped to [-1023, 1023]. The largest |a_i|
// has the largest high word (sign shifted out), so a tree of 32-bit maxima (associative: the
// order does not matter) gives its exponent field: for a normal maximum the field is the
// exponent; a subnormal maximum has an exponent below -1022, which the clamp makes -1023; Inf
// and NaN give 0; and when every high word is zero the low words tell zero from subnormal.
template <int L> __device__ __forceinline__ int matrix_exponent(const double (&a)[L]) {
    unsigned h[L];
#pragma unroll
    for (int i = 0; i < L; ++i) h[i] = (unsigned)__double2hiint(a[i]) << 1;
#pragma unroll
    for (int w = 1; w < L; w *= 2)
#pragma unroll
        for (int i = 0; i + w < L; i += 2 * w) h[i] = h[i] > h[i + w] ? h[i] : h[i + w];
    const int field = (int)(h[0] >> 21);
    if (field == 2047) return 0;          // Inf or NaN
    if (field != 0) return field - 1023;  // normal: in [-1022, 1023]
    if (h[0] != 0) return -1023;          // subnormal
    unsigned lo = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) lo |= (unsigned)__double2loint(a[i]);
    return lo != 0 ? -1023 : 0;           // subnormal, or all zero
}

// A key whose unsigned order is that of |x| between values of distinct high words (the high
// 32 bits with the sign shifted out): key(x) < key(y) implies |x| < |y|; a NaN has a key above
// every finite value's.
__device__ __forceinline__ unsigned mag_key(double x) { return (unsigned)__double2hiint(x) << 1; }
__device__ __forceinline__ unsigned mag_key(float x) { return __float_as_uint(x) << 1; }

// The correctly rounded reciprocal: the bits of 1 / x.
__device__ __forceinline__ double crcp(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float crcp(float x) { return __frcp_rn(x); }

// headroom(n) = 2 + ceil(log2 n) (src/linear/factors.jl:890), a constant of the size.
__host__ __device__ constexpr int headroom(int n) {
    int b = 0;
    unsigned v = unsigned(n - 1);
    while (v) {
        ++b;
        v >>= 1;
    }
    return 2 + b;
}

// rhs_exponent (src/linear/factors.jl:880-885).
template <int L> __device__ __forceinline__ int rhs_exponent(const double (&r)[L], int e) {
    int m = matrix_exponent<L>(r);
    int lo = e < 0 ? e : 0;
    int a = m > 0 ? 0 : (m < lo ? lo : m);
    int b = m - (1023 - headroom(L));
    return a > b ? a : b;
}

// True when rhs_exponent(r, 0) is 0: with e = 0 that exponent is max(0, m - (1023 - headroom)),
// m the exponent of the largest |r_i| (0 when that is Inf or NaN), so it is 0 unless the largest
// |r_i| is finite with an exponent above 1023 - headroom. Decided on the exponent field of the
// largest high word, as matrix_exponent reads it.
template <int L> __device__ __forceinline__ bool rhs_unscaled(const double (&r)[L]) {
    unsigned h = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        const unsigned v = (unsigned)__double2hiint(r[i]) << 1;
        h = h > v ? h : v;
    }
    const int field = (int)(h >> 21);
    return field == 2047 || field - 1023 <= 1023 - headroom(L);
}

static __device__ __noinline__ double ldexp2_slow(double x, int e) { return ldexp2(x, e); }
static __device__ __noinline__ float ldexp2_slow(float x, int e) { return ldexp2(x, e); }

}  // namespace gsb
