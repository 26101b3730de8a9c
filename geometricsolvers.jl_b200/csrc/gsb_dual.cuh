// Forward-mode dual numbers on the device, so that a residual family written once as a template
// over its scalar type gets its Jacobian from one K-partial pass and its JVP from one 1-partial
// pass, as the reference's R1 Jacobian (`jacobian!!`, src/ad/forwarddiff_static.jl:50-65) and
// JVP (`jvp!!`, src/ad/jvp.jl:96-107) do with ForwardDiff's duals (ForwardDiff 1.4,
// Project.toml:11): a value and K partials, each rule the value operation on the values and the
// derivative rule times the partials (`_mul_partials`, `_div_partials`).
//
// `Real` is the plain value type of the same residual code. Every operation of both types is one
// IEEE operation with its own rounding (no contraction into FMAs) unless the family asks for a
// fused multiply-add (`fmac`), so a family evaluates with the bits its CPU restatement gives.
#pragma once

namespace gsb {

struct Real {
    double v;
};

__device__ __forceinline__ Real operator+(Real a, Real b) { return {__dadd_rn(a.v, b.v)}; }
__device__ __forceinline__ Real operator+(Real a, double c) { return {__dadd_rn(a.v, c)}; }
__device__ __forceinline__ Real operator+(double c, Real a) { return {__dadd_rn(c, a.v)}; }
__device__ __forceinline__ Real operator-(Real a, Real b) { return {__dsub_rn(a.v, b.v)}; }
__device__ __forceinline__ Real operator-(Real a, double c) { return {__dsub_rn(a.v, c)}; }
__device__ __forceinline__ Real operator-(double c, Real a) { return {__dsub_rn(c, a.v)}; }
__device__ __forceinline__ Real operator-(Real a) { return {-a.v}; }
__device__ __forceinline__ Real operator*(Real a, Real b) { return {__dmul_rn(a.v, b.v)}; }
__device__ __forceinline__ Real operator*(double c, Real a) { return {__dmul_rn(c, a.v)}; }
__device__ __forceinline__ Real operator*(Real a, double c) { return {__dmul_rn(a.v, c)}; }
__device__ __forceinline__ Real operator/(Real a, Real b) { return {__ddiv_rn(a.v, b.v)}; }
__device__ __forceinline__ Real operator/(Real a, double c) { return {__ddiv_rn(a.v, c)}; }
__device__ __forceinline__ Real operator/(double c, Real a) { return {__ddiv_rn(c, a.v)}; }
// fma(c, x, acc): the family's own fused product-and-sum
__device__ __forceinline__ Real fmac(double c, Real x, Real acc) { return {__fma_rn(c, x.v, acc.v)}; }
__device__ __forceinline__ Real cst(double c, Real) { return {c}; }
__device__ __forceinline__ double value(Real a) { return a.v; }

template <int K> struct Dual {
    double v;
    double p[K];
};

template <int K> __device__ __forceinline__ Dual<K> cst(double c, const Dual<K>&) {
    Dual<K> r;
    r.v = c;
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = 0.0;
    return r;
}
template <int K> __device__ __forceinline__ double value(const Dual<K>& a) { return a.v; }

template <int K> __device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = __dadd_rn(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __dadd_rn(a.p[k], b.p[k]);
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, double c) {
    Dual<K> r = a;
    r.v = __dadd_rn(a.v, c);
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator+(double c, const Dual<K>& a) {
    Dual<K> r = a;
    r.v = __dadd_rn(c, a.v);
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = __dsub_rn(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __dsub_rn(a.p[k], b.p[k]);
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, double c) {
    Dual<K> r = a;
    r.v = __dsub_rn(a.v, c);
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator-(double c, const Dual<K>& a) {
    Dual<K> r;
    r.v = __dsub_rn(c, a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = -a.p[k];
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator-(const Dual<K>& a) {
    Dual<K> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = -a.p[k];
    return r;
}
// x * y: partials px vy + py vx
template <int K> __device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = __dmul_rn(a.v, b.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __dadd_rn(__dmul_rn(a.p[k], b.v), __dmul_rn(b.p[k], a.v));
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator*(double c, const Dual<K>& a) {
    Dual<K> r;
    r.v = __dmul_rn(c, a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __dmul_rn(c, a.p[k]);
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, double c) {
    Dual<K> r;
    r.v = __dmul_rn(a.v, c);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __dmul_rn(a.p[k], c);
    return r;
}
// x / y: partials px (1 / vy) + py (-(vx / (vy vy)))
template <int K> __device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = __ddiv_rn(a.v, b.v);
    const double ib = __ddiv_rn(1.0, b.v);
    const double q = -__ddiv_rn(a.v, __dmul_rn(b.v, b.v));
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __dadd_rn(__dmul_rn(a.p[k], ib), __dmul_rn(b.p[k], q));
    return r;
}
template <int K> __device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, double c) {
    Dual<K> r;
    r.v = __ddiv_rn(a.v, c);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __ddiv_rn(a.p[k], c);
    return r;
}
// fma(c, x, acc) with a constant c: the value and each partial fused
template <int K>
__device__ __forceinline__ Dual<K> fmac(double c, const Dual<K>& x, const Dual<K>& acc) {
    Dual<K> r;
    r.v = __fma_rn(c, x.v, acc.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.p[k] = __fma_rn(c, x.p[k], acc.p[k]);
    return r;
}

}  // namespace gsb
