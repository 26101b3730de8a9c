// The warp form of the per-system Newton solve, for systems too large for one thread's
// registers (n = 12 ... 32): a team of T = 16 or 32 lanes (an aligned part of a warp) runs one
// system. Lane i < n owns component i of every vector (iterate, residual, direction, trial) and
// row i of the Jacobian's factor; the factor lives in shared memory, so the column loop of the
// elimination and the row exchanges of partial pivoting take runtime indices.
//
// Every operation is the one-thread solve's (gsb_newton.cuh) in the same order: the LU of
// src/linear/static/lu.jl:24-92 (first largest pivot, info = first zero pivot), the scalings of
// factor_matrix and ldiv!! (src/linear/factors.jl:802-949), the left-fold norms and products of
// src/base/reductions.jl, Backtracking and Static (src/globalization/linefunction.jl:114-199,
// backtracking.jl:62-132), refinement (src/nonlinear/refinement.jl:211-244) and the mixed
// step's promotion (src/nonlinear/newton.jl:1604-1720). A fold over a distributed vector
// broadcasts its entries in index order, so each lane computes the same left fold bit for bit
// and the control flow of a team stays uniform; under unfused arithmetic the results equal the
// oracle's exactly, as the one-thread kernels' do.
#pragma once

#include <type_traits>

#include "../../include/gsb.h"
#include "gsb_families.cuh"
#include "gsb_newton.cuh"
#include "gsb_numerics.cuh"
#include "gsb_team.cuh"

namespace gsb {

// Leading dimension of a factor row in shared memory: odd, so that the lanes' rows fall in
// distinct 8-byte bank slots.
__host__ __device__ constexpr int warp_ld(int n) { return (n % 2 == 1) ? n : n + 1; }

// The cubic-affine family in row form: F_i(x) = (A x)_i + 0.1 x_i^3 - b_i with the one-thread
// family's operations (gsb_families.cuh). `p` is the system's parameter block in shared memory:
// A column-major with an odd column stride LDA (so that lanes reading along a row, as lanes
// reading down a column, fall in distinct bank slots), then b.
//
// SA (BatchParams, src/nonlinear/batched.jl:34-47): A shared by the batch, staged once per CTA
// into shared memory with the same odd column stride; a system's block is b alone.
template <int N_, bool SA = false> struct WarpCubic {
    static constexpr int N = N_, LDA = warp_ld(N_);
    static constexpr int NP = SA ? N_ : N_ * N_ + N_, SP = SA ? N_ : N_ * LDA + N_;
    static constexpr bool kSharedA = SA;
    static constexpr bool kDiagState = true;  // J = A except a diagonal held by the lanes
    const double* p;
    const double* shared;  // SA: the CTA's copy of A in shared memory; otherwise unused
    struct JState {
        double d;  // J_ii of the lane's row i
    };
    // place of parameter k (A column-major, then b) in the shared-memory block
    __host__ __device__ static constexpr int place(int k) {
        if (SA) return k;
        return k < N * N ? (k % N) + (k / N) * LDA : N * LDA + (k - N * N);
    }
    __device__ __forceinline__ double par(int k) const { return lds(smem_addr(p) + 8u * k); }
    __device__ __forceinline__ double A(int i, int k) const {
        if constexpr (SA) return lds(smem_addr(shared) + 8u * (i + k * LDA));
        else return par(i + k * LDA);
    }
    __device__ __forceinline__ double bv(int r) const { return SA ? par(r) : par(N * LDA + r); }

    // Row i (< N) of F; every lane of the team calls it (x_j arrive by broadcast).
    template <int T>
    __device__ __forceinline__ double F(const Team<T>& tm, int i, double xl) const {
        const int r = i < N ? i : N - 1;
        double t = __dmul_rn(A(r, 0), tm.bcast(xl, 0));
#pragma unroll 8
        for (int j = 1; j < N; ++j) t = __fma_rn(A(r, j), tm.bcast(xl, j), t);
        const double c = __dmul_rn(__dmul_rn(xl, xl), xl);
        return __dsub_rn(__fma_rn(0.1, c, t), bv(r));
    }
    // The diagonal of J at x (the rest of J is A).
    __device__ __forceinline__ double diag(int i, double xi) const {
        const int r = i < N ? i : N - 1;
        const double cp = __dadd_rn(__dmul_rn(__dadd_rn(xi, xi), xi), __dmul_rn(xi, xi));
        return __fma_rn(0.1, cp, A(r, r));
    }
    __device__ __forceinline__ double J(int i, int k, double diag_i) const {
        return i == k ? diag_i : A(i, k);
    }
    // the Jacobian at x: the lane's diagonal entry
    template <int T>
    __device__ __forceinline__ JState jacobian(const Team<T>& tm, double xl) const {
        return {diag(tm.lane, xl)};
    }
    // J_ik where i == k only for the lane's own row i (jmul, the factor, column folds)
    __device__ __forceinline__ double Jent(const JState& js, int i, int k) const {
        return i == k ? js.d : A(i, k);
    }
    // J_ik for a fold over all entries; dk = J_kk, broadcast by col_diag
    template <int T>
    __device__ __forceinline__ double col_diag(const Team<T>& tm, const JState& js, int k) const {
        return tm.bcast(js.d, k);
    }
    __device__ __forceinline__ double Jall(const JState&, int i, int k, double dk) const {
        return i == k ? dk : A(i, k);
    }
    template <int T>
    __device__ __forceinline__ double jvp(const Team<T>& tm, int i, double xi, double vl) const {
        const int r = i < N ? i : N - 1;
        double t = __dmul_rn(A(r, 0), tm.bcast(vl, 0));
#pragma unroll 8
        for (int j = 1; j < N; ++j) t = __fma_rn(A(r, j), tm.bcast(vl, j), t);
        const double xv = __dmul_rn(vl, xi);
        const double x2p = __dadd_rn(xv, xv);
        const double cp = __dadd_rn(__dmul_rn(x2p, xi), __dmul_rn(vl, __dmul_rn(xi, xi)));
        return __fma_rn(0.1, cp, t);
    }
};

// The Gauss–Legendre 3-stage equations of the Hénon–Heiles field in row form:
// G(Z) = Z - h (A ⊗ I) f(y + Z), Z = (Z_1, Z_2, Z_3) stacked stage increments, row r = 4 i + k.
// The operations and their order are those of the stage residual (test/helpers/
// stage_problems.jl:205-222, restated in the oracle), each product and sum rounded alone. The
// Jacobian is the forward-mode one (src/ad/forwarddiff_static.jl:50-65), written out for this
// field: row r's partials are exact dual-rule values, and a lane computes its own row into the
// held Jacobian in shared memory. `p` holds the state y (4 doubles), then the held Jacobian
// (12 x LD); `shared` (device memory) holds h and the tableau A column-major.
struct WarpIrk {
    static constexpr int N = 12, NP = 4, LD = warp_ld(12), SP = 4 + 12 * LD;
    static constexpr bool kDiagState = false;
    const double* p;
    const double* shared;
    struct JState {
        const double* J;  // the held Jacobian, row i at J + i * LD
    };
    __host__ __device__ static constexpr int place(int k) { return k; }
    __device__ __forceinline__ double y(int k) const { return lds(smem_addr(p) + 8u * k); }
    __device__ __forceinline__ double coef(int i, int j) const {
        return __dmul_rn(__ldg(shared), __ldg(shared + 1 + i + 3 * j));  // h * A_ij
    }

    // one field component k at the stage value Y
    __device__ __forceinline__ static double field(int k, double Y0, double Y1, double Y2, double Y3) {
        if (k == 0) return Y2;
        if (k == 1) return Y3;
        if (k == 2) return __dsub_rn(-Y0, __dmul_rn(2.0, __dmul_rn(Y0, Y1)));
        return __dadd_rn(__dsub_rn(-Y1, __dmul_rn(Y0, Y0)), __dmul_rn(Y1, Y1));
    }

    template <int T>
    __device__ __forceinline__ double F(const Team<T>& tm, int r, double zl) const {
        const int rr = r < N ? r : N - 1;
        const int i = rr / 4, kk = rr % 4;
        double out = zl;
        for (int j = 0; j < 3; ++j) {
            const double Y0 = __dadd_rn(y(0), tm.bcast(zl, 4 * j));
            const double Y1 = __dadd_rn(y(1), tm.bcast(zl, 4 * j + 1));
            const double Y2 = __dadd_rn(y(2), tm.bcast(zl, 4 * j + 2));
            const double Y3 = __dadd_rn(y(3), tm.bcast(zl, 4 * j + 3));
            out = __dsub_rn(out, __dmul_rn(coef(i, j), field(kk, Y0, Y1, Y2, Y3)));
        }
        return out;
    }

    // The lane's row of J into the held Jacobian: J_rc = [c == r] - a_ij df_k/dY_m for c = 4 j + m.
    template <int T>
    __device__ __forceinline__ JState jacobian(const Team<T>& tm, double zl) const {
        double* J = const_cast<double*>(p) + 4;
        const int r = tm.lane;
        const int i = (r < N ? r : N - 1) / 4, kk = (r < N ? r : N - 1) % 4;
        for (int j = 0; j < 3; ++j) {
            const double Y0 = __dadd_rn(y(0), tm.bcast(zl, 4 * j));
            const double Y1 = __dadd_rn(y(1), tm.bcast(zl, 4 * j + 1));
            const double a = coef(i, j);
            // df_kk / dY_m by the dual rules
            double fp[4] = {0.0, 0.0, 0.0, 0.0};
            if (kk == 0) fp[2] = 1.0;
            else if (kk == 1) fp[3] = 1.0;
            else if (kk == 2) {
                fp[0] = __dsub_rn(-1.0, __dmul_rn(2.0, Y1));
                fp[1] = -__dmul_rn(2.0, Y0);
            } else {
                fp[0] = -__dadd_rn(Y0, Y0);
                fp[1] = __dadd_rn(-1.0, __dadd_rn(Y1, Y1));
            }
            if (r < N) {
#pragma unroll
                for (int m = 0; m < 4; ++m) {
                    const int c = 4 * j + m;
                    const double t = __dmul_rn(a, fp[m]);
                    J[r * LD + c] = c == r ? __dsub_rn(1.0, t) : -t;
                }
            }
        }
        __syncwarp(tm.mask);
        return {J};
    }
    __device__ __forceinline__ double Jent(const JState& js, int i, int k) const {
        return lds(smem_addr(js.J) + 8u * (i * LD + k));
    }
    template <int T>
    __device__ __forceinline__ double col_diag(const Team<T>&, const JState&, int) const { return 0.0; }
    __device__ __forceinline__ double Jall(const JState& js, int i, int k, double) const {
        return Jent(js, i, k);
    }

    // Row r of J(Z) v by the one-partial dual rules.
    template <int T>
    __device__ __forceinline__ double jvp(const Team<T>& tm, int r, double zl, double vl) const {
        const int rr = r < N ? r : N - 1;
        const int i = rr / 4, kk = rr % 4;
        double out = vl;
        for (int j = 0; j < 3; ++j) {
            const double Y0 = __dadd_rn(y(0), tm.bcast(zl, 4 * j));
            const double Y1 = __dadd_rn(y(1), tm.bcast(zl, 4 * j + 1));
            const double p0 = tm.bcast(vl, 4 * j), p1 = tm.bcast(vl, 4 * j + 1);
            const double p2 = tm.bcast(vl, 4 * j + 2), p3 = tm.bcast(vl, 4 * j + 3);
            double fp;
            if (kk == 0) fp = p2;
            else if (kk == 1) fp = p3;
            else if (kk == 2)
                fp = __dsub_rn(-p0, __dmul_rn(2.0, __dadd_rn(__dmul_rn(p0, Y1), __dmul_rn(p1, Y0))));
            else
                fp = __dadd_rn(__dsub_rn(-p1, __dadd_rn(__dmul_rn(p0, Y0), __dmul_rn(p0, Y0))),
                               __dadd_rn(__dmul_rn(p1, Y1), __dmul_rn(p1, Y1)));
            out = __dsub_rn(out, __dmul_rn(coef(i, j), fp));
        }
        return out;
    }
};

// Ordered folds over a vector distributed one entry per lane (lanes >= N hold padding).
template <int N, int T, bool F> struct WarpVec {
    using A = Arith<F>;
    const Team<T>& tm;
    __device__ WarpVec(const Team<T>& t) : tm(t) {}

    __device__ __forceinline__ double norm2(double v) const {
        const double v0 = tm.bcast(v, 0);
        double s = A::mul(v0, v0);
#pragma unroll 8
        for (int i = 1; i < N; ++i) {
            const double vi = tm.bcast(v, i);
            s = A::madd(vi, vi, s);
        }
        return s;
    }
    __device__ __forceinline__ double dot(double a, double b) const {
        double s = A::mul(tm.bcast(a, 0), tm.bcast(b, 0));
#pragma unroll 8
        for (int i = 1; i < N; ++i) s = A::madd(tm.bcast(a, i), tm.bcast(b, i), s);
        return s;
    }
    __device__ __forceinline__ double maxabs(double v) const {
        double m = fabs(tm.bcast(v, 0));
#pragma unroll 8
        for (int i = 1; i < N; ++i) m = jmax(m, fabs(tm.bcast(v, i)));
        return m;
    }
    // rnorm_from: the norm from its norm2 s, with the scaled fallback.
    __device__ double rnorm_from(double v, double s) const {
        if (isfin(s) && s >= double(N) * kFloatmin) return sqrt(s);
        double m = jmax(fabs(tm.bcast(v, 0)), 0.0);
        for (int i = 1; i < N; ++i) m = jmax(m, jmax(fabs(tm.bcast(v, i)), 0.0));
        if (m == 0.0 || !isfin(m)) return m;
        const int e = jexponent(m);
        const double t = ldexp2_slow(tm.bcast(v, 0), -e);
        double acc = A::mul(t, t);
        for (int i = 1; i < N; ++i) {
            const double u = ldexp2_slow(tm.bcast(v, i), -e);
            acc = A::madd(u, u, acc);
        }
        return ldexp2_slow(sqrt(acc), e);
    }
    __device__ __forceinline__ double rnorm(double v) const { return rnorm_from(v, norm2(v)); }
    // matrix_exponent over the entries of the vector (factors.jl:833-843)
    __device__ __forceinline__ int exponent(double v, bool mine) const {
        unsigned long long b = mine ? (FBits<double>::bits(v) & ~FBits<double>::sign_mask) : 0ull;
        const double m = FBits<double>::from(tm.umax(b));
        if (!(isfin(m) && m != 0.0)) return 0;
        const int e = jexponent(m);
        return e > 1023 ? 1023 : (e < -1023 ? -1023 : e);
    }
};

// The pivot row of the warp factor in shared memory: written by the lane that holds it, read by
// every lane of the team, pairs of entries as one 16-byte (Float64) or 8-byte (Float32) access.
__device__ __forceinline__ void sts_one(unsigned a, double v) {
    asm volatile("st.shared.f64 [%0], %1;" ::"r"(a), "d"(v) : "memory");
}
__device__ __forceinline__ void sts_one(unsigned a, float v) {
    asm volatile("st.shared.f32 [%0], %1;" ::"r"(a), "f"(v) : "memory");
}
__device__ __forceinline__ void sts_pair(unsigned a, double v0, double v1) { sts2(a, v0, v1); }
__device__ __forceinline__ void sts_pair(unsigned a, float v0, float v1) {
    asm volatile("st.shared.v2.f32 [%0], {%1, %2};" ::"r"(a), "f"(v0), "f"(v1) : "memory");
}
__device__ __forceinline__ void lds_one(unsigned a, double& v) { v = lds(a); }
__device__ __forceinline__ void lds_one(unsigned a, float& v) {
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(v) : "r"(a));
}
__device__ __forceinline__ void lds_pair(unsigned a, double& v0, double& v1) { lds2(a, v0, v1); }
__device__ __forceinline__ void lds_pair(unsigned a, float& v0, float& v1) {
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(v0), "=f"(v1) : "r"(a));
}

// The pivoted LU of an N x N matrix held in registers: lane i < N keeps row i of the matrix it
// was given, and the factor's row exchanges (lu.jl:24-64: the first largest |a_ik|, i >= k, a
// NaN on the diagonal keeping k) move positions instead of rows. `pos` is the position the
// lane's row holds after the exchanges so far; position k's lane writes its row into a shared
// buffer at step k and the other lanes update their rows from it. Every entry goes through the
// operations of the elimination with physical exchanges, in the same order, so the factor's
// values, the pivot sequence and `info` are those of the reference's LU bit for bit. Row k of
// the factor is the row of lane `owner` of lane k.
//
// The pivot search is a maximum over the team of a 64-bit key, the bits of |a_ik| plus one
// (a NaN at position k counts as +Inf, one below never wins, a lane that holds no candidate has
// key 0), then the smallest position among the lanes that hold it: three warp reductions and a
// ballot in place of a butterfly of shuffles. Every member function is inlined, so that the
// rows stay in registers.
template <int N, int T, bool F, class TF> struct WarpRegLU {
    // the fused factor divides by multiplying with pivot reciprocals (see LUFactor); in the
    // back substitution that takes a division off each of the N sequential steps
    static constexpr bool kRecip = F;
    static constexpr int kBuf = ((N + 1) / 2) * 2 * (sizeof(double) / sizeof(TF));  // in TF
    using A = Arith<F>;
    TF* buf;  // two pivot-row buffers of kBuf entries, 16-byte aligned
    TF r[N];  // the lane's row: multipliers left of its pivot column, then the U part
    int pos;  // the row's position (-1 in a lane that holds no row)
    int owner;  // in lane k < N: the lane whose row is row k of the factor
    int info, e;

    __device__ __forceinline__ unsigned slot(int k) const {
        return smem_addr(buf) + (unsigned)(((k & 1) * kBuf) * sizeof(TF));
    }

    // Row k of the factor (from column k on) into buffer k & 1, by the lane that holds it, and
    // back out in every lane
    // entries K..N-1: one alone where K is odd, then pairs (even first index), then the last
    template <int K> __device__ __forceinline__ void put_row(unsigned b) const {
        constexpr int S = K + (K & 1);
        if constexpr (K & 1) sts_one(b + K * (unsigned)sizeof(TF), r[K]);
#pragma unroll
        for (int j = S; j + 1 < N; j += 2) sts_pair(b + j * (unsigned)sizeof(TF), r[j], r[j + 1]);
        if constexpr (S < N && ((N - S) & 1)) sts_one(b + (N - 1) * (unsigned)sizeof(TF), r[N - 1]);
    }
    template <int K> __device__ __forceinline__ void get_row(unsigned b, TF (&p)[N]) const {
        constexpr int S = K + (K & 1);
        if constexpr (K & 1) lds_one(b + K * (unsigned)sizeof(TF), p[K]);
#pragma unroll
        for (int j = S; j + 1 < N; j += 2) lds_pair(b + j * (unsigned)sizeof(TF), p[j], p[j + 1]);
        if constexpr (S < N && ((N - S) & 1)) lds_one(b + (N - 1) * (unsigned)sizeof(TF), p[N - 1]);
    }

    // One step of the elimination: pivot search in column K, then the update of every row
    // below position K.
    template <int K> __device__ __forceinline__ void step(const Team<T>& tm) {
        const int lane = tm.lane;
        unsigned long long key = 0ull;
        if (pos >= K) {
            const double v = double(fabs(r[K]));
            key = v != v ? (pos == K ? FBits<double>::bits(kInf) + 1ull : 0ull)
                         : FBits<double>::bits(v) + 1ull;
        }
        const unsigned kh = (unsigned)(key >> 32), kl = (unsigned)key;
        const unsigned mh = __reduce_max_sync(tm.mask, kh);
        const unsigned ml = __reduce_max_sync(tm.mask, kh == mh ? kl : 0u);
        const bool top = kh == mh && kl == ml;
        const int wi = (int)__reduce_min_sync(tm.mask, top ? (unsigned)pos : 0xffffffffu);
        const unsigned hold = __ballot_sync(tm.mask, pos == wi) & tm.mask;
        const int pl = (__ffs(hold) - 1) & (T - 1);
        if (lane == K) owner = pl;
        if (lane == pl) pos = K;
        else if (pos == K) pos = wi;
        const unsigned b = slot(K);
        if (lane == pl) put_row<K>(b);
        __syncwarp(tm.mask);
        TF p[N];
        get_row<K>(b, p);
        const TF akk = p[K];
        const bool dok = akk != TF(0);
        if (!dok && info == 0) info = K + 1;
        const TF rk = (kRecip && dok) ? TF(1) / akk : TF(0);
        if (dok && pos > K) {
            const TF l = kRecip ? r[K] * rk : r[K] / akk;
            r[K] = l;
#pragma unroll
            for (int j = K + 1; j < N; ++j) r[j] = A::msub(l, p[j], r[j]);
        }
        // the reciprocal replaces the pivot for the back substitution
        if (dok && kRecip && lane == pl) r[K] = rk;
    }
    template <int K> __device__ __forceinline__ void eliminate(const Team<T>& tm) {
        if constexpr (K < N) {
            step<K>(tm);
            eliminate<K + 1>(tm);
        }
    }

    // J into the lane's row, factor_matrix's scaling, then the elimination (lu.jl:24-64).
    template <class Fam>
    __device__ __forceinline__ void factor(const Team<T>& tm, const Fam& fam, const typename Fam::JState& js) {
        const int lane = tm.lane;
        const bool mine = lane < N;
        const int i = mine ? lane : N - 1;
        constexpr bool same = sizeof(TF) == sizeof(double);
        unsigned long long mb = 0ull;
        if constexpr (same) {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                r[k] = fam.Jent(js, i, k);
                const unsigned long long bk = FBits<double>::bits(r[k]) & ~FBits<double>::sign_mask;
                mb = bk > mb ? bk : mb;
            }
        } else {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const unsigned long long bk =
                    FBits<double>::bits(fam.Jent(js, i, k)) & ~FBits<double>::sign_mask;
                mb = bk > mb ? bk : mb;
            }
        }
        if (!mine) mb = 0ull;
        const double mm = FBits<double>::from(tm.umax(mb));
        if constexpr (same) {
            int ex = 0;
            if (isfin(mm) && mm != 0.0) {
                ex = jexponent(mm);
                ex = ex > 1023 ? 1023 : (ex < -1023 ? -1023 : ex);
            }
            e = ex < 0 ? ex : 0;
            if (e < 0) {
#pragma unroll
                for (int k = 0; k < N; ++k) r[k] = scale2_in(r[k], -e);  // -e in [1, 1023]
            }
        } else {
            e = (isfin(mm) && mm != 0.0) ? max(-1023, min(1023, jexponent(mm))) : 0;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const double v = fam.Jent(js, i, k);
                r[k] = TF(e == 0 ? v : scale2_in(v, -e));  // -e in [-1023, 1023]
            }
        }
        if (!mine) {
#pragma unroll
            for (int k = 0; k < N; ++k) r[k] = TF(0);
        }
        info = 0;
        pos = mine ? lane : -1;
        owner = lane;
        eliminate<0>(tm);
        __syncwarp(tm.mask);  // the last buffer is read before a later factor writes it
    }

    // The substitution steps, instantiated one by one (a loop over them is not always
    // unrolled, and a row indexed at run time would live in local memory).
    template <int K> __device__ __forceinline__ void forward(const Team<T>& tm, TF& x) const {
        if constexpr (K < N) {
            const TF xk = tm.bcast(x, tm.bcast(owner, K));
            if (pos > K) x = A::msub(r[K], xk, x);
            forward<K + 1>(tm, x);
        }
    }
    template <int K> __device__ __forceinline__ void backward(const Team<T>& tm, TF& x) const {
        if constexpr (K >= 0) {
            if (pos == K) x = kRecip ? x * r[K] : x / r[K];
            const TF xk = tm.bcast(x, tm.bcast(owner, K));
            if (pos >= 0 && pos < K) x = A::msub(r[K], xk, x);
            backward<K - 1>(tm, x);
        }
    }
    // lu.jl:67-92 on the distributed right-hand side: lane i enters with entry i and leaves
    // with entry i of the solution. The exchanges applied to the right-hand side move entry i
    // to position pos, where lane i already holds it; the substitutions run over positions,
    // and the unknown of column k is found in lane owner(k).
    __device__ __forceinline__ void backsolve(const Team<T>& tm, TF& x) const {
        forward<0>(tm, x);
        backward<N - 1>(tm, x);
        x = tm.bcast(x, owner);
    }

    // ldiv!!: same type (factors.jl:931-936) or mixed type (factors.jl:943-949).
    __device__ __forceinline__ double ldiv(const Team<T>& tm, const WarpVec<N, T, F>& wv, double rr) const {
        const bool mine = tm.lane < N;
        if constexpr (sizeof(TF) == sizeof(double)) {
            // rhs_exponent (factors.jl:880-885)
            const int m = wv.exponent(rr, mine);
            const int lo = e < 0 ? e : 0;
            const int aa = m > 0 ? 0 : (m < lo ? lo : m);
            const int bb = m - (1023 - headroom(N));
            const int k = aa > bb ? aa : bb;
            TF x = k == 0 ? rr : scale2_in(rr, -k);  // -k in [-6, 1023]
            backsolve(tm, x);
            const int e2 = k - e;
            return e2 == 0 ? double(x) : scale2_in(double(x), e2);  // e2 in [0, 1029]
        } else {
            const double s = wv.maxabs(rr);
            if (s == 0.0) return 0.0;
            TF x = TF(kRecip ? __dmul_rn(rr, __drcp_rn(s)) : __ddiv_rn(rr, s));
            backsolve(tm, x);
            int ex = 0;
            double frac = isfin(s) ? frexp(s, &ex) : s;
            if (!isfin(s)) ex = 0;
            double d = __dmul_rn(double(x), frac);
            const int E = ex - e;
            return (E >= -1074 && E <= 2046) ? scale2_in(d, E) : ldexp2_slow(d, E);
        }
    }
};

// The pivoted LU of an N x N matrix in shared memory, rows at a + i * LD; lane k keeps the
// pivot of column k in `piv`. The factor of the 16-lane teams (n = 12 and 16), two systems to a
// warp: measured faster there than the register factor below (n = 12: 1.65 against 1.96 ms for
// 262,144 systems), whose pivot search and row broadcasts cost about what they save.
template <int N, int T, bool F, class TF> struct WarpSmemLU {
    static constexpr int LD = warp_ld(N);
    // the fused factor divides by multiplying with pivot reciprocals (see LUFactor); in the
    // back substitution that takes a division off each of the N sequential steps
    static constexpr bool kRecip = F;
    using A = Arith<F>;
    TF* a;
    int piv;
    int info, e;

    __device__ __forceinline__ TF& at(int i, int j) const { return a[i * LD + j]; }

    // J into the factor (row `lane` from the lane's row values), factor_matrix's scaling, then
    // the elimination (lu.jl:24-64).
    template <class Fam>
    __device__ void factor(const Team<T>& tm, const Fam& fam, const typename Fam::JState& js) {
        const int lane = tm.lane;
        const bool mine = lane < N;
        constexpr bool same = sizeof(TF) == sizeof(double);
        unsigned long long mb = 0ull;
        if (mine)
            for (int k = 0; k < N; ++k) {
                const unsigned long long b =
                    FBits<double>::bits(fam.Jent(js, lane, k)) & ~FBits<double>::sign_mask;
                mb = b > mb ? b : mb;
            }
        const double mm = FBits<double>::from(tm.umax(mb));
        if constexpr (same) {
            int ex = 0;
            if (isfin(mm) && mm != 0.0) {
                ex = jexponent(mm);
                ex = ex > 1023 ? 1023 : (ex < -1023 ? -1023 : ex);
            }
            e = ex < 0 ? ex : 0;
            if (mine)
                for (int k = 0; k < N; ++k) {
                    const double v = fam.Jent(js, lane, k);
                    at(lane, k) = e < 0 ? scale2_in(v, -e) : v;  // -e in [1, 1023]
                }
        } else {
            e = (isfin(mm) && mm != 0.0) ? max(-1023, min(1023, jexponent(mm))) : 0;
            if (mine)
                for (int k = 0; k < N; ++k) {
                    const double v = fam.Jent(js, lane, k);
                    at(lane, k) = TF(e == 0 ? v : scale2_in(v, -e));  // -e in [-1023, 1023]
                }
        }
        __syncwarp(tm.mask);
        info = 0;
        piv = lane;
        // The first largest |a_ik|, i >= k (a NaN on the diagonal keeps k; a NaN below it never
        // wins), as a (value, index) maximum with the smaller index on ties.
        auto pivot = [&](int k) {
            double w = -2.0;
            if (lane == k) {
                const double v = double(fabs(at(k, k)));
                w = v != v ? kInf : v;
            } else if (lane > k && lane < N) {
                const double v = double(fabs(at(lane, k)));
                w = v != v ? -1.0 : v;
            }
            int wi = lane;
#pragma unroll
            for (int off = T / 2; off > 0; off >>= 1) {
                const double ow = __shfl_xor_sync(tm.mask, w, off, T);
                const int oi = __shfl_xor_sync(tm.mask, wi, off, T);
                if (ow > w || (ow == w && oi < wi)) {
                    w = ow;
                    wi = oi;
                }
            }
            if (lane == k) piv = wi;
            if (wi != k) {  // rows k and wi exchanged whole, lane c taking column c
                if (mine) {
                    const TF t = at(k, lane);
                    at(k, lane) = at(wi, lane);
                    at(wi, lane) = t;
                }
                __syncwarp(tm.mask);
            }
        };
        // Two steps of the elimination per pass (the same operations on every entry, in the same
        // order, as one step at a time): step k's multipliers and its update of column k + 1,
        // which step k + 1's pivot search reads; step k + 1's pivot row brought up to date one
        // entry per lane; then both updates of every other entry in one pass, one read and one
        // write of the lane's row per entry instead of two.
        for (int k = 0; k < N; k += 2) {
            pivot(k);
            const TF akk = at(k, k);
            const bool dok = akk != TF(0);
            if (!dok && info == 0) info = k + 1;
            const TF rk = (kRecip && dok) ? TF(1) / akk : TF(0);
            const int k1 = k + 1;
            if (k1 == N) {
                if (dok && kRecip && lane == k) at(k, k) = rk;
                __syncwarp(tm.mask);
                break;
            }
            if (dok && lane > k && lane < N) {
                const TF l = kRecip ? at(lane, k) * rk : at(lane, k) / akk;
                at(lane, k) = l;
                at(lane, k1) = A::msub(l, at(k, k1), at(lane, k1));
            }
            // the reciprocal replaces the pivot for the back substitution
            if (dok && kRecip && lane == k) at(k, k) = rk;
            __syncwarp(tm.mask);
            pivot(k1);
            if (dok && lane > k1 && lane < N)
                at(k1, lane) = A::msub(at(k1, k), at(k, lane), at(k1, lane));
            __syncwarp(tm.mask);
            const TF ak1 = at(k1, k1);
            const bool dok1 = ak1 != TF(0);
            if (!dok1 && info == 0) info = k1 + 1;
            const TF r1 = (kRecip && dok1) ? TF(1) / ak1 : TF(0);
            if (lane > k1 && lane < N) {
                const TF l0 = dok ? at(lane, k) : TF(0);  // this row's step-k multiplier
                TF l1 = TF(0);
                if (dok1) {
                    l1 = kRecip ? at(lane, k1) * r1 : at(lane, k1) / ak1;
                    at(lane, k1) = l1;
                }
                for (int j = k1 + 1; j < N; ++j) {
                    TF v = at(lane, j);
                    if (dok) v = A::msub(l0, at(k, j), v);
                    if (dok1) v = A::msub(l1, at(k1, j), v);
                    at(lane, j) = v;
                }
            }
            if (dok1 && kRecip && lane == k1) at(k1, k1) = r1;
            __syncwarp(tm.mask);
        }
    }

    // lu.jl:67-92 on the distributed right-hand side x.
    __device__ void backsolve(const Team<T>& tm, TF& x) const {
        const int lane = tm.lane;
        for (int k = 0; k < N; ++k) {
            const int p = tm.bcast(piv, k);
            if (p != k) {
                const TF xk = tm.bcast(x, k);
                const TF xp = tm.bcast(x, p);
                if (lane == k) x = xp;
                else if (lane == p) x = xk;
            }
        }
        for (int k = 0; k < N; ++k) {
            const TF xk = tm.bcast(x, k);
            if (lane > k && lane < N) x = A::msub(at(lane, k), xk, x);
        }
        for (int k = N - 1; k >= 0; --k) {
            if (lane == k) x = kRecip ? x * at(k, k) : x / at(k, k);
            const TF xk = tm.bcast(x, k);
            if (lane < k) x = A::msub(at(lane, k), xk, x);
        }
    }

    // ldiv!!: same type (factors.jl:931-936) or mixed type (factors.jl:943-949).
    __device__ double ldiv(const Team<T>& tm, const WarpVec<N, T, F>& wv, double r) const {
        const bool mine = tm.lane < N;
        if constexpr (sizeof(TF) == sizeof(double)) {
            // rhs_exponent (factors.jl:880-885)
            const int m = wv.exponent(r, mine);
            const int lo = e < 0 ? e : 0;
            const int aa = m > 0 ? 0 : (m < lo ? lo : m);
            const int bb = m - (1023 - headroom(N));
            const int k = aa > bb ? aa : bb;
            TF x = k == 0 ? r : scale2_in(r, -k);  // -k in [-6, 1023]
            backsolve(tm, x);
            const int e2 = k - e;
            return e2 == 0 ? double(x) : scale2_in(double(x), e2);  // e2 in [0, 1029]
        } else {
            const double s = wv.maxabs(r);
            if (s == 0.0) return 0.0;
            TF x = TF(kRecip ? __dmul_rn(r, __drcp_rn(s)) : __ddiv_rn(r, s));
            backsolve(tm, x);
            int ex = 0;
            double frac = isfin(s) ? frexp(s, &ex) : s;
            if (!isfin(s)) ex = 0;
            double d = __dmul_rn(double(x), frac);
            const int E = ex - e;
            return (E >= -1074 && E <= 2046) ? scale2_in(d, E) : ldexp2_slow(d, E);
        }
    }
};

// The factor of a team: rows in registers for the 32-lane teams, in shared memory for 16.
template <int N, int T, bool F, class TF>
using WarpLU = typename std::conditional<T == 32, WarpRegLU<N, T, F, TF>, WarpSmemLU<N, T, F, TF>>::type;

// Shared memory of a system's factor, in doubles.
template <int N, int T> __host__ __device__ constexpr int warp_lu_doubles() {
    return T == 32 ? 2 * (((N + 1) / 2) * 2) : N * warp_ld(N);
}

template <class Fam, int T, bool F, bool Mixed, bool PlainRef> struct WarpSolver {
    static constexpr int N = Fam::N, LD = warp_ld(N);
    using A = Arith<F>;
    using JS = typename Fam::JState;
    const Fam& fam;
    const GsbMethod& m;
    const GsbOptions& o;
    const Team<T>& tm;
    double* lu;  // the factor's shared memory (warp_lu_doubles<N, T>() doubles)
    WarpVec<N, T, F> wv;

    __device__ WarpSolver(const Fam& f, const GsbMethod& mm, const GsbOptions& oo,
                          const Team<T>& t, double* l)
        : fam(f), m(mm), o(oo), tm(t), lu(l), wv(t) {}

    __device__ __forceinline__ bool has_merit() const { return m.globalization == GSB_BACKTRACKING; }
    __device__ __forceinline__ double Fr(double xl) const { return fam.template F<T>(tm, tm.lane, xl); }

    // J v with the held Jacobian, row `lane`, as a left fold over the columns.
    __device__ __forceinline__ double jmul(const JS& js, double vl) const {
        const int i = tm.lane < N ? tm.lane : N - 1;
        double s = A::mul(fam.Jent(js, i, 0), tm.bcast(vl, 0));
        for (int k = 1; k < N; ++k) s = A::madd(fam.Jent(js, i, k), tm.bcast(vl, k), s);
        return s;
    }

    // grad_ratio_and_norm, src/nonlinear/newton.jl:1287-1298.
    __device__ void grad_ratio_and_norm(const JS& js, double Fl, double fnorm, double& gr,
                                        double& jnorm) const {
        double s = 0.0;
        if constexpr (F) {
            // Under the fused arithmetic (whose FMAs already round this sum apart from the
            // reference's) each lane folds its own row and the lanes combine in a butterfly,
            // which leaves the same bits in every lane: N + log2(T) dependent steps instead of
            // N^2. ‖J‖_F feeds only the reported gradient ratio.
            if (tm.lane < N) {
                const int i = tm.lane;
                const double v0 = fam.Jent(js, i, 0);
                s = A::mul(v0, v0);
                for (int k = 1; k < N; ++k) {
                    const double v = fam.Jent(js, i, k);
                    s = A::madd(v, v, s);
                }
            }
            s = tm.sum(s);
        } else {
            // ‖J‖_F as the column-major left fold: every lane folds all entries
            for (int k = 0; k < N; ++k) {
                const double dk = fam.template col_diag<T>(tm, js, k);
                for (int i = 0; i < N; ++i) {
                    const double v = fam.Jall(js, i, k, dk);
                    s = (i == 0 && k == 0) ? A::mul(v, v) : A::madd(v, v, s);
                }
            }
        }
        double mx = 0.0;
        const bool direct = isfin(s) && s >= double(N * N) * kFloatmin;
        if (!direct) {
            // the scaled fallback of rnorm over the N*N entries
            for (int k = 0; k < N; ++k) {
                const double dk = fam.template col_diag<T>(tm, js, k);
                for (int i = 0; i < N; ++i) mx = jmax(mx, jmax(fabs(fam.Jall(js, i, k, dk)), 0.0));
            }
        }
        if (direct) {
            jnorm = sqrt(s);
        } else if (mx == 0.0 || !isfin(mx)) {
            jnorm = mx;
        } else {
            const int e = jexponent(mx);
            double acc = 0.0;
            for (int k = 0; k < N; ++k) {
                const double dk = fam.template col_diag<T>(tm, js, k);
                for (int i = 0; i < N; ++i) {
                    const double u = scale2_in(fam.Jall(js, i, k, dk), -e);
                    acc = (i == 0 && k == 0) ? A::mul(u, u) : A::madd(u, u, acc);
                }
            }
            jnorm = scale2_in(sqrt(acc), e);
        }
        if (jnorm == 0.0 || fnorm == 0.0) {
            gr = 0.0;
            return;
        }
        // g_j = sum_i J_ij F_i: lane j folds column j (its own diagonal entry where i == j)
        const int j = tm.lane < N ? tm.lane : N - 1;
        double g = A::mul(fam.Jent(js, 0, j), tm.bcast(Fl, 0));
        for (int i = 1; i < N; ++i) g = A::madd(fam.Jent(js, i, j), tm.bcast(Fl, i), g);
        const double gnorm = wv.rnorm(g);
        if (isfin(gnorm) || !(isfin(jnorm) && isfin(fnorm))) {
            gr = __ddiv_rn(__ddiv_rn(gnorm, jnorm), fnorm);
            return;
        }
        const int e = jexponent(fnorm);
        const double sc = ldexp(1.0, -e);
        g = A::mul(fam.Jent(js, 0, j), __dmul_rn(tm.bcast(Fl, 0), sc));
        for (int i = 1; i < N; ++i) g = A::madd(fam.Jent(js, i, j), __dmul_rn(tm.bcast(Fl, i), sc), g);
        gr = __ddiv_rn(__ddiv_rn(wv.rnorm(g), jnorm), ldexp(fnorm, -e));
    }

    __device__ __forceinline__ double residual_norm(const DevState& st, double Fl) const {
        if (has_merit()) {
            if (isfin(st.merit) && st.merit >= double(N) * kFloatmin) return sqrt(st.merit);
            return wv.rnorm(Fl);
        }
        return isnan(st.fnorm) ? wv.rnorm(Fl) : st.fnorm;
    }

    // The merit of x + a d: the lane's trial entries and norm2 of the trial residual.
    __device__ __forceinline__ double trial(double xl, double dl, double a, double& xt,
                                            double& Ft) const {
        xt = A::madd(a, dl, xl);
        Ft = Fr(xt);
        return wv.norm2(Ft);
    }

    __device__ __forceinline__ double slope0(double xl, double dl) const {
        const double x0 = A::madd(0.0, dl, xl);
        const double F0 = Fr(x0);
        const double Jv = fam.template jvp<T>(tm, tm.lane, x0, dl);
        return 2.0 * wv.dot(F0, Jv);
    }

    __device__ void globalize(double& xl, double& Fl, double dl, bool exact, double& merit,
                              StepInfo& info) const {
        if (m.globalization == GSB_STATIC) {
            const double s = m.static_alpha;
            const double dn = wv.rnorm(dl);
            const double stepnorm = __dmul_rn(fabs(s), dn);
            if (!isfin(stepnorm)) {
                info = {NONFINITE, wv.rnorm(Fl), stepnorm, 0, false, false, false};
                return;
            }
            double xp, Fp;
            const double fn = wv.rnorm_from(Fp, trial(xl, dl, s, xp, Fp));
            if (!isfin(fn)) {
                info = {NONFINITE, wv.rnorm(Fl), stepnorm, 0, false, false, false};
                return;
            }
            xl = xp;
            Fl = Fp;
            info = {SUCCESS, fn, stepnorm, 0, false, false, false};
            return;
        }
        const double phi0 = merit;
        const double dn = wv.rnorm(dl);
        if (!isfin(dn)) {
            info = {NONFINITE, wv.rnorm(Fl), dn, 0, false, false, false};
            return;
        }
        double alpha = 1.0;
        const double d0 = exact ? -2.0 * phi0 : slope0(xl, dl);
        int code;
        double aa = alpha, pa = kNaN;
        double xt = xl, Ft = Fl;
        if (!(isfin(phi0) && isfin(d0) && d0 < 0.0)) {
            code = (isfin(phi0) && isfin(d0)) ? (d0 > 0.0 ? LINESEARCH_FAILED : STALLED) : NONFINITE;
        } else {
            const double tau = jmax(__dmul_rn(4.0 * kEps, fabs(phi0)), 4.0 * 4.9406564584124654e-324);
            const double amin = jmax(__ddiv_rn(tau, fabs(d0)), kFloatmin);
            alpha = jmin(jmax(alpha, amin), kInf);
            double ap = kNaN, pp = kNaN;
            int frozen = 0, trips = 0;
            code = LINESEARCH_FAILED;
            bool done = false;
            const double c1 = m.bt_c1, p = m.bt_p;
            while (!done && trips < m.bt_maxiter) {
                ++trips;
                aa = alpha;
                pa = trial(xl, dl, alpha, xt, Ft);
                frozen = (pa == phi0 && alpha <= kSqrtEps) ? frozen + 1 : 0;
                const double demand = __dmul_rn(__dmul_rn(c1, alpha), d0);
                if (__dsub_rn(pa, phi0) <= jmin(0.0, __dadd_rn(demand, tau))) {
                    if (isfin(pa) && __dsub_rn(pa, phi0) < -tau) code = SUCCESS;
                    else code = fabs(__dsub_rn(pa, phi0)) <= tau ? STALLED : LINESEARCH_FAILED;
                    done = true;
                } else if (frozen >= 2) {
                    code = STALLED;
                    done = true;
                } else if (alpha <= amin) {
                    code = fabs(__dsub_rn(pa, phi0)) <= tau ? STALLED : LINESEARCH_FAILED;
                    done = true;
                } else {
                    double an;
                    if (isfin(pa)) {
                        an = kNaN;
                        const double s = fabs(d0);
                        const double r1 = __dadd_rn(__ddiv_rn(__dsub_rn(pa, phi0), s), alpha);
                        if (!(ap > 0.0)) {
                            if (r1 > 0.0) an = __ddiv_rn(__dmul_rn(alpha, alpha), __dmul_rn(2.0, r1));
                        } else if (isfin(pp) && alpha != ap) {
                            const double q1 = __ddiv_rn(r1, __dmul_rn(alpha, alpha));
                            const double q2 = __ddiv_rn(__dadd_rn(__ddiv_rn(__dsub_rn(pp, phi0), s), ap),
                                                        __dmul_rn(ap, ap));
                            const double da = __dsub_rn(alpha, ap);
                            const double Aq = __ddiv_rn(__dsub_rn(q1, q2), da);
                            const double Bq =
                                __ddiv_rn(__dsub_rn(__dmul_rn(alpha, q2), __dmul_rn(ap, q1)), da);
                            const double disc = __dadd_rn(__dmul_rn(Bq, Bq), __dmul_rn(3.0, Aq));
                            if (disc >= 0.0)
                                an = Bq > 0.0 ? __ddiv_rn(1.0, __dadd_rn(Bq, sqrt(disc)))
                                              : __ddiv_rn(__dadd_rn(-Bq, sqrt(disc)), __dmul_rn(3.0, Aq));
                        }
                        if (!(isfin(an) && an > 0.0)) an = __dmul_rn(p, alpha);
                        an = jmin(jmax(an, __dmul_rn(0.1, alpha)), __dmul_rn(p, alpha));
                    } else {
                        an = jmin(__dmul_rn(0.1, alpha), __dmul_rn(sqrt(alpha), sqrt(amin)));
                    }
                    ap = alpha;
                    pp = pa;
                    alpha = jmax(an, amin);
                }
            }
        }
        if (code == SUCCESS) {
            xl = xt;
            Fl = Ft;
            info = {SUCCESS, sqrt(pa), __dmul_rn(aa, dn), 0, false, false, aa < 1.0};
            merit = pa;
        } else if (code == LINESEARCH_FAILED) {
            if (isfin(pa) && pa < phi0) {
                xl = xt;
                Fl = Ft;
                info = {LINESEARCH_FAILED, sqrt(pa), __dmul_rn(aa, dn), 1, false, false, aa < 1.0};
                merit = pa;
            } else {
                info = {LINESEARCH_FAILED, wv.rnorm(Fl), 0.0, 1, false, false, false};
            }
        } else if (code == STALLED) {
            info = {STALLED, wv.rnorm(Fl), 0.0, 0, false, false, false};
        } else {
            info = {NONFINITE, wv.rnorm(Fl), 0.0, 0, false, false, false};
        }
    }

    // refine_passes!! with the held Jacobian (refinement.jl:211-244); returns `failed`.
    template <class Fac>
    __device__ bool refine(double& dl, const Fac& fac, const JS& js, double Fl) const {
        const double fnorm = wv.rnorm(Fl);
        if (fnorm == 0.0) return false;
        if (!isfin(fnorm)) return true;
        const double thr = __dmul_rn(jmax(m.refine_eta, kSqrtEps), fnorm);
        double r = jmul(js, dl);
        r = __dadd_rn(-Fl, -r);
        double rprev = wv.rnorm(r);
        if (!isfin(rprev)) return true;
        if (rprev <= thr) return false;
        for (int it = 1; it <= m.refine_maxiter; ++it) {
            double dc = fac.ldiv(tm, wv, r);
            dc = __dadd_rn(dl, dc);
            r = jmul(js, dc);
            r = __dadd_rn(-Fl, -r);
            const double rc = wv.rnorm(r);
            if (!(rc < rprev)) return true;
            dl = dc;
            rprev = rc;
            if (rc <= thr) return false;
        }
        return true;
    }

    __device__ void step_plain(DevState& st, double& xl, double& Fl, StepInfo& info) const {
        const double fnorm = residual_norm(st, Fl);
        const JS js = fam.template jacobian<T>(tm, xl);
        double gr, jn;
        grad_ratio_and_norm(js, Fl, fnorm, gr, jn);
        double merit = st.merit;
        WarpLU<N, T, F, double> fac{lu};
        fac.factor(tm, fam, js);
        if (fac.info > 0) {
            info = {SINGULAR, wv.rnorm(Fl), 0.0, 0, false, false, false};
        } else {
            double dl = -fac.ldiv(tm, wv, Fl);
            if constexpr (PlainRef) refine(dl, fac, js, Fl);
            globalize(xl, Fl, dl, !PlainRef, merit, info);
        }
        st.gradratio = gr;
        st.jnorm = jn;
        st.merit = merit;
        st.fnorm = info.fnorm;
    }

    __device__ void step_mixed(DevState& st, double& xl, double& Fl, StepInfo& info) const {
        const double fnorm_old = residual_norm(st, Fl);
        const bool was_promoted = st.promoted;
        const JS js = fam.template jacobian<T>(tm, xl);
        double gr, jn;
        grad_ratio_and_norm(js, Fl, fnorm_old, gr, jn);
        st.gradratio = gr;
        st.jnorm = jn;
        const bool ref = m.refinement == GSB_REFINEMENT;
        double dl = 0.0;
        bool ok = true;
        int failures = 0;
        double lin_rel = 0.0;
        bool md_promoted = was_promoted;
        bool fallback = was_promoted;
        if (!was_promoted) {
            WarpLU<N, T, F, float> fac{reinterpret_cast<float*>(lu)};
            fac.factor(tm, fam, js);
            bool ref_failed;
            if (fac.info > 0) {
                ref_failed = true;
            } else {
                dl = -fac.ldiv(tm, wv, Fl);
                ref_failed = ref ? refine(dl, fac, js, Fl) : false;
            }
            if (ref_failed || fac.info > 0) {
                failures += 1;
                md_promoted = true;
                fallback = true;
            } else if (fnorm_old == 0.0 || !isfin(fnorm_old)) {
                lin_rel = 0.0;
            } else {
                const double lin = __dadd_rn(Fl, jmul(js, dl));
                lin_rel = __ddiv_rn(wv.rnorm(lin), fnorm_old);
            }
        }
        if (fallback) {
            WarpLU<N, T, F, double> ft{lu};
            ft.factor(tm, fam, js);
            if (ft.info > 0) {
                ok = false;
            } else {
                dl = -ft.ldiv(tm, wv, Fl);
                if (was_promoted && ref) refine(dl, ft, js, Fl);
            }
        }
        if (!ok) {
            st.promoted = md_promoted;
            info = {SINGULAR, wv.rnorm(Fl), 0.0, failures, md_promoted, false, false};
            return;
        }
        const bool promoted_step = md_promoted && !was_promoted;
        const bool exact_step = md_promoted;
        double merit = st.merit;
        globalize(xl, Fl, dl, exact_step, merit, info);
        info.failures += failures;
        if (promoted_step) {
            info.promoted = true;
            st.promoted = true;
            st.slow_steps = 0;
        } else if (!was_promoted) {
            const double eta_lin = 1e-4;
            if (info.fnorm > __dmul_rn(0.5, fnorm_old) && lin_rel > eta_lin) {
                const int slow = st.slow_steps + 1;
                if (slow >= 2) {
                    st.promoted = true;
                    st.slow_steps = 0;
                    info.failures += 1;
                    info.promoted = true;
                } else {
                    st.promoted = false;
                    st.slow_steps = slow;
                }
            } else {
                st.promoted = false;
                st.slow_steps = 0;
            }
        }
        st.merit = merit;
        st.fnorm = info.fnorm;
    }

    __device__ __forceinline__ bool residual_converged(const DevStatus& s, double ft,
                                                       double ft0) const {
        if (!(s.iterations >= o.min_iterations)) return false;
        return ft <= jmax(o.f_abstol, __dmul_rn(o.f_reltol, ft0));
    }

    // solve!!, src/nonlinear/solver.jl:277-378; the lane's entry of x in `xl`.
    __device__ DevStatus solve(double& xl, double& gr_out) const {
        double Fl = Fr(xl);
        const double n2 = wv.norm2(Fl);
        const double fnorm0 = wv.rnorm_from(Fl, n2);
        DevState st;
        st.merit = has_merit() ? n2 : kNaN;
        st.fnorm = fnorm0;
        st.gradratio = kNaN;
        st.jnorm = 0.0;
        st.promoted = false;
        st.slow_steps = 0;
        DevStatus s;
        s.code = SUCCESS;
        s.iterations = 0;
        s.fnorm = fnorm0;
        s.stepnorm = 0.0;
        s.step_failures = 0;
        s.promoted = false;
        s.stationary = false;
        s.rate = kNaN;
        s.contracted = false;
        gr_out = kNaN;
        if (!isfin(fnorm0)) {
            s.code = NONFINITE;
            return s;
        }
        const double ftest0 = o.norm == 1 ? wv.maxabs(Fl) : fnorm0;
        if (residual_converged(s, ftest0, ftest0)) return s;
        if (o.max_iterations == 0) {
            s.code = MAXITERS;
            return s;
        }
        int stalls = 0;
        while (true) {
            const double rate_k = s.rate;
            StepInfo info;
            if (Mixed) step_mixed(st, xl, Fl, info);
            else step_plain(st, xl, Fl, info);
            record(s, info);
            gr_out = st.gradratio;
            if (info.code == SINGULAR || info.code == NONFINITE || info.code == MAXITERS) return s;
            if (info.code == LINESEARCH_FAILED && info.stepnorm == 0.0) return s;
            const double ft = o.norm == 1 ? wv.maxabs(Fl) : s.fnorm;
            if (residual_converged(s, ft, ftest0)) {
                s.code = SUCCESS;
                s.stationary = false;
                s.contracted = false;
                return s;
            }
            const bool steptested = !(info.code == STALLED || info.limited);
            const double xnorm = steptested ? wv.rnorm(xl) : kNaN;
            bool contracted = false;
            if (!info.shortened && o.rate_test && s.iterations >= o.min_iterations) {
                const double th = jmax(s.rate, rate_k);
                if (s.stepnorm > 0.0 && th < 1.0)
                    contracted = __dmul_rn(__ddiv_rn(th, __dsub_rn(1.0, th)), s.stepnorm) <=
                                 __dmul_rn(o.kappa, jmax(o.x_abstol, __dmul_rn(o.x_reltol, xnorm)));
            }
            bool stepc = false;
            if (steptested && s.iterations >= o.min_iterations) {
                stepc = s.iterations > 0 && s.stepnorm > 0.0 &&
                        s.stepnorm <= jmax(o.x_abstol, __dmul_rn(o.x_reltol, xnorm));
                stepc = stepc || (info.code == SUCCESS && info.stepnorm == 0.0);
                stepc = stepc || (o.roundoff && s.rate >= 1.0 && rate_k < 1.0);
            }
            if (contracted || stepc) {
                s.code = contracted ? SUCCESS : STALLED;
                s.stationary = false;
                s.contracted = contracted;
                return s;
            }
            if (info.code == STALLED) {
                stalls += 1;
                if (stalls >= o.max_stalls) {
                    s.code = STALLED;
                    s.stationary = false;
                    s.contracted = false;
                    return s;
                }
            } else {
                stalls = 0;
            }
            if (s.iterations >= o.max_iterations) {
                s.code = MAXITERS;
                s.stationary = false;
                s.contracted = false;
                return s;
            }
        }
    }
};

}  // namespace gsb
