// The team form of the per-system Newton solve: T lanes of a warp (T = 2, 4, 8, 16 or 32, an
// aligned group) share one system. Row i of the Jacobian, of its factor and of the residual
// belongs to lane i % T (local slot i / T); the iterate x and the direction d are held by every
// lane. The pivot search, the pivot row and the solve's unknowns move between lanes by
// shuffles restricted to the team's mask, so teams of one warp may diverge (finish at different
// iterations) independently.
//
// Every lane of a team runs the same control flow: the scalars that steer it (norms, merits,
// the pivot index) come from butterfly reductions whose sums and maxima are commutative, so each
// lane holds the same bits. The arithmetic is fused (FMA); the reductions combine partial sums
// across lanes, so a team solve meets the batch contract within its tolerance rather than bit for
// bit (the one-thread solve in gsb_newton.cuh provides the unfused, bit-reproducible form).
//
// The solve follows GeometricSolvers.jl's R1 loop `solve!!` (src/nonlinear/solver.jl:277-378),
// the Newton step (src/nonlinear/newton.jl:1679-1720, mixed :1604-1666), the static LU
// (src/linear/static/lu.jl:24-92) with factor_matrix and ldiv!! scaling
// (src/linear/factors.jl:802-949), Backtracking and Static (src/globalization/linefunction.jl:
// 114-199, backtracking.jl:62-132) and refinement (src/nonlinear/refinement.jl:211-244).
#pragma once

#include "../../include/gsb.h"
#include "gsb_families.cuh"
#include "gsb_newton.cuh"
#include "gsb_numerics.cuh"

namespace gsb {

// a ? x : y with a runtime condition, as one PTX select, so that a choice among register-array
// entries by a runtime index cannot become an indexed (local-memory) access.
__device__ __forceinline__ double sel(bool c, double x, double y) {
    double r;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.s32 q, %1, 0;\n\tselp.f64 %0, %2, %3, q;\n\t}"
        : "=d"(r) : "r"((int)c), "d"(x), "d"(y));
    return r;
}
__device__ __forceinline__ float sel(bool c, float x, float y) {
    float r;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.s32 q, %1, 0;\n\tselp.f32 %0, %2, %3, q;\n\t}"
        : "=f"(r) : "r"((int)c), "f"(x), "f"(y));
    return r;
}

// Entry s * T + lane of a vector that every lane of a team holds: the lane's own entry of slot s.
template <int N, int T> __device__ __forceinline__ double own(const double (&x)[N], int s, int lane) {
    double v = x[s * T];
#pragma unroll
    for (int l = 1; l < T; ++l) v = sel(lane == l, x[s * T + l], v);
    return v;
}

template <int T> struct Team {
    unsigned mask;
    int lane;  // 0..T-1 within the team

    __device__ __forceinline__ Team() {
        const int l = threadIdx.x & 31;
        lane = l & (T - 1);
        mask = T == 32 ? 0xffffffffu : (((1u << T) - 1u) << (l & ~(T - 1)));
    }
    __device__ __forceinline__ double bcast(double v, int src) const {
        return __shfl_sync(mask, v, src, T);
    }
    __device__ __forceinline__ float bcast(float v, int src) const {
        return __shfl_sync(mask, v, src, T);
    }
    __device__ __forceinline__ int bcast(int v, int src) const {
        return __shfl_sync(mask, v, src, T);
    }
    __device__ __forceinline__ double sum(double v) const {
#pragma unroll
        for (int off = T / 2; off > 0; off >>= 1) v += __shfl_xor_sync(mask, v, off, T);
        return v;
    }
    __device__ __forceinline__ double max(double v) const {
#pragma unroll
        for (int off = T / 2; off > 0; off >>= 1) v = jmax(v, __shfl_xor_sync(mask, v, off, T));
        return v;
    }
    __device__ __forceinline__ unsigned long long umax(unsigned long long v) const {
#pragma unroll
        for (int off = T / 2; off > 0; off >>= 1) {
            unsigned long long o = __shfl_xor_sync(mask, v, off, T);
            v = o > v ? o : v;
        }
        return v;
    }
    __device__ __forceinline__ bool any(bool b) const { return (__ballot_sync(mask, b) & mask) != 0u; }
};

// The pivoted LU of a distributed matrix: lane holds rows lane, lane + T, ... (R = N / T slots).
template <int N, int T, class TF> struct TeamLU {
    static constexpr int R = N / T;
    TF a[R][N];
    int ipiv[N];  // the same in every lane
    int info, e;

    // factor_matrix's scaling and the partial-pivot LU (src/linear/static/lu.jl:24-64): the
    // first largest |a_ik|, info = the first zero pivot, no early exit.
    // jrow(s, out) gives the lane's row of slot s.
    template <class Row>
    __device__ __forceinline__ void factor(const Team<T>& tm, Row jrow) {
        double jm[R][N];
#pragma unroll
        for (int s = 0; s < R; ++s) jrow(s, jm[s]);
        unsigned long long mb = 0;
#pragma unroll
        for (int s = 0; s < R; ++s)
#pragma unroll
            for (int j = 0; j < N; ++j) {
                unsigned long long b = FBits<double>::bits(jm[s][j]) & ~FBits<double>::sign_mask;
                mb = b > mb ? b : mb;
            }
        mb = tm.umax(mb);
        double mm = FBits<double>::from(mb);
        e = (isfin(mm) && mm != 0.0) ? ::max(-1023, ::min(1023, jexponent(mm))) : 0;
        constexpr bool same = sizeof(TF) == sizeof(double);
        if (same && !(e < 0)) e = 0;
#pragma unroll
        for (int s = 0; s < R; ++s)
#pragma unroll
            for (int j = 0; j < N; ++j) a[s][j] = TF(e == 0 ? jm[s][j] : scale2_in(jm[s][j], -e));
        info = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int ks = k / T, kl = k % T;
            // pivot search: key |a_ik| (NaN never chosen, except a NaN a_kk, which keeps k)
            double bestv = -1.0;
            int besti = N;
#pragma unroll
            for (int s = 0; s < R; ++s) {
                const int i = s * T + tm.lane;
                double v = fabs(double(a[s][k]));
                if (i == k) v = isnan(v) ? kInf : v;
                else if (isnan(v)) v = -1.0;
                if (i >= k && (v > bestv || (v == bestv && i < besti))) {
                    bestv = v;
                    besti = i;
                }
            }
#pragma unroll
            for (int off = T / 2; off > 0; off >>= 1) {
                double ov = __shfl_xor_sync(tm.mask, bestv, off, T);
                int oi = __shfl_xor_sync(tm.mask, besti, off, T);
                if (ov > bestv || (ov == bestv && oi < besti)) {
                    bestv = ov;
                    besti = oi;
                }
            }
            const int p = besti;
            ipiv[k] = p;
            if (p != k) {
                // exchange rows k and p: row k is slot ks of lane kl, row p slot p / T of lane p % T
                const int pl = p % T, ps = p / T;
#pragma unroll
                for (int j = 0; j < N; ++j) {
                    TF kv = tm.bcast(a[ks][j], kl);
                    TF mine = a[0][j];
#pragma unroll
                    for (int s = 1; s < R; ++s) mine = sel(s == ps, a[s][j], mine);
                    TF pv = tm.bcast(mine, pl);
                    a[ks][j] = sel(tm.lane == kl, pv, a[ks][j]);
#pragma unroll
                    for (int s = 0; s < R; ++s) a[s][j] = sel(tm.lane == pl && s == ps, kv, a[s][j]);
                }
            }
            const TF akk = tm.bcast(a[ks][k], kl);
            if (akk == TF(0)) {
                if (info == 0) info = k + 1;
            } else {
                TF piv[N];
#pragma unroll
                for (int j = k + 1; j < N; ++j) piv[j] = tm.bcast(a[ks][j], kl);
#pragma unroll
                for (int s = 0; s < R; ++s) {
                    const int i = s * T + tm.lane;
                    if (i > k) {
                        const TF l = a[s][k] / akk;
                        a[s][k] = l;
#pragma unroll
                        for (int j = k + 1; j < N; ++j) a[s][j] = Arith<true>::msub(l, piv[j], a[s][j]);
                    }
                }
            }
        }
    }

    // The distributed back-solve (lu.jl:67-92): r holds the lane's rows of the right-hand side;
    // the solution comes back in every lane (each unknown is broadcast as it is found).
    __device__ __forceinline__ void backsolve(const Team<T>& tm, TF (&r)[R], TF (&x)[N]) const {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const int p = ipiv[k];
            if (p != k) {
                const int kl = k % T, ks = k / T, pl = p % T, ps = p / T;
                TF kv = tm.bcast(r[ks], kl);
                TF mine = r[0];
#pragma unroll
                for (int s = 1; s < R; ++s) mine = sel(s == ps, r[s], mine);
                TF pv = tm.bcast(mine, pl);
                r[ks] = sel(tm.lane == kl, pv, r[ks]);
#pragma unroll
                for (int s = 0; s < R; ++s) r[s] = sel(tm.lane == pl && s == ps, kv, r[s]);
            }
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const TF yk = tm.bcast(r[k / T], k % T);
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (s * T + tm.lane > k) r[s] = Arith<true>::msub(a[s][k], yk, r[s]);
        }
#pragma unroll
        for (int k = N - 1; k >= 0; --k) {
            const int ks = k / T, kl = k % T;
            TF xk = r[ks] / a[ks][k];  // meaningful on the owner lane
            xk = tm.bcast(xk, kl);
            x[k] = xk;
#pragma unroll
            for (int s = 0; s < R; ++s)
                if (s * T + tm.lane < k) r[s] = Arith<true>::msub(a[s][k], xk, r[s]);
        }
    }

    // ldiv!!: same type (factors.jl:931-936) or mixed type (factors.jl:943-949), for the
    // lane's rows of the right-hand side; the solution is returned in every lane.
    __device__ __forceinline__ void ldiv(const Team<T>& tm, const double (&rr)[R], double (&d)[N]) const {
        if constexpr (sizeof(TF) == sizeof(double)) {
            unsigned long long mb = 0;
#pragma unroll
            for (int s = 0; s < R; ++s) {
                unsigned long long b = FBits<double>::bits(rr[s]) & ~FBits<double>::sign_mask;
                mb = b > mb ? b : mb;
            }
            mb = tm.umax(mb);
            double mm = FBits<double>::from(mb);
            const int m = (isfin(mm) && mm != 0.0) ? ::max(-1023, ::min(1023, jexponent(mm))) : 0;
            const int lo = e < 0 ? e : 0;
            const int ka = m > 0 ? 0 : (m < lo ? lo : m);
            const int kb = m - (1023 - headroom(N));
            const int k = ka > kb ? ka : kb;
            TF r[R], x[N];
#pragma unroll
            for (int s = 0; s < R; ++s) r[s] = k == 0 ? rr[s] : scale2_in(rr[s], -k);
            backsolve(tm, r, x);
            const int e2 = k - e;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = e2 == 0 ? double(x[i]) : scale2_in(double(x[i]), e2);
        } else {
            double s0 = 0.0;
#pragma unroll
            for (int s = 0; s < R; ++s) s0 = jmax(s0, fabs(rr[s]));
            const double sc = tm.max(s0);
            if (sc == 0.0) {
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = 0.0;
                return;
            }
            TF r[R], x[N];
#pragma unroll
            for (int s = 0; s < R; ++s) r[s] = TF(__ddiv_rn(rr[s], sc));
            backsolve(tm, r, x);
            int ex = 0;
            const double frac = isfin(sc) ? frexp(sc, &ex) : sc;
            if (!isfin(sc)) ex = 0;
            const int E = ex - e;
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const double v = __dmul_rn(double(x[i]), frac);
                d[i] = (E >= -1074 && E <= 2046) ? scale2_in(v, E) : ldexp2_slow(v, E);
            }
        }
    }
};

// A family in team form: row i of the residual, of the Jacobian and of the JVP, with the
// iterate held by every lane.
template <int N_> struct TeamCubic {
    static constexpr int N = N_, M = N_, NP = N_ * N_ + N_;
    static constexpr bool lsq = false;
    const double* p;
    __device__ __forceinline__ double par(int k) const { return lds(smem_addr(p) + 8u * k); }
    // Row i of F; xi = x[i], which the caller takes from its own slot.
    __device__ __forceinline__ double F(int i, double xi, const double (&x)[N]) const {
        double t = __dmul_rn(par(i), x[0]);
#pragma unroll
        for (int j = 1; j < N; ++j) t = __fma_rn(par(i + j * N), x[j], t);
        double c = __dmul_rn(__dmul_rn(xi, xi), xi);
        return __dsub_rn(__fma_rn(0.1, c, t), par(N * N + i));
    }
    __device__ __forceinline__ void J(int i, double xi, double (&row)[N]) const {
#pragma unroll
        for (int j = 0; j < N; ++j) row[j] = par(i + j * N);
        const double cp = __dadd_rn(__dmul_rn(__dadd_rn(xi, xi), xi), __dmul_rn(xi, xi));
        const double dii = __fma_rn(0.1, cp, par(i + i * N));
#pragma unroll
        for (int j = 0; j < N; ++j) row[j] = sel(j == i, dii, row[j]);
    }
    __device__ __forceinline__ double jvp(int i, double xi, double vi, const double (&v)[N]) const {
        double t = __dmul_rn(par(i), v[0]);
#pragma unroll
        for (int j = 1; j < N; ++j) t = __fma_rn(par(i + j * N), v[j], t);
        const double xv = __dmul_rn(vi, xi);
        const double x2p = __dadd_rn(xv, xv);
        const double cp = __dadd_rn(__dmul_rn(x2p, xi), __dmul_rn(vi, __dmul_rn(xi, xi)));
        return __fma_rn(0.1, cp, t);
    }
};

template <class Fam, int T, bool Mixed> struct TeamSolver {
    static constexpr int N = Fam::N, R = N / T;
    using A = Arith<true>;
    const Fam& fam;
    const GsbMethod& m;
    const GsbOptions& o;
    Team<T> tm;

    __device__ TeamSolver(const Fam& f, const GsbMethod& mm, const GsbOptions& oo) : fam(f), m(mm), o(oo) {}

    __device__ __forceinline__ bool has_merit() const { return m.globalization == GSB_BACKTRACKING; }
    __device__ __forceinline__ int row(int s) const { return s * T + tm.lane; }

    // The lane's rows of F(x) and norm2 over all rows.
    __device__ __forceinline__ double residual(const double (&x)[N], double (&F)[R]) const {
        double s2 = 0.0;
#pragma unroll
        for (int s = 0; s < R; ++s) {
            F[s] = fam.F(row(s), own<N, T>(x, s, tm.lane), x);
            s2 = __fma_rn(F[s], F[s], s2);
        }
        return tm.sum(s2);
    }

    // rnorm of a distributed vector whose norm2 is n2 (src/base/reductions.jl:348-364).
    __device__ double rnorm_dist(const double (&v)[R], double n2) const {
        if (isfin(n2) && n2 >= double(N) * kFloatmin) return sqrt(n2);
        double mx = 0.0;
#pragma unroll
        for (int s = 0; s < R; ++s) mx = jmax(mx, jmax(fabs(v[s]), 0.0));
        mx = tm.max(mx);
        if (mx == 0.0 || !isfin(mx)) return mx;
        const int e = jexponent(mx);
        double acc = 0.0;
#pragma unroll
        for (int s = 0; s < R; ++s) {
            const double u = scale2_in(v[s], -e);
            acc = __fma_rn(u, u, acc);
        }
        return scale2_in(sqrt(tm.sum(acc)), e);
    }
    __device__ __forceinline__ double rnorm_dist(const double (&v)[R]) const {
        double s2 = 0.0;
#pragma unroll
        for (int s = 0; s < R; ++s) s2 = __fma_rn(v[s], v[s], s2);
        return rnorm_dist(v, tm.sum(s2));
    }

    // grad_ratio_and_norm (src/nonlinear/newton.jl:1287-1298) on the distributed Jacobian.
    __device__ void grad_ratio(const double (&x)[N], const double (&F)[R], double fnorm, double& gr,
                               double& jnorm) const {
        double g[N];
        double js = 0.0;
#pragma unroll
        for (int j = 0; j < N; ++j) g[j] = 0.0;
#pragma unroll
        for (int s = 0; s < R; ++s) {
            double jr[N];
            fam.J(row(s), own<N, T>(x, s, tm.lane), jr);
#pragma unroll
            for (int j = 0; j < N; ++j) {
                js = __fma_rn(jr[j], jr[j], js);
                g[j] = __fma_rn(jr[j], F[s], g[j]);
            }
        }
        js = tm.sum(js);
        if (isfin(js) && js >= double(N * N) * kFloatmin) {
            jnorm = sqrt(js);
        } else {
            double mx = 0.0, acc = 0.0;
#pragma unroll
            for (int s = 0; s < R; ++s) {
                double jr[N];
                fam.J(row(s), own<N, T>(x, s, tm.lane), jr);
#pragma unroll
                for (int j = 0; j < N; ++j) mx = jmax(mx, fabs(jr[j]));
            }
            mx = tm.max(mx);
            if (mx == 0.0 || !isfin(mx)) {
                jnorm = mx;
            } else {
                const int e = jexponent(mx);
#pragma unroll
                for (int s = 0; s < R; ++s) {
                    double jr[N];
                    fam.J(row(s), own<N, T>(x, s, tm.lane), jr);
#pragma unroll
                    for (int j = 0; j < N; ++j) {
                        const double u = scale2_in(jr[j], -e);
                        acc = __fma_rn(u, u, acc);
                    }
                }
                jnorm = scale2_in(sqrt(tm.sum(acc)), e);
            }
        }
        if (jnorm == 0.0 || fnorm == 0.0) {
            gr = 0.0;
            return;
        }
#pragma unroll
        for (int j = 0; j < N; ++j) g[j] = tm.sum(g[j]);
        const double gnorm = rnorm<true, N>(g);
        gr = __ddiv_rn(__ddiv_rn(gnorm, jnorm), fnorm);  // the overflow rescue is not taken here
    }

    // J(x) v for the lane's rows (the held-Jacobian product of a refinement).
    __device__ __forceinline__ void jmul(const double (&x)[N], const double (&v)[N], double (&out)[R]) const {
#pragma unroll
        for (int s = 0; s < R; ++s) {
            double jr[N];
            fam.J(row(s), own<N, T>(x, s, tm.lane), jr);
            double t = __dmul_rn(jr[0], v[0]);
#pragma unroll
            for (int j = 1; j < N; ++j) t = __fma_rn(jr[j], v[j], t);
            out[s] = t;
        }
    }

    __device__ __forceinline__ double residual_norm(double merit, double fnorm, const double (&F)[R]) const {
        if (has_merit()) {
            if (isfin(merit) && merit >= double(N) * kFloatmin) return sqrt(merit);
            return rnorm_dist(F);
        }
        return isnan(fnorm) ? rnorm_dist(F) : fnorm;
    }

    // φ′(0) = 2 <F(x), J(x) d>.
    __device__ __forceinline__ double slope0(const double (&x)[N], const double (&d)[N]) const {
        double x0[N];
#pragma unroll
        for (int i = 0; i < N; ++i) x0[i] = __fma_rn(0.0, d[i], x[i]);
        double s = 0.0;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const double xq = own<N, T>(x0, q, tm.lane);
            s = __fma_rn(fam.F(row(q), xq, x0), fam.jvp(row(q), xq, own<N, T>(d, q, tm.lane), d), s);
        }
        return 2.0 * tm.sum(s);
    }

    // The globalizations, as the one-thread solve states them.
    __device__ void globalize(double (&x)[N], double (&F)[R], const double (&d)[N], bool exact,
                              double& merit, StepInfo& info) const {
        double xt[N], Ft[R];
        if (m.globalization == GSB_STATIC) {
            const double sa = m.static_alpha;
            const double dn = rnorm<true, N>(d);
            const double stepnorm = __dmul_rn(fabs(sa), dn);
            if (!isfin(stepnorm)) {
                info = {NONFINITE, rnorm_dist(F), stepnorm, 0, false, false, false};
                return;
            }
#pragma unroll
            for (int i = 0; i < N; ++i) xt[i] = __fma_rn(sa, d[i], x[i]);
            const double fn = rnorm_dist(Ft, residual(xt, Ft));
            if (!isfin(fn)) {
                info = {NONFINITE, rnorm_dist(F), stepnorm, 0, false, false, false};
                return;
            }
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = xt[i];
#pragma unroll
            for (int s = 0; s < R; ++s) F[s] = Ft[s];
            info = {SUCCESS, fn, stepnorm, 0, false, false, false};
            return;
        }
        const double phi0 = merit;
        const double dn = rnorm<true, N>(d);
        if (!isfin(dn)) {
            info = {NONFINITE, rnorm_dist(F), dn, 0, false, false, false};
            return;
        }
        double alpha = 1.0;
        const double d0 = exact ? -2.0 * phi0 : slope0(x, d);
        int code;
        double aa = alpha, pa = kNaN;
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
            const double c1 = m.bt_c1, pfac = m.bt_p;
            while (!done && trips < m.bt_maxiter) {
                ++trips;
                aa = alpha;
#pragma unroll
                for (int i = 0; i < N; ++i) xt[i] = __fma_rn(alpha, d[i], x[i]);
                pa = residual(xt, Ft);
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
                        const double sd = fabs(d0);
                        const double r1 = __dadd_rn(__ddiv_rn(__dsub_rn(pa, phi0), sd), alpha);
                        if (!(ap > 0.0)) {
                            if (r1 > 0.0) an = __ddiv_rn(__dmul_rn(alpha, alpha), __dmul_rn(2.0, r1));
                        } else if (isfin(pp) && alpha != ap) {
                            const double q1 = __ddiv_rn(r1, __dmul_rn(alpha, alpha));
                            const double q2 = __ddiv_rn(__dadd_rn(__ddiv_rn(__dsub_rn(pp, phi0), sd), ap),
                                                        __dmul_rn(ap, ap));
                            const double da = __dsub_rn(alpha, ap);
                            const double Aq = __ddiv_rn(__dsub_rn(q1, q2), da);
                            const double Bq = __ddiv_rn(__dsub_rn(__dmul_rn(alpha, q2), __dmul_rn(ap, q1)), da);
                            const double disc = __dadd_rn(__dmul_rn(Bq, Bq), __dmul_rn(3.0, Aq));
                            if (disc >= 0.0)
                                an = Bq > 0.0 ? __ddiv_rn(1.0, __dadd_rn(Bq, sqrt(disc)))
                                              : __ddiv_rn(__dadd_rn(-Bq, sqrt(disc)), __dmul_rn(3.0, Aq));
                        }
                        if (!(isfin(an) && an > 0.0)) an = __dmul_rn(pfac, alpha);
                        an = jmin(jmax(an, __dmul_rn(0.1, alpha)), __dmul_rn(pfac, alpha));
                    } else {
                        an = jmin(__dmul_rn(0.1, alpha), __dmul_rn(sqrt(alpha), sqrt(amin)));
                    }
                    ap = alpha;
                    pp = pa;
                    alpha = jmax(an, amin);
                }
            }
        }
        if (code == SUCCESS || (code == LINESEARCH_FAILED && isfin(pa) && pa < phi0)) {
#pragma unroll
            for (int i = 0; i < N; ++i) x[i] = xt[i];
#pragma unroll
            for (int s = 0; s < R; ++s) F[s] = Ft[s];
            info = {code, sqrt(pa), __dmul_rn(aa, dn), code == SUCCESS ? 0 : 1, false, false, aa < 1.0};
            merit = pa;
        } else if (code == LINESEARCH_FAILED) {
            info = {LINESEARCH_FAILED, rnorm_dist(F), 0.0, 1, false, false, false};
        } else if (code == STALLED) {
            info = {STALLED, rnorm_dist(F), 0.0, 0, false, false, false};
        } else {
            info = {NONFINITE, rnorm_dist(F), 0.0, 0, false, false, false};
        }
    }

    template <class Fac>
    __device__ bool refine(double (&d)[N], const Fac& fac, const double (&x)[N], const double (&F)[R]) const {
        const double fnorm = rnorm_dist(F);
        if (fnorm == 0.0) return false;
        if (!isfin(fnorm)) return true;
        const double thr = __dmul_rn(jmax(m.refine_eta, kSqrtEps), fnorm);
        double Jv[R], r[R];
        jmul(x, d, Jv);
#pragma unroll
        for (int s = 0; s < R; ++s) r[s] = __dadd_rn(-F[s], -Jv[s]);
        double rprev = rnorm_dist(r);
        if (!isfin(rprev)) return true;
        if (rprev <= thr) return false;
        for (int it = 1; it <= m.refine_maxiter; ++it) {
            double dd[N], dc[N];
            fac.ldiv(tm, r, dd);
#pragma unroll
            for (int i = 0; i < N; ++i) dc[i] = __dadd_rn(d[i], dd[i]);
            jmul(x, dc, Jv);
#pragma unroll
            for (int s = 0; s < R; ++s) r[s] = __dadd_rn(-F[s], -Jv[s]);
            const double rc = rnorm_dist(r);
            if (!(rc < rprev)) return true;
#pragma unroll
            for (int i = 0; i < N; ++i) d[i] = dc[i];
            rprev = rc;
            if (rc <= thr) return false;
        }
        return true;
    }

    __device__ void step(DevState& st, double (&x)[N], double (&F)[R], StepInfo& info) const {
        const double fnorm = residual_norm(st.merit, st.fnorm, F);
        const bool was_promoted = st.promoted;
        double gr, jn;
        grad_ratio(x, F, fnorm, gr, jn);
        st.gradratio = gr;
        st.jnorm = jn;
        const bool ref = m.refinement == GSB_REFINEMENT;
        double xo[R];
#pragma unroll
        for (int q = 0; q < R; ++q) xo[q] = own<N, T>(x, q, tm.lane);
        auto jrow = [&](int q, double (&out)[N]) { fam.J(row(q), xo[q], out); };
        double d[N];
        bool ok = true;
        int failures = 0;
        double lin_rel = 0.0;
        bool md_promoted = was_promoted;
        bool fallback = !Mixed || was_promoted;
        if constexpr (Mixed) {
            if (!was_promoted) {
                TeamLU<N, T, float> fac;
                fac.factor(tm, jrow);
                bool ref_failed;
                if (fac.info > 0) {
                    ref_failed = true;
                } else {
                    fac.ldiv(tm, F, d);
#pragma unroll
                    for (int i = 0; i < N; ++i) d[i] = -d[i];
                    ref_failed = ref ? refine(d, fac, x, F) : false;
                }
                if (ref_failed || fac.info > 0) {
                    failures += 1;
                    md_promoted = true;
                    fallback = true;
                } else if (fnorm == 0.0 || !isfin(fnorm)) {
                    lin_rel = 0.0;
                } else {
                    double Jd[R], lin[R];
                    jmul(x, d, Jd);
#pragma unroll
                    for (int s = 0; s < R; ++s) lin[s] = __dadd_rn(F[s], Jd[s]);
                    lin_rel = __ddiv_rn(rnorm_dist(lin), fnorm);
                }
            }
        }
        if (fallback) {
            TeamLU<N, T, double> ft;
            ft.factor(tm, jrow);
            if (ft.info > 0) {
                ok = false;
            } else {
                ft.ldiv(tm, F, d);
#pragma unroll
                for (int i = 0; i < N; ++i) d[i] = -d[i];
                if (ref && (!Mixed || was_promoted)) refine(d, ft, x, F);
            }
        }
        if (!ok) {
            if (Mixed) st.promoted = md_promoted;
            info = {SINGULAR, rnorm_dist(F), 0.0, failures, Mixed && md_promoted, false, false};
            if (!Mixed) st.fnorm = info.fnorm;
            return;
        }
        const bool exact = Mixed ? md_promoted : !ref;
        double merit = st.merit;
        globalize(x, F, d, exact, merit, info);
        if constexpr (Mixed) {
            info.failures += failures;
            if (md_promoted && !was_promoted) {
                info.promoted = true;
                st.promoted = true;
                st.slow_steps = 0;
            } else if (!was_promoted) {
                if (info.fnorm > __dmul_rn(0.5, fnorm) && lin_rel > 1e-4) {
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
        }
        st.merit = merit;
        st.fnorm = info.fnorm;
    }

    __device__ __forceinline__ bool residual_converged(const DevStatus& s, double ft, double ft0) const {
        if (!(s.iterations >= o.min_iterations)) return false;
        return ft <= jmax(o.f_abstol, __dmul_rn(o.f_reltol, ft0));
    }

    __device__ double maxabs(const double (&F)[R]) const {
        double mx = fabs(F[0]);
#pragma unroll
        for (int s = 1; s < R; ++s) mx = jmax(mx, fabs(F[s]));
        return tm.max(mx);
    }

    // solve!!, src/nonlinear/solver.jl:277-378 (square problems).
    __device__ DevStatus solve(double (&x)[N], double& gr_out) const {
        double F[R];
        const double n2 = residual(x, F);
        const double fnorm0 = rnorm_dist(F, n2);
        DevState st{has_merit() ? n2 : kNaN, fnorm0, kNaN, 0.0, false, 0};
        DevStatus s{SUCCESS, 0, fnorm0, 0.0, 0, false, false, kNaN, false};
        gr_out = kNaN;
        if (!isfin(fnorm0)) {
            s.code = NONFINITE;
            return s;
        }
        const double ftest0 = o.norm == 1 ? maxabs(F) : fnorm0;
        if (residual_converged(s, ftest0, ftest0)) return s;
        if (o.max_iterations == 0) {
            s.code = MAXITERS;
            return s;
        }
        int stalls = 0;
        while (true) {
            const double rate_k = s.rate;
            StepInfo info;
            step(st, x, F, info);
            record(s, info);
            gr_out = st.gradratio;
            if (info.code == SINGULAR || info.code == NONFINITE || info.code == MAXITERS) return s;
            if (info.code == LINESEARCH_FAILED && info.stepnorm == 0.0) return s;
            const double ft = o.norm == 1 ? maxabs(F) : s.fnorm;
            if (residual_converged(s, ft, ftest0)) {
                s.code = SUCCESS;
                return s;
            }
            const bool steptested = !(info.code == STALLED || info.limited);
            const double xnorm = steptested ? rnorm<true, N>(x) : kNaN;
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
                s.contracted = contracted;
                return s;
            }
            if (info.code == STALLED) {
                if (++stalls >= o.max_stalls) {
                    s.code = STALLED;
                    return s;
                }
            } else {
                stalls = 0;
            }
            if (s.iterations >= o.max_iterations) {
                s.code = MAXITERS;
                return s;
            }
        }
    }
};

}  // namespace gsb
