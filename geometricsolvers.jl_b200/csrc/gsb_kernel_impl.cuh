// The batch kernel template: parameter staging, one Newton solve per thread, the stores of the
// iterate and the 72-byte status, and the tally of the count form. Instantiated per family and
// size in the gsb_inst_*.cu translation units.
#pragma once

#include <cuda_runtime.h>

#include "../../include/gsb.h"
#include "gsb_families.cuh"
#include "gsb_lm.cuh"
#include "gsb_newton.cuh"
#include "gsb_numerics.cuh"
#include "gsb_team.cuh"
#include "gsb_umma.cuh"
#include "gsb_warp.cuh"

namespace gsb {

constexpr int kThreads = 128;

// batch_summary partials (src/nonlinear/batched.jl:63-89): Σ fnorm², max |fnorm|, failures,
// max and Σ iterations, whether a fnorm was NaN.
struct SummaryAcc {
    double sumsq;
    unsigned long long maxbits;  // bits of max |fnorm| (non-negative doubles order as integers)
    unsigned long long failures;
    unsigned long long total_iterations;
    int max_iterations;
    int nan_seen;
};

// One thread's share of a batch summary: the statuses it closed.
struct SummaryPart {
    double sumsq = 0.0;
    unsigned long long maxbits = 0, failures = 0, iterations = 0;
    int max_iterations = 0, nan = 0;

    __device__ __forceinline__ void add(const DevStatus& s) {
        sumsq = __fma_rn(s.fnorm, s.fnorm, sumsq);
        const unsigned long long b = (unsigned long long)__double_as_longlong(fabs(s.fnorm));
        maxbits = b > maxbits ? b : maxbits;
        nan |= s.fnorm != s.fnorm;
        failures += s.code != 0;
        iterations += (unsigned long long)s.iterations;
        max_iterations = s.iterations > max_iterations ? s.iterations : max_iterations;
    }

    // The parts of the active lanes of the warp, added up by the first of them into acc.
    __device__ __forceinline__ void flush(SummaryAcc* acc) const {
        const unsigned mask = __activemask();
        const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
        double sq = 0.0;
        unsigned long long mb = 0, fl = 0, it = 0;
        int mx = 0, nn = 0;
        for (int l = 0; l < 32; ++l) {
            if (!(mask & (1u << l))) continue;
            sq += __shfl_sync(mask, sumsq, l);
            const unsigned long long b = __shfl_sync(mask, maxbits, l);
            mb = b > mb ? b : mb;
            fl += __shfl_sync(mask, failures, l);
            it += __shfl_sync(mask, iterations, l);
            const int m = __shfl_sync(mask, max_iterations, l);
            mx = m > mx ? m : mx;
            nn |= __shfl_sync(mask, nan, l);
        }
        if (lane == leader) {
            atomicAdd(&acc->sumsq, sq);
            atomicMax(&acc->maxbits, mb);
            atomicAdd(&acc->failures, fl);
            atomicAdd(&acc->total_iterations, it);
            atomicMax(&acc->max_iterations, mx);
            atomicOr(&acc->nan_seen, nn);
        }
    }
};

struct Launch {
    double* X;
    int x_layout;
    void* S;
    int s_kind;
    const double* P;
    int p_layout;
    const int64_t* order;
    int order_base;
    int64_t nsys;
    const double* shared;
    unsigned long long* tally;  // 6 counters or nullptr
    // Ragged batches (systems of different sizes packed back to back): the offsets, in doubles,
    // of each system's iterate in X and parameter block in P, indexed like S; nullptr for the
    // uniform layouts.
    const int64_t* x_off;
    const int64_t* p_off;
    // Persistent launches: a counter of CTA-sized chunks taken so far (zero at launch); nullptr
    // for one chunk per CTA.
    unsigned long long* queue;
    // A bucket of a ragged batch: {count, first} in device memory, written on the device before
    // the launch; the launch then solves order[first .. first + count) instead of order[0 ..
    // nsys). nullptr otherwise.
    const unsigned long long* bucket;
    // Set to nonzero when a wait for a staging copy ran out (the systems of that CTA are then
    // left unsolved); nullptr for none.
    unsigned* fault;
    // The batch summary of the statuses the launch writes, accumulated as they close (the
    // fused batch_summary); nullptr for none.
    SummaryAcc* summary;
};

// The systems a launch solves: `n` entries of `order` (or 0 .. n-1 without one).
struct Range {
    int64_t n;
    const int64_t* order;
};

__device__ __forceinline__ Range launch_range(const Launch& L) {
    if (L.bucket) return {(int64_t)L.bucket[0], L.order + L.bucket[1]};
    return {L.nsys, L.order};
}

// The CTA's chunks: one per CTA, or (persistent launches) chunks taken from the work queue
// until the batch is exhausted (systems_per_chunk systems each).
template <bool Persistent, class Body>
__device__ __forceinline__ void for_each_chunk(const Launch& L, int64_t systems_per_chunk, Body body) {
    const Range r = launch_range(L);
    if constexpr (!Persistent) {
        // one chunk per CTA: no loop around the solve, whose registers it would hold
        body((int64_t)blockIdx.x * systems_per_chunk, r);
        return;
    }
    // Each chunk's ticket is taken one chunk ahead, so that its atomic's round trip overlaps
    // the solve of the chunk before it: thread 0 writes slot b ^ 1 while the CTA reads slot b,
    // and the barrier at the end of each chunk orders the two (a CTA that leaves has taken one
    // ticket past the end, which only counts the queue further past it).
    __shared__ unsigned long long next[2];
    if (threadIdx.x == 0) next[0] = atomicAdd(L.queue, 1ull);
    __syncthreads();
    int b = 0;
    while (true) {
        const int64_t base = (int64_t)next[b] * systems_per_chunk;
        if (base >= r.n) return;
        if (threadIdx.x == 0) next[b ^ 1] = atomicAdd(L.queue, 1ull);
        body(base, r);
        __syncthreads();  // the chunk's shared memory is free again; next[b ^ 1] is written
        b ^= 1;
    }
}

__device__ __forceinline__ const double* param_block(const Launch& L, int64_t idx, int np) {
    return L.p_off ? L.P + L.p_off[idx] : L.P + idx * np;
}
__device__ __forceinline__ double* x_block(const Launch& L, int64_t idx, int n) {
    return L.x_off ? L.X + L.x_off[idx] : L.X + idx * n;
}

// Row of a thread's shared memory: its parameter block (np doubles), then 2n doubles where the
// iterate and the residual wait while a factor holds the registers; the stride is odd, so that
// thread t's entry k (address t*RS + k) falls in a distinct 8-byte bank slot for the 16 threads
// of each half-warp access.
__host__ __device__ constexpr int row_stride(int np, int n) {
    return ((np + 2 * n) % 2 == 1) ? np + 2 * n : np + 2 * n + 1;
}

// The row stride of the one-thread kernel. A family that reads its block in aligned pairs
// (PairsOf) takes 16-byte aligned rows, staged by one bulk copy each: a stride of 2 mod 4
// doubles, at which the 16-byte accesses of each quarter-warp fall on distinct banks.
template <class Fam> __host__ __device__ constexpr int newton_row_stride() {
    if constexpr (PairsOf<Fam>::value) {
        constexpr int need = Fam::NP + 2 * Fam::N;
        return need + ((2 - need % 4) + 4) % 4;
    } else {
        return row_stride(Fam::NP, Fam::N);
    }
}

// Polls of a staging wait before it gives up: far beyond the microseconds a copy of a few hundred
// bytes takes, and finite.
constexpr uint32_t kStageWaitPolls = 1u << 22;

// Stage one system's parameter block (NP doubles from src) into a 16-byte aligned shared row by
// one bulk copy that completes on `bar` (the thread arrives with the bytes it expects), or, when
// the source is not 16-byte aligned, by loads and stores of its own followed by a plain arrival.
template <int NP>
__device__ __forceinline__ void stage_row_bulk(double* row, const double* src, uint64_t* bar) {
    static_assert((NP * 8) % 16 == 0, "a bulk copy moves a multiple of 16 bytes");
    const unsigned b = smem_addr(bar);
    if ((reinterpret_cast<uintptr_t>(src) & 15u) == 0) {
        umma::fence_async_shared();  // earlier generic accesses of the row before the copy's writes
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(NP * 8)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                smem_addr(row)),
            "l"(src), "r"(NP * 8), "r"(b)
            : "memory");
        return;
    }
#pragma unroll 4
    for (int k = 0; k < NP; ++k) row[k] = __ldg(src + k);
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(b) : "memory");
}
// A system's start iterate into registers (AoS, SoA, or ragged offsets).
template <int N>
__device__ __forceinline__ void load_x(const Launch& L, int64_t idx, double (&x)[N]) {
    const double* xb = x_block(L, idx, N);
#pragma unroll
    for (int k = 0; k < N; ++k) x[k] = L.x_layout == GSB_SOA ? L.X[(int64_t)k * L.nsys + idx] : xb[k];
}

__device__ __forceinline__ void stage_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// The 72-byte status record (GsbStatus64) of a system as nine 8-byte words.
__device__ __forceinline__ void status_words(const DevStatus& s, double gr, unsigned long long (&w)[9]) {
    w[0] = (unsigned long long)(unsigned char)s.code |
           ((unsigned long long)(unsigned int)s.iterations << 32);
    w[1] = (unsigned long long)__double_as_longlong(s.fnorm);
    w[2] = (unsigned long long)__double_as_longlong(s.stepnorm);
    w[3] = (unsigned long long)(unsigned int)s.step_failures |
           ((unsigned long long)(s.promoted ? 1u : 0u) << 32) |
           ((unsigned long long)(s.stationary ? 1u : 0u) << 40);
    w[4] = (unsigned long long)(unsigned int)(-1);
    w[5] = (unsigned long long)__double_as_longlong(kNaN);
    w[6] = (unsigned long long)__double_as_longlong(gr);
    w[7] = (unsigned long long)__double_as_longlong(s.rate);
    w[8] = (unsigned long long)(s.contracted ? 1u : 0u) | ((unsigned long long)(s.reused ? 1u : 0u) << 8);
}

__device__ __forceinline__ void store_status(void* S, int64_t idx, const DevStatus& s, double gr) {
    unsigned long long* o = reinterpret_cast<unsigned long long*>(
        reinterpret_cast<unsigned char*>(S) + idx * 72);
    unsigned long long w[9];
    status_words(s, gr, w);
#pragma unroll
    for (int k = 0; k < 9; ++k) o[k] = w[k];
}

__device__ __forceinline__ void tally_code(unsigned long long* tally, int code) {
    unsigned mask = __activemask();
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        unsigned b = __ballot_sync(mask, code == c);
        if (lane == leader && b) atomicAdd(tally + c, (unsigned long long)__popc(b));
    }
}

// Stage the contiguous AoS parameter chunk of a CTA (`rows_left` blocks of NP doubles from src,
// at most ROWS) into rows of stride RS in shared memory (entry k of a block at `place(k)`), as
// asynchronous 8-byte global-to-shared copies: the warp's lanes copy consecutive doubles
// (coalesced), every copy of a thread is in flight at once and holds no register, and the
// thread waits once for all of them. The caller's barrier then publishes the rows to the CTA.
struct IdentityPlace {
    __device__ __forceinline__ int operator()(int k) const { return k; }
};

template <int NP, int RS, int ROWS, class Place = IdentityPlace>
__device__ __forceinline__ void stage_aos(double* smem, const double* src, int64_t rows_left, int tid,
                                          Place place = Place()) {
    constexpr int TOTAL = ROWS * NP;
    const int total = rows_left < ROWS ? (int)rows_left * NP : TOTAL;
    for (int q = tid; q < total; q += kThreads) {
        const int s = q / NP;
        const unsigned dst = smem_addr(smem + s * RS + place(q - s * NP));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src + q) : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// The same for a CTA of `nthreads` threads staging `rows` rows (the CTA size chosen at launch).
template <int NP, int RS, class Place = IdentityPlace>
__device__ __forceinline__ void stage_aos_rows(double* smem, const double* src, int64_t rows_left,
                                               int rows, int tid, int nthreads,
                                               Place place = Place()) {
    const int total = (rows_left < rows ? (int)rows_left : rows) * NP;
    for (int q = tid; q < total; q += nthreads) {
        const int s = q / NP;
        const unsigned dst = smem_addr(smem + s * RS + place(q - s * NP));
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(src + q) : "memory");
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// Resident 128-thread blocks per SM that the register allocation must allow, by system size.
// Measured on B200 for 1M systems: n = 4 runs 18-21% faster at 4 blocks (128 registers) than at
// the allocator's own choice, n = 6 30% (plain, 4 blocks) and 20% (mixed, 3 blocks); n = 8 needs
// more than 170 registers, and capping it spills (plain 1.75 ms at 2 blocks, 2.12 ms at 3).
template <class Fam, bool Mixed> constexpr int min_blocks() {
#ifdef GSB_MIN_BLOCKS
    return GSB_MIN_BLOCKS;
#else
    return Fam::N <= 4 ? 4 : Fam::N <= 6 ? (Mixed ? 3 : 4) : 1;
#endif
}

// The Newton solve of one system by its thread, once its parameter row is staged.
template <class Fam, bool F, bool Mixed, bool PlainRef, bool Qr, int Kind = kStepNewton>
__device__ __forceinline__ DevStatus solve_one(const GsbMethod& m, const GsbOptions& o,
                                               const double* smem, double* prow,
                                               double (&x)[Fam::N], double& gr) {
    constexpr int N = Fam::N, NP = Fam::NP;
    Fam fam{prow};
    if constexpr (SharedLen<Fam>::value > 0) fam.a = smem;
    Solver<Fam, F, Mixed, PlainRef, Qr, Kind> sv(fam, m, o, N >= 6 ? prow + NP : nullptr);
    return sv.solve(x, gr);
}

// A warp's stores of 32 consecutive systems (base .. base + 31, AoS iterates, 72-byte statuses,
// both arrays 16-byte aligned): each lane puts its status words and then its iterate into `buf`
// (shared memory the warp no longer reads, 16-byte aligned, at least 32 * max(9, N) doubles),
// and the warp copies the 2,304 status bytes and the 32 * 8N iterate bytes out as 16-byte stores
// that fill whole lines.
template <int N>
__device__ __forceinline__ void store_warp(const Launch& L, int64_t base, int lane, double* buf,
                                           const double (&x)[N], const DevStatus& s, double gr) {
    static_assert((N * 8) % 16 == 0, "16-byte pieces of the iterates");
    const unsigned b = smem_addr(buf);
    unsigned long long w[9];
    status_words(s, gr, w);
#pragma unroll
    for (int k = 0; k < 9; ++k) sts(b + 8u * (lane * 9 + k), __longlong_as_double((long long)w[k]));
    __syncwarp();
    unsigned char* sb = reinterpret_cast<unsigned char*>(L.S) + base * 72;
#pragma unroll
    for (int q = lane; q < 144; q += 32) {
        double v0, v1;
        lds2(b + 16u * q, v0, v1);
        asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(sb + 16 * q), "d"(v0), "d"(v1) : "memory");
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < N; ++k) sts(b + 8u * (lane * N + k), x[k]);
    __syncwarp();
    double* xb = L.X + base * N;
#pragma unroll
    for (int q = lane; q < 32 * N / 2; q += 32) {
        double v0, v1;
        lds2(b + 16u * q, v0, v1);
        asm volatile("st.global.v2.f64 [%0], {%1, %2};" ::"l"(xb + 2 * q), "d"(v0), "d"(v1) : "memory");
    }
}

// The thread's stores of its system's iterate and status (or code).
template <int N>
__device__ __forceinline__ void store_one(const Launch& L, int64_t idx, const double (&x)[N],
                                          const DevStatus& s, double gr) {
    double* xb = x_block(L, idx, N);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (L.x_layout == GSB_SOA) L.X[(int64_t)k * L.nsys + idx] = x[k];
        else xb[k] = x[k];
    }
    if (L.s_kind == GSB_STATUS64) store_status(L.S, idx, s, gr);
    else reinterpret_cast<unsigned char*>(L.S)[idx] = (unsigned char)s.code;
}

template <class Fam, bool F, bool Mixed, bool PlainRef, bool Persistent, bool Qr = false,
          int Kind = kStepNewton>
__global__ void __launch_bounds__(kThreads, (min_blocks<Fam, Mixed>())) newton_kernel(const __grid_constant__ GsbMethod m,
                                 const __grid_constant__ GsbOptions o,
                                 const __grid_constant__ Launch L) {
    extern __shared__ __align__(16) double smem[];
    constexpr int N = Fam::N, NP = Fam::NP, RS = newton_row_stride<Fam>();
    // a family's block shared by the batch (BatchParams) first, then one row per thread
    constexpr int SH = SharedLen<Fam>::value, SHP = ((SH + 1) / 2) * 2;
    const int tid = threadIdx.x;
    double* rows = smem + SHP;
    double* prow = rows + tid * RS;
    if constexpr (SH > 0) {
        for (int q = tid; q < SH; q += kThreads) smem[q] = __ldg(L.shared + q);
        __syncthreads();
    }
    if constexpr (PairsOf<Fam>::value) {
        // Each warp works on its own: it stages the rows of its 32 systems (one bulk copy per
        // system, completing on the warp's mbarrier), solves them, and takes its next 32 (from a
        // fixed stride over the grid's warps, or from the launch's work queue), so that one
        // warp's wait for its copies overlaps the arithmetic of the others and no warp waits for
        // the slowest system of another. The grid holds the resident CTAs only.
        constexpr int W = kThreads / 32;
        const int warp = tid >> 5, lane = tid & 31;
        __shared__ __align__(8) uint64_t wbar[W];
        if (lane == 0) {
            umma::mbar_init(&wbar[warp], 32);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        __syncwarp();
        const Range r = launch_range(L);
        uint32_t phase = 0;
        SummaryPart part;  // the lane's statuses, for a fused batch summary
        int64_t c = (int64_t)blockIdx.x * W + warp;
        // persistent launches: lane 0 takes each ticket one chunk ahead, so that the atomic's
        // round trip overlaps the chunk before it
        unsigned long long ahead = 0;
        if constexpr (Persistent) {
            if (lane == 0) ahead = atomicAdd(L.queue, 1ull);
        }
        while (true) {
            if constexpr (Persistent) {
                c = (int64_t)__shfl_sync(0xffffffffu, ahead, 0);
                if (lane == 0 && c * 32 < r.n) ahead = atomicAdd(L.queue, 1ull);
            }
            if (c * 32 >= r.n) break;
            const int64_t i = c * 32 + lane;
            const bool mine = i < r.n;
            const int64_t idx = mine ? (r.order ? r.order[i] - L.order_base : i) : 0;
            double x[N];
            if (mine) {
                if (L.p_layout == GSB_SOA) {
#pragma unroll 4
                    for (int k = 0; k < NP; ++k) prow[k] = __ldg(L.P + (int64_t)k * L.nsys + idx);
                    stage_arrive(&wbar[warp]);
                } else {
                    stage_row_bulk<NP>(prow, param_block(L, idx, NP), &wbar[warp]);
                }
                load_x<N>(L, idx, x);  // in flight while the copies land
            } else {
                stage_arrive(&wbar[warp]);
            }
            const bool staged =
                __all_sync(0xffffffffu, umma::mbar_wait(&wbar[warp], phase, kStageWaitPolls));
            phase ^= 1u;
            if (!staged) {
                // the copies did not land: record it, give them a second bounded wait, and
                // leave this warp's systems unsolved
                if (L.fault && lane == 0) *reinterpret_cast<volatile unsigned*>(L.fault) = 1u;
                umma::mbar_wait(&wbar[warp], phase ^ 1u, kStageWaitPolls);
                break;
            }
            __syncwarp();  // the lanes' own stores of their rows (SoA) before any read
            DevStatus st{};
            double gr = kNaN;
            if (mine) st = solve_one<Fam, F, Mixed, PlainRef, Qr, Kind>(m, o, smem, prow, x, gr);
            __syncwarp();  // the rows are free again
            static_assert(RS >= 9 && RS >= N, "a warp's rows hold its 32 statuses and iterates");
            if (c * 32 + 32 <= r.n && r.order == nullptr && L.s_kind == GSB_STATUS64 &&
                L.x_layout == GSB_AOS && L.x_off == nullptr &&
                ((reinterpret_cast<uintptr_t>(L.S) | reinterpret_cast<uintptr_t>(L.X)) & 15u) == 0) {
                // whole lines: the warp's statuses and iterates pass through its own free rows
                store_warp<N>(L, c * 32, lane, rows + warp * 32 * RS, x, st, gr);
                __syncwarp();
            } else if (mine) {
                store_one<N>(L, idx, x, st, gr);
            }
            if (L.tally && mine) tally_code(L.tally, st.code);
            if (L.summary && mine) part.add(st);
            if constexpr (!Persistent) c += (int64_t)gridDim.x * W;
        }
        if (L.summary) part.flush(L.summary);  // every lane leaves the loop together
        return;
    } else {
        for_each_chunk<Persistent>(L, kThreads, [&](int64_t base, const Range& r) {
            const int64_t i = base + tid;
            if (r.order == nullptr && L.p_layout == GSB_AOS && L.p_off == nullptr) {
                stage_aos<NP, RS, kThreads>(rows, L.P + base * NP, r.n - base, tid);
            } else if (i < r.n) {
                const int64_t idx = r.order ? r.order[i] - L.order_base : i;
                if (L.p_layout == GSB_SOA) {
#pragma unroll 4
                    for (int k = 0; k < NP; ++k) prow[k] = __ldg(L.P + (int64_t)k * L.nsys + idx);
                } else {
                    const double* pb = param_block(L, idx, NP);
#pragma unroll 4
                    for (int k = 0; k < NP; ++k) prow[k] = __ldg(pb + k);
                }
            }
            __syncthreads();
            if (i >= r.n) return;
            const int64_t idx = r.order ? r.order[i] - L.order_base : i;
            double x[N];
            load_x<N>(L, idx, x);
            double gr;
            const DevStatus st = solve_one<Fam, F, Mixed, PlainRef, Qr, Kind>(m, o, smem, prow, x, gr);
            store_one<N>(L, idx, x, st, gr);
            if (L.tally) tally_code(L.tally, st.code);
            if (L.summary) {
                SummaryPart part;
                part.add(st);
                part.flush(L.summary);
            }
        });
    }
}


// The team form: T lanes per system, kThreads / T systems per CTA, each system's parameter block
// staged into a shared-memory row that its lanes read.
template <class Fam, int T, bool Mixed, bool Persistent>
__global__ void __launch_bounds__(kThreads) team_kernel(const __grid_constant__ GsbMethod m,
                                 const __grid_constant__ GsbOptions o,
                                 const __grid_constant__ Launch L) {
    extern __shared__ double smem[];
    constexpr int N = Fam::N, NP = Fam::NP, RS = (NP % 2 == 1) ? NP : NP + 1;
    constexpr int SPB = kThreads / T;
    const int tid = threadIdx.x;
    const int team = tid / T;
    for_each_chunk<Persistent>(L, SPB, [&](int64_t base, const Range& r) {
        const int64_t i = base + team;
        if (r.order == nullptr && L.p_layout == GSB_AOS && L.p_off == nullptr) {
            stage_aos<NP, RS, SPB>(smem, L.P + base * NP, r.n - base, tid);
        } else if (i < r.n) {
            const int64_t idx = r.order ? r.order[i] - L.order_base : i;
            double* prow = smem + team * RS;
            const double* pb = param_block(L, idx, NP);
            for (int k = tid % T; k < NP; k += T)
                prow[k] = L.p_layout == GSB_SOA ? __ldg(L.P + (int64_t)k * L.nsys + idx) : __ldg(pb + k);
        }
        __syncthreads();
        if (i >= r.n) return;
        const int64_t idx = r.order ? r.order[i] - L.order_base : i;
        Fam fam{smem + team * RS};
        double* xb = x_block(L, idx, N);
        double x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = L.x_layout == GSB_SOA ? L.X[(int64_t)k * L.nsys + idx] : xb[k];
        TeamSolver<Fam, T, Mixed> sv(fam, m, o);
        double gr;
        DevStatus s = sv.solve(x, gr);
        const int lane = tid % T;
#pragma unroll
        for (int q = 0; q < N / T; ++q) {
            const int k = q * T + lane;
            const double v = own<N, T>(x, q, lane);
            if (L.x_layout == GSB_SOA) L.X[(int64_t)k * L.nsys + idx] = v;
            else xb[k] = v;
        }
        if (lane == 0) {
            if (L.s_kind == GSB_STATUS64) store_status(L.S, idx, s, gr);
            else reinterpret_cast<unsigned char*>(L.S)[idx] = (unsigned char)s.code;
            if (L.tally) tally_code(L.tally, s.code);
            if (L.summary) {
                SummaryPart part;
                part.add(s);
                part.flush(L.summary);
            }
        }
    });
}

// The least-squares form: one Levenberg–Marquardt solve per thread, with the thread's
// observations in a shared-memory row and the abscissae shared by the CTA. Iteration counts
// differ widely between systems (in the exponential-sum batch about half run to max_iterations
// while the rest converge early) and a warp steps as long as its slowest lane, so the grid holds
// the resident CTAs only, each CTA works through a contiguous range of systems, and a lane whose
// system closes stores it and takes the range's next system from a shared-memory counter. Each
// system's solve is the same sequence of steps as a solve of its own. Two CTAs per SM: the solve
// then fits its registers without spilling, which measured faster than three CTAs at 168.
template <class Fam, bool F, bool Mixed>
__global__ void __launch_bounds__(kThreads, 2) lm_kernel(const __grid_constant__ GsbMethod m,
                                 const __grid_constant__ GsbOptions o,
                                 const __grid_constant__ Launch L) {
    extern __shared__ double smem[];
    __shared__ unsigned long long next;
    constexpr int N = Fam::N, M = Fam::M, RS = (M % 2 == 1) ? M : M + 1;
    const int tid = threadIdx.x;
    const int64_t chunk = (L.nsys + gridDim.x - 1) / gridDim.x;
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t count = (L.nsys - lo < chunk ? L.nsys - lo : chunk);
    if (count <= 0) return;  // the whole CTA
    double* prow = smem + tid * RS;
    double* tsh = smem + kThreads * RS;
    for (int k = tid; k < M; k += blockDim.x) tsh[k] = __ldg(L.shared + k);
    auto index = [&](int64_t i) { return L.order ? L.order[i] - L.order_base : i; };
    auto load_row = [&](int64_t idx) {
        if (L.p_layout == GSB_SOA) {
#pragma unroll 4
            for (int k = 0; k < M; ++k) prow[k] = __ldg(L.P + (int64_t)k * L.nsys + idx);
        } else {
#pragma unroll 4
            for (int k = 0; k < M; ++k) prow[k] = __ldg(L.P + idx * M + k);
        }
    };
    // the range's first kThreads systems, staged together
    const int64_t first = count < kThreads ? count : kThreads;
    if (L.order == nullptr && L.p_layout == GSB_AOS) {
        stage_aos<M, RS, kThreads>(smem, L.P + lo * M, first, tid);
    } else if (tid < first) {
        load_row(index(lo + tid));
    }
    if (tid == 0) next = (unsigned long long)first;
    __syncthreads();
    Fam fam{prow, tsh};
    LMSolver<Fam, F, Mixed> sv(fam, m, o);
    typename LMSolver<Fam, F, Mixed>::Run run;
    double x[N];
    auto start = [&](int64_t idx) {
#pragma unroll
        for (int k = 0; k < N; ++k)
            x[k] = L.x_layout == GSB_SOA ? L.X[(int64_t)k * L.nsys + idx] : L.X[idx * N + k];
        sv.begin(x, run);
    };
    bool active = tid < first;
    int64_t idx = active ? index(lo + tid) : 0;
    if (active) start(idx);
    while (true) {
        while (active && run.done) {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                if (L.x_layout == GSB_SOA) L.X[(int64_t)k * L.nsys + idx] = x[k];
                else L.X[idx * N + k] = x[k];
            }
            if (L.s_kind == GSB_STATUS64) store_status(L.S, idx, run.s, run.gr);
            else reinterpret_cast<unsigned char*>(L.S)[idx] = (unsigned char)run.s.code;
            if (L.tally) tally_code(L.tally, run.s.code);
            if (L.summary) {
                SummaryPart part;
                part.add(run.s);
                part.flush(L.summary);
            }
            const long long q = (long long)atomicAdd(&next, 1ull);
            active = q < count;
            if (active) {
                idx = index(lo + q);
                load_row(idx);
                start(idx);
            }
        }
        if (!active) break;
        sv.iterate(x, run);
    }
}

// The warp form (n = 12 ... 32): T lanes per system, blockDim.x / T systems per CTA (up to
// kThreads / T; the launch chooses). Each system's shared memory holds its parameter block in
// the family's layout (SP doubles), then its factor's part (the whole factor for teams of 16,
// the two pivot-row buffers for teams of 32, whose rows live in the lanes' registers).
template <class Fam, int T> __host__ __device__ constexpr int warp_sys_stride() {
    return ((Fam::SP + 1) / 2) * 2 + warp_lu_doubles<Fam::N, T>();
}

// Shared memory of a batch-wide matrix at the start of a warp-form CTA (BatchParams), in doubles
// (A with the family's column stride, rounded up to 16 bytes); 0 for a per-system block.
template <class Fam, class = void> struct WarpSharedA {
    static constexpr int doubles = 0;
};
template <class Fam> struct WarpSharedA<Fam, decltype(void(Fam::kSharedA))> {
    static constexpr int doubles = Fam::kSharedA ? ((Fam::N * Fam::LDA + 1) / 2) * 2 : 0;
};

// Parameter k of a system to its place in the family's shared-memory layout.
template <class Fam> struct WarpPlace {
    __device__ __forceinline__ int operator()(int k) const { return Fam::place(k); }
};

// Resident 128-thread blocks per SM that the warp kernel's register allocation must allow (0:
// no bound). Measured on B200 (65,536 systems, 2 steps each): a team of 32 at n = 32 runs 1.74
// ms at 3 blocks (168 registers, a few spilled) against 2.34 ms at the allocator's 179 registers
// (2 blocks); n = 24 1.19 ms at 4 blocks (128 registers) against 1.24 ms. The 16-lane teams
// (n = 12, 16; factor in shared memory) run fastest unbounded (94 registers); a 32-lane team at
// n = 12 or 16 takes a minimum of one block, without which the allocator holds it to 96
// registers and spills.
template <class Fam, int T> constexpr int warp_min_blocks() {
#ifdef GSB_WARP_MIN_BLOCKS
    return GSB_WARP_MIN_BLOCKS;
#else
    return T != 32 ? 0 : Fam::N >= 32 ? 3 : Fam::N >= 24 ? 4 : 1;
#endif
}

template <class Fam, int T, bool F, bool Mixed, bool PlainRef, bool Persistent>
__global__ void __launch_bounds__(kThreads, (warp_min_blocks<Fam, T>())) warp_kernel(const __grid_constant__ GsbMethod m,
                                 const __grid_constant__ GsbOptions o,
                                 const __grid_constant__ Launch L) {
    extern __shared__ double smem[];
    constexpr int N = Fam::N, NP = Fam::NP, SS = warp_sys_stride<Fam, T>();
    constexpr int SHA = WarpSharedA<Fam>::doubles;
    const int tid = threadIdx.x;
    const int team = tid / T;
    const int spb = (int)blockDim.x / T;
    double* sys = smem + SHA + team * SS;
    if constexpr (SHA > 0) {
        // the batch's A (column-major, n x n) once per CTA, at the family's column stride
        for (int q = tid; q < N * N; q += (int)blockDim.x)
            smem[(q % N) + (q / N) * Fam::LDA] = __ldg(L.shared + q);
        __syncthreads();
    }
    const double* fam_shared = SHA > 0 ? smem : L.shared;
    for_each_chunk<Persistent>(L, spb, [&](int64_t base, const Range& r) {
        const int64_t i = base + team;
        if (r.order == nullptr && L.p_layout == GSB_AOS && L.p_off == nullptr) {
            stage_aos_rows<NP, SS>(smem + SHA, L.P + base * NP, r.n - base, spb, tid,
                                   (int)blockDim.x, WarpPlace<Fam>());
        } else if (i < r.n) {
            const int64_t idx = r.order ? r.order[i] - L.order_base : i;
            const double* pb = param_block(L, idx, NP);
            if (L.p_layout == GSB_SOA) {
                for (int k = tid % T; k < NP; k += T)
                    sys[Fam::place(k)] = __ldg(L.P + (int64_t)k * L.nsys + idx);
            } else {
                // the team's block by asynchronous 8-byte copies, all in flight at once (a
                // ragged bucket or an `order` reaches here)
                for (int k = tid % T; k < NP; k += T) {
                    const unsigned dst = smem_addr(sys + Fam::place(k));
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst), "l"(pb + k)
                                 : "memory");
                }
                asm volatile("cp.async.wait_all;" ::: "memory");
            }
        }
        __syncthreads();
        if (i >= r.n) return;
        const int64_t idx = r.order ? r.order[i] - L.order_base : i;
        Team<T> tm;
        const int lane = tm.lane;
        Fam fam{sys, fam_shared};
        double* xb = x_block(L, idx, N);
        double xl = 0.0;
        if (lane < N) xl = L.x_layout == GSB_SOA ? L.X[(int64_t)lane * L.nsys + idx] : xb[lane];
        WarpSolver<Fam, T, F, Mixed, PlainRef> sv(fam, m, o, tm, sys + ((Fam::SP + 1) / 2) * 2);
        double gr;
        DevStatus s = sv.solve(xl, gr);
        if (lane < N) {
            if (L.x_layout == GSB_SOA) L.X[(int64_t)lane * L.nsys + idx] = xl;
            else xb[lane] = xl;
        }
        if (lane == 0) {
            if (L.s_kind == GSB_STATUS64) store_status(L.S, idx, s, gr);
            else reinterpret_cast<unsigned char*>(L.S)[idx] = (unsigned char)s.code;
            if (L.tally) tally_code(L.tally, s.code);
            if (L.summary) {
                SummaryPart part;
                part.add(s);
                part.flush(L.summary);
            }
        }
    });
}

using KernelFn = void (*)(GsbMethod, GsbOptions, Launch);

struct KernelEntry {
    KernelFn fn;             // one chunk per CTA
    KernelFn fn_persistent;  // chunks from the launch's work queue
    int smem_doubles;  // dynamic shared memory of a CTA, in doubles
    int systems_per_block;
    bool attr_set[64];
    bool resident = false;  // fn works through ranges of systems: launch the resident CTAs only
    // The warp form takes its CTA size at launch: `lanes` threads and `sys_doubles` doubles of
    // shared memory per system (0: the CTA size is fixed at kThreads).
    int lanes = 0;
    int sys_doubles = 0;
};

template <class Fam, bool F, bool Mixed, bool PlainRef> KernelEntry* entry() {
    // the kernels of a family with aligned rows work warp by warp over the whole batch: launch
    // the resident CTAs only
    static KernelEntry e{newton_kernel<Fam, F, Mixed, PlainRef, false>,
                         newton_kernel<Fam, F, Mixed, PlainRef, true>,
                         ((SharedLen<Fam>::value + 1) / 2) * 2 + kThreads * newton_row_stride<Fam>(),
                         kThreads, {}, PairsOf<Fam>::value};
    return &e;
}

// The Float64 LU step with factor reuse (Kind = kStepReuse) or with the DogLeg trust region
// (kStepDogLeg), no refinement.
template <class Fam, bool F, int Kind> KernelEntry* kind_entry() {
    static KernelEntry e{newton_kernel<Fam, F, false, false, false, false, Kind>,
                         newton_kernel<Fam, F, false, false, true, false, Kind>,
                         ((SharedLen<Fam>::value + 1) / 2) * 2 + kThreads * newton_row_stride<Fam>(),
                         kThreads, {}, PairsOf<Fam>::value};
    return &e;
}

// The mixed LU step (Float32 factor, refinement as the method says) with its line-search trials
// in Float32 (kStepTrial32).
template <class Fam, bool F> KernelEntry* trial32_entry() {
    static KernelEntry e{newton_kernel<Fam, F, true, false, false, false, kStepTrial32>,
                         newton_kernel<Fam, F, true, false, true, false, kStepTrial32>,
                         ((SharedLen<Fam>::value + 1) / 2) * 2 + kThreads * newton_row_stride<Fam>(),
                         kThreads, {}, PairsOf<Fam>::value};
    return &e;
}

// The step with the static QR factor (QRFactorization): Float64 with or without the refinement
// passes (Ref), or the mixed step's Float32 factor (Mixed; refinement as the method says).
template <class Fam, bool F, bool Ref = false, bool Mixed = false> KernelEntry* qr_entry() {
    static KernelEntry e{newton_kernel<Fam, F, Mixed, Ref, false, true>,
                         newton_kernel<Fam, F, Mixed, Ref, true, true>,
                         ((SharedLen<Fam>::value + 1) / 2) * 2 + kThreads * newton_row_stride<Fam>(),
                         kThreads, {}};
    return &e;
}

template <class Fam, bool F, bool Mixed> KernelEntry* lm_entry() {
    constexpr int RS = (Fam::M % 2 == 1) ? Fam::M : Fam::M + 1;
    static KernelEntry e{lm_kernel<Fam, F, Mixed>, nullptr, kThreads * RS + Fam::M, kThreads, {}, true};
    return &e;
}

template <class Fam, int T, bool F, bool Mixed, bool PlainRef> KernelEntry* warp_entry() {
    // (a batch-wide A, staged at the CTA's start, is a per-call form: the ragged batch, which
    // sizes CTAs by sys_doubles, has per-system blocks only)
    static KernelEntry e{warp_kernel<Fam, T, F, Mixed, PlainRef, false>,
                         warp_kernel<Fam, T, F, Mixed, PlainRef, true>,
                         WarpSharedA<Fam>::doubles + (kThreads / T) * warp_sys_stride<Fam, T>(),
                         kThreads / T, {}, false, T, warp_sys_stride<Fam, T>()};
    return &e;
}

// The six warp-form kernels of a family at team size T.
template <class Fam, int T> KernelEntry* pick_warp(bool fused, bool mixed, bool refine) {
    if (fused) {
        if (mixed) return warp_entry<Fam, T, true, true, false>();
        return refine ? warp_entry<Fam, T, true, false, true>() : warp_entry<Fam, T, true, false, false>();
    }
    if (mixed) return warp_entry<Fam, T, false, true, false>();
    return refine ? warp_entry<Fam, T, false, false, true>() : warp_entry<Fam, T, false, false, false>();
}

template <class Fam, int T, bool Mixed> KernelEntry* team_entry() {
    constexpr int RS = (Fam::NP % 2 == 1) ? Fam::NP : Fam::NP + 1;
    static KernelEntry e{team_kernel<Fam, T, Mixed, false>, team_kernel<Fam, T, Mixed, true>,
                         (kThreads / T) * RS, kThreads / T, {}};
    return &e;
}

template <class Fam, int T> KernelEntry* pick_team(bool mixed) {
    return mixed ? team_entry<Fam, T, true>() : team_entry<Fam, T, false>();
}

// The six kernels of a family: arithmetic fused or unfused; factor Float32, or Float64 with or
// without refinement.
template <class Fam> KernelEntry* pick(bool fused, bool mixed, bool refine) {
    if (fused) {
        if (mixed) return entry<Fam, true, true, false>();
        return refine ? entry<Fam, true, false, true>() : entry<Fam, true, false, false>();
    }
    if (mixed) return entry<Fam, false, true, false>();
    return refine ? entry<Fam, false, false, true>() : entry<Fam, false, false, false>();
}

#define GSB_DECLARE_ENTRY(NAME) KernelEntry* entry_##NAME(bool fused, bool mixed, bool refine)
#define GSB_DECLARE_QR(NAME) KernelEntry* qr_##NAME(bool fused, bool refine, bool mixed)
#define GSB_DEFINE_QR(NAME, ...)                                                              \
    KernelEntry* qr_##NAME(bool fused, bool refine, bool mixed) {                             \
        if (mixed)                                                                            \
            return fused ? qr_entry<__VA_ARGS__, true, false, true>()                         \
                         : qr_entry<__VA_ARGS__, false, false, true>();                       \
        if (refine)                                                                           \
            return fused ? qr_entry<__VA_ARGS__, true, true>() : qr_entry<__VA_ARGS__, false, true>(); \
        return fused ? qr_entry<__VA_ARGS__, true>() : qr_entry<__VA_ARGS__, false>();        \
    }
#define GSB_DECLARE_TEAM(NAME) KernelEntry* team_##NAME(int T, bool mixed)
#define GSB_DECLARE_TRIAL32(NAME) KernelEntry* trial32_##NAME(bool fused)
#define GSB_DEFINE_TRIAL32(NAME, ...)                                                         \
    KernelEntry* trial32_##NAME(bool fused) {                                                 \
        return fused ? trial32_entry<__VA_ARGS__, true>() : trial32_entry<__VA_ARGS__, false>(); \
    }
#define GSB_DECLARE_KIND(NAME) KernelEntry* kind_##NAME(bool fused, int kind)
#define GSB_DEFINE_KIND(NAME, ...)                                                            \
    KernelEntry* kind_##NAME(bool fused, int kind) {                                          \
        if (kind == kStepReuse)                                                               \
            return fused ? kind_entry<__VA_ARGS__, true, kStepReuse>()                        \
                         : kind_entry<__VA_ARGS__, false, kStepReuse>();                      \
        return fused ? kind_entry<__VA_ARGS__, true, kStepDogLeg>()                           \
                     : kind_entry<__VA_ARGS__, false, kStepDogLeg>();                         \
    }
#define GSB_DEFINE_ENTRY(NAME, ...)                                          \
    KernelEntry* entry_##NAME(bool fused, bool mixed, bool refine) {         \
        return pick<__VA_ARGS__>(fused, mixed, refine);                      \
    }

}  // namespace gsb
