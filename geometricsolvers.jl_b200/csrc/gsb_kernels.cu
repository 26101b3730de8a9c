// libgsb: the batch kernels and the C-ABI of include/gsb.h.
//
// One launch solves a batch: one thread per system (the work item of the reference's
// `_solve_kernel!`, src/nonlinear/batched.jl:171-179). A CTA first stages the parameter blocks
// of its systems into shared memory (coalesced loads of the CTA's contiguous AoS chunk, or one
// coalesced load per entry for SoA), each system's block in a row of odd stride so that the
// per-thread reads are free of bank conflicts; then each thread runs its solve in registers and
// writes its iterate and its 72-byte status.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gsb.h"
#include "gsb_kernel_impl.cuh"

namespace gsb {


__global__ void summary_kernel(const unsigned char* S, int64_t nsys, SummaryAcc* acc, int scale_e,
                               int pass) {
    double sq = 0.0;
    unsigned long long mb = 0, fails = 0, tot = 0;
    int mx = 0, nan = 0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nsys;
         q += (int64_t)gridDim.x * blockDim.x) {
        const unsigned char* st = S + q * 72;
        int code = st[0];
        int it = *reinterpret_cast<const int*>(st + 4);
        double fn = *reinterpret_cast<const double*>(st + 8);
        if (pass == 0) {
            sq = __fma_rn(fn, fn, sq);
            unsigned long long b = (unsigned long long)__double_as_longlong(fabs(fn));
            if (fn != fn) nan = 1;
            mb = b > mb ? b : mb;
            fails += code != SUCCESS;
            tot += (unsigned long long)it;
            mx = it > mx ? it : mx;
        } else {
            double u = ldexp2(fn, -scale_e);
            sq = __fma_rn(u, u, sq);
        }
    }
    for (int off = 16; off; off >>= 1) {
        sq += __shfl_xor_sync(0xffffffffu, sq, off);
        unsigned long long ob = __shfl_xor_sync(0xffffffffu, mb, off);
        mb = ob > mb ? ob : mb;
        fails += __shfl_xor_sync(0xffffffffu, fails, off);
        tot += __shfl_xor_sync(0xffffffffu, tot, off);
        int om = __shfl_xor_sync(0xffffffffu, mx, off);
        mx = om > mx ? om : mx;
        nan |= __shfl_xor_sync(0xffffffffu, nan, off);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(&acc->sumsq, sq);
        if (pass == 0) {
            atomicMax(&acc->maxbits, mb);
            atomicAdd(&acc->failures, fails);
            atomicAdd(&acc->total_iterations, tot);
            atomicMax(&acc->max_iterations, mx);
            atomicOr(&acc->nan_seen, nan);
        }
    }
}


// ─── the working memory of gsb_solve_batch_counts_noalloc ─────────────────────────────────
// One static array per device that loads the library: words 0..5 are the six counters of the
// count form, word 6 the error flags of the `order` check (1: an entry out of range, 2: an
// entry seen twice), word 7 unused, and the rest one bit per system for that check.
constexpr int kNoallocHead = 8;
constexpr int64_t kNoallocBitmapWords = (int64_t)GSB_NOALLOC_MAX_ORDERED / 64;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoallocHead + kNoallocBitmapWords];

// Clears the counters, the flags and the first `words` bitmap words.
__global__ void noalloc_clear(unsigned long long* scratch, int64_t words) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < kNoallocHead + words;
         q += (int64_t)gridDim.x * blockDim.x)
        scratch[q] = 0ull;
}

// Marks each entry of `order` in the bitmap and flags out-of-range and repeated entries.
__global__ void noalloc_check_order(const int64_t* order, int order_base, int64_t nsys,
                                    unsigned long long* scratch) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nsys;
         q += (int64_t)gridDim.x * blockDim.x) {
        int64_t v = order[q] - order_base;
        if (v < 0 || v >= nsys) {
            atomicOr(scratch + 6, 1ull);
            continue;
        }
        unsigned long long bit = 1ull << (v & 63);
        unsigned long long old = atomicOr(scratch + kNoallocHead + (v >> 6), bit);
        if (old & bit) atomicOr(scratch + 6, 2ull);
    }
}
}  // namespace gsb

using namespace gsb;

// The structs that cross the boundary have the layouts of the reference's types.
#include <cstddef>
static_assert(sizeof(GsbStatus64) == 72 && offsetof(GsbStatus64, fnorm) == 8 &&
                  offsetof(GsbStatus64, step_failures) == 24 && offsetof(GsbStatus64, rank) == 32 &&
                  offsetof(GsbStatus64, gradratio) == 48 && offsetof(GsbStatus64, reused) == 65,
              "GsbStatus64 is SolverStatus{Float64}");
static_assert(sizeof(GsbSummary) == 40 && offsetof(GsbSummary, all_converged) == 8 &&
                  offsetof(GsbSummary, failure_count) == 16 &&
                  offsetof(GsbSummary, max_iterations) == 24 &&
                  offsetof(GsbSummary, total_iterations) == 32,
              "GsbSummary is BatchSummary{Float64}");

// ─── host side ──────────────────────────────────────────────────────────────────────────────

namespace {

thread_local std::string g_err;

int set_err(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

int cuda_err(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return 0;
    return set_err(GSB_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// Per-device workspace: the tally counters and the summary accumulator.
struct Workspace {
    unsigned long long* tally = nullptr;
    SummaryAcc* acc = nullptr;
};
std::mutex g_ws_mu;
Workspace g_ws[64];

int workspace(Workspace** out) {
    int dev = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (dev < 0 || dev >= 64) return set_err(GSB_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_ws_mu);
    Workspace& w = g_ws[dev];
    if (!w.tally) {
        if (int rc = cuda_err(cudaMalloc(&w.tally, 6 * sizeof(unsigned long long)), "cudaMalloc"))
            return rc;
        if (int rc = cuda_err(cudaMalloc(&w.acc, sizeof(SummaryAcc)), "cudaMalloc")) return rc;
    }
    *out = &w;
    return 0;
}

// A word of mapped pinned host memory that a batch kernel sets when one of its staging waits
// ran out (its systems then stay unsolved): allocated once per process, read by the host after a
// synchronisation without a copy. nullptr when the allocation failed (no word is then set).
std::mutex g_fault_mu;
unsigned* g_fault = nullptr;
bool g_fault_tried = false;

unsigned* fault_word() {
    std::lock_guard<std::mutex> lk(g_fault_mu);
    if (!g_fault_tried) {
        g_fault_tried = true;
        void* h = nullptr;
        if (cudaHostAlloc(&h, sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable) ==
            cudaSuccess) {
            *static_cast<volatile unsigned*>(h) = 0u;
            g_fault = static_cast<unsigned*>(h);
        } else {
            cudaGetLastError();  // the failed allocation's error is not the caller's
        }
    }
    return g_fault;
}

// After a synchronisation: an error if a kernel reported a staging wait that ran out.
int check_fault() {
    if (g_fault && *reinterpret_cast<volatile unsigned*>(g_fault) != 0u) {
        *reinterpret_cast<volatile unsigned*>(g_fault) = 0u;
        return set_err(GSB_ERR_CUDA,
                       "a batch kernel's wait for its staging copies ran out; systems of that "
                       "launch were left unsolved");
    }
    return 0;
}

// The cubic family's BatchParams form: the batch's matrix A in prob->shared (n^2 doubles).
bool shared_matrix(const GsbProblem* p) {
    return p->family == GSB_FAMILY_CUBIC_AFFINE && p->shared && p->shared_len == (int64_t)p->n * p->n;
}

int64_t param_count(const GsbProblem* p) {
    switch (p->family) {
    case GSB_FAMILY_CUBIC_AFFINE:
        if (!(p->n >= 1 && p->n <= 32)) return GSB_ERR_ARGUMENT;
        // with A shared by the batch (shared_len = n^2), a system's block is b alone
        return shared_matrix(p) ? (int64_t)p->n : (int64_t)p->n * p->n + p->n;
    case GSB_FAMILY_EXPSUM3_LSQ: return p->m;
    case GSB_FAMILY_IRK3_HENON_HEILES: return 4;
    case GSB_FAMILY_HETERO6: return 1;
    case GSB_FAMILY_COUPLED2: return 2;
    case GSB_FAMILY_WOOD: return p->n == 4 ? 1 : GSB_ERR_ARGUMENT;
    case GSB_FAMILY_CUBIC_AFFINE_DUAL:
        return (p->n >= 2 && p->n <= 4) ? (int64_t)p->n * p->n + p->n : GSB_ERR_ARGUMENT;
    default: return GSB_ERR_ARGUMENT;
    }
}

}  // namespace

namespace gsb {
GSB_DECLARE_ENTRY(cubic2);
GSB_DECLARE_ENTRY(cubic3);
GSB_DECLARE_ENTRY(cubic4);
GSB_DECLARE_ENTRY(cubic6);
GSB_DECLARE_ENTRY(cubic8);
GSB_DECLARE_QR(cubic2);
GSB_DECLARE_QR(cubic3);
GSB_DECLARE_QR(cubic4);
GSB_DECLARE_QR(cubic6);
GSB_DECLARE_QR(cubic8);
GSB_DECLARE_QR(hetero6);
GSB_DECLARE_QR(coupled2);
GSB_DECLARE_ENTRY(cubic2s);
GSB_DECLARE_ENTRY(cubic3s);
GSB_DECLARE_ENTRY(cubic4s);
GSB_DECLARE_ENTRY(cubic6s);
GSB_DECLARE_ENTRY(cubic8s);
GSB_DECLARE_ENTRY(hetero6);
GSB_DECLARE_ENTRY(coupled2);
GSB_DECLARE_ENTRY(wood);
GSB_DECLARE_ENTRY(cubicdual2);
GSB_DECLARE_ENTRY(cubicdual3);
GSB_DECLARE_ENTRY(cubicdual4);
GSB_DECLARE_TEAM(cubic6);
GSB_DECLARE_TEAM(cubic8);
GSB_DECLARE_KIND(cubic2);
GSB_DECLARE_KIND(cubic3);
GSB_DECLARE_KIND(cubic4);
GSB_DECLARE_KIND(cubic6);
GSB_DECLARE_KIND(cubic8);
GSB_DECLARE_KIND(hetero6);
GSB_DECLARE_KIND(coupled2);
GSB_DECLARE_TRIAL32(cubic2);
GSB_DECLARE_TRIAL32(cubic3);
GSB_DECLARE_TRIAL32(cubic4);
GSB_DECLARE_TRIAL32(cubic6);
GSB_DECLARE_TRIAL32(cubic8);
KernelEntry* lm_expsum3_64(bool fused, bool mixed);
KernelEntry* warp_cubic12(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic16(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic24(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic32(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic12s(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic16s(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic24s(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_cubic32s(bool fused, bool mixed, bool refine, int T);
KernelEntry* warp_irk(bool fused, bool mixed, bool refine, int T);
}  // namespace gsb

namespace {

// The tuned lanes per system of a family and size. Measured on B200 (1,048,576 systems of the
// cubic family, ms per batch, plain / FP32-factor): n = 6: T=1 1.12 / 1.39, T=2 2.16 / 2.85;
// n = 8: T=1 1.78 / 2.39, T=2 3.03 / 3.99, T=4 4.21 / 5.81, T=8 4.60 / 6.67. One lane per system
// wins wherever its factor fits in registers.
int tuned_team(const GsbProblem* prob, bool mixed) {
    (void)prob;
    (void)mixed;
    return 1;
}

// The kernel of a QRFactorization call: the one-thread step with the static QR factor (Float64
// with or without the refinement passes, or the mixed step's Float32 factor), for the square
// families with per-system parameter blocks.
KernelEntry* select_qr_kernel(const GsbProblem* prob, bool fused, bool refine, bool mixed, int T) {
    if (T > 1 || shared_matrix(prob)) return nullptr;
    switch (prob->family) {
    case GSB_FAMILY_CUBIC_AFFINE:
        switch (prob->n) {
        case 2: return qr_cubic2(fused, refine, mixed);
        case 3: return qr_cubic3(fused, refine, mixed);
        case 4: return qr_cubic4(fused, refine, mixed);
        case 6: return qr_cubic6(fused, refine, mixed);
        case 8: return qr_cubic8(fused, refine, mixed);
        default: return nullptr;
        }
    case GSB_FAMILY_HETERO6: return qr_hetero6(fused, refine, mixed);
    case GSB_FAMILY_COUPLED2: return qr_coupled2(fused, refine, mixed);
    default: return nullptr;
    }
}

// The kernel of a step with factor reuse or with DogLeg: one thread per system, a Float64 LU
// factor, no refinement, a per-system parameter block.
KernelEntry* select_kind_kernel(const GsbProblem* prob, bool fused, int kind, int T) {
    if (T > 1 || shared_matrix(prob)) return nullptr;
    switch (prob->family) {
    case GSB_FAMILY_CUBIC_AFFINE:
        switch (prob->n) {
        case 2: return kind_cubic2(fused, kind);
        case 3: return kind_cubic3(fused, kind);
        case 4: return kind_cubic4(fused, kind);
        case 6: return kind_cubic6(fused, kind);
        case 8: return kind_cubic8(fused, kind);
        default: return nullptr;
        }
    case GSB_FAMILY_HETERO6: return kind_hetero6(fused, kind);
    case GSB_FAMILY_COUPLED2: return kind_coupled2(fused, kind);
    default: return nullptr;
    }
}

// The kernel of the mixed step whose line-search trials run in Float32: one thread per system,
// the cubic-affine family, a per-system parameter block.
KernelEntry* select_trial32_kernel(const GsbProblem* prob, bool fused, int T) {
    if (T > 1 || shared_matrix(prob) || prob->family != GSB_FAMILY_CUBIC_AFFINE) return nullptr;
    switch (prob->n) {
    case 2: return trial32_cubic2(fused);
    case 3: return trial32_cubic3(fused);
    case 4: return trial32_cubic4(fused);
    case 6: return trial32_cubic6(fused);
    case 8: return trial32_cubic8(fused);
    default: return nullptr;
    }
}

// The kernel of a call: the one-thread solve for T = 1, else the team solve (fused only).
KernelEntry* select_kernel(const GsbProblem* prob, bool fused, bool mixed, bool refine, int T) {
    if (shared_matrix(prob)) {
        // BatchParams: A shared by the batch and staged once per CTA, b per system; one thread
        // per system up to n = 8, the warp form above (the team form reads a whole (A, b)
        // block per system)
        if (prob->n >= 12) {
            if (T == 0) T = prob->n <= 16 ? 16 : 32;
            if (!(T == 32 || (T == 16 && prob->n <= 16))) return nullptr;
            switch (prob->n) {
            case 12: return warp_cubic12s(fused, mixed, refine, T);
            case 16: return warp_cubic16s(fused, mixed, refine, T);
            case 24: return warp_cubic24s(fused, mixed, refine, T);
            case 32: return warp_cubic32s(fused, mixed, refine, T);
            default: return nullptr;
            }
        }
        if (T > 1) return nullptr;
        switch (prob->n) {
        case 2: return entry_cubic2s(fused, mixed, refine);
        case 3: return entry_cubic3s(fused, mixed, refine);
        case 4: return entry_cubic4s(fused, mixed, refine);
        case 6: return entry_cubic6s(fused, mixed, refine);
        case 8: return entry_cubic8s(fused, mixed, refine);
        default: return nullptr;
        }
    }
    if (prob->family == GSB_FAMILY_CUBIC_AFFINE && prob->n >= 12) {
        // the warp form: 16 lanes per system up to n = 16 (or a whole warp), a whole warp above
        if (T == 0) T = prob->n <= 16 ? 16 : 32;
        if (!(T == 32 || (T == 16 && prob->n <= 16))) return nullptr;
        switch (prob->n) {
        case 12: return warp_cubic12(fused, mixed, refine, T);
        case 16: return warp_cubic16(fused, mixed, refine, T);
        case 24: return warp_cubic24(fused, mixed, refine, T);
        case 32: return warp_cubic32(fused, mixed, refine, T);
        default: return nullptr;
        }
    }
    if (prob->family == GSB_FAMILY_IRK3_HENON_HEILES) {
        if (T == 0) T = 16;
        return (T == 16 || T == 32) ? warp_irk(fused, mixed, refine, T) : nullptr;
    }
    if (T == 0) T = fused ? tuned_team(prob, mixed) : 1;
    if (T != 1) {
        if (!fused || prob->family != GSB_FAMILY_CUBIC_AFFINE) return nullptr;
        switch (prob->n) {
        case 6: return team_cubic6(T, mixed);
        case 8: return team_cubic8(T, mixed);
        default: return nullptr;
        }
    }
    switch (prob->family) {
    case GSB_FAMILY_CUBIC_AFFINE:
        switch (prob->n) {
        case 2: return entry_cubic2(fused, mixed, refine);
        case 3: return entry_cubic3(fused, mixed, refine);
        case 4: return entry_cubic4(fused, mixed, refine);
        case 6: return entry_cubic6(fused, mixed, refine);
        case 8: return entry_cubic8(fused, mixed, refine);
        default: return nullptr;
        }
    case GSB_FAMILY_HETERO6: return entry_hetero6(fused, mixed, refine);
    case GSB_FAMILY_COUPLED2: return entry_coupled2(fused, mixed, refine);
    case GSB_FAMILY_WOOD: return entry_wood(fused, mixed, refine);
    case GSB_FAMILY_CUBIC_AFFINE_DUAL:
        switch (prob->n) {
        case 2: return entry_cubicdual2(fused, mixed, refine);
        case 3: return entry_cubicdual3(fused, mixed, refine);
        case 4: return entry_cubicdual4(fused, mixed, refine);
        default: return nullptr;
        }
    default: return nullptr;
    }
}

bool nonneg(double v) { return v >= 0.0; }

int check_options(const GsbOptions* o) {
    if (!(nonneg(o->f_abstol) && nonneg(o->f_reltol) && nonneg(o->x_abstol) &&
          nonneg(o->x_reltol) && nonneg(o->g_tol)))
        return set_err(GSB_ERR_ARGUMENT, "tolerances must be non-negative");
    if (o->min_iterations < 0) return set_err(GSB_ERR_ARGUMENT, "min_iterations must be non-negative");
    if (o->max_iterations < o->min_iterations)
        return set_err(GSB_ERR_ARGUMENT, "max_iterations is below min_iterations");
    if (o->max_stalls < 1) return set_err(GSB_ERR_ARGUMENT, "max_stalls must be at least 1");
    if (!(o->kappa > 0.0 && o->kappa < 1.0))
        return set_err(GSB_ERR_ARGUMENT, "kappa must be finite and in (0, 1)");
    if (o->norm != 0 && o->norm != 1) return set_err(GSB_ERR_ARGUMENT, "norm must be L2 or Max");
    return 0;
}

int check_method(const GsbMethod* m) {
    if (m->linsolve != GSB_LU && m->linsolve != GSB_QR)
        return set_err(GSB_ERR_ARGUMENT, "linsolve must be LU or QR");
    if (m->factor_precision != GSB_F64 && m->factor_precision != GSB_F32)
        return set_err(GSB_ERR_ARGUMENT, "factor precision must be F64 or F32");
    if (m->globalization < GSB_STATIC || m->globalization > GSB_DOGLEG)
        return set_err(GSB_ERR_ARGUMENT, "unknown globalization");
    if (m->reuse < 0) return set_err(GSB_ERR_ARGUMENT, "Newton reuse must be >= 1 or nothing (0)");
    if (m->reuse > 0 && m->globalization == GSB_LEVENBERG_MARQUARDT)
        return set_err(GSB_ERR_ARGUMENT,
                       "Newton with a LevenbergMarquardt globalization takes no reuse");
    if (m->reuse > 0 && m->globalization == GSB_DOGLEG)
        return set_err(GSB_ERR_ARGUMENT, "DogLeg takes no factor reuse");
    if (!(m->dogleg_radius >= 0.0 && isfinite(m->dogleg_radius)))
        return set_err(GSB_ERR_ARGUMENT, "the radius of DogLeg must be positive and finite");
    if (m->globalization == GSB_STATIC && !(m->static_alpha > 0.0 && isfinite(m->static_alpha)))
        return set_err(GSB_ERR_ARGUMENT, "the step of Static must be positive and finite");
    if (m->globalization == GSB_BACKTRACKING &&
        !(m->bt_c1 > 0 && m->bt_c1 < 1 && m->bt_p > 0 && m->bt_p < 1 && m->bt_maxiter >= 1))
        return set_err(GSB_ERR_ARGUMENT, "Backtracking needs 0 < c1 < 1, 0 < p < 1, maxiter >= 1");
    if (m->refinement == GSB_REFINEMENT &&
        !(m->refine_maxiter >= 1 && m->refine_eta > 0 && m->refine_eta < 1))
        return set_err(GSB_ERR_ARGUMENT, "Refinement needs maxiter >= 1 and 0 < eta < 1");
    if (m->globalization == GSB_LEVENBERG_MARQUARDT && m->refinement == GSB_REFINEMENT)
        return set_err(GSB_ERR_UNSUPPORTED,
                       "Newton with a LevenbergMarquardt globalization takes no refinement");
    if (m->regularization != 0.0)
        return set_err(GSB_ERR_UNSUPPORTED, "the batch path takes regularization = 0");
    if (m->arithmetic != GSB_FUSED && m->arithmetic != GSB_UNFUSED)
        return set_err(GSB_ERR_ARGUMENT, "arithmetic must be GSB_FUSED or GSB_UNFUSED");
    {
        const int t = m->threads_per_system;
        if (!(t == 0 || t == 1 || t == 2 || t == 4 || t == 8 || t == 16 || t == 32))
            return set_err(GSB_ERR_ARGUMENT, "threads_per_system must be 0, 1, 2, 4, 8, 16 or 32");
    }
    if (m->trial_precision != GSB_F64 && m->trial_precision != GSB_F32)
        return set_err(GSB_ERR_ARGUMENT, "trial precision must be F64 or F32");
    if (m->trial_precision == GSB_F32 &&
        !(m->linsolve == GSB_LU && m->factor_precision == GSB_F32 && m->reuse == 0 &&
          (m->globalization == GSB_BACKTRACKING || m->globalization == GSB_STATIC)))
        return set_err(GSB_ERR_UNSUPPORTED,
                       "Float32 line-search trials go with a Float32 LUFactorization, no reuse, "
                       "and Backtracking or Static");
    return 0;
}


// The device address of g_noalloc_scratch on the current device, looked up once per device (a
// host-side name of a __device__ array is not a device address). No allocation.
std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_ptr[64] = {};

int noalloc_scratch(unsigned long long** out) {
    int dev = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (dev < 0 || dev >= 64) return set_err(GSB_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        unsigned long long* p = nullptr;
        if (int rc = cuda_err(cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_noalloc_scratch),
                              "cudaGetSymbolAddress"))
            return rc;
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

// Pick the kernel for the call and launch it on `st` (arguments already checked).
// The kernel of a call (family, size, method): the least-squares family's LevenbergMarquardt
// kernel, the QRFactorization kernel, or the LU kernels of select_kernel. An error (and no
// kernel) for a combination without one.
int select_entry(const GsbProblem* prob, const GsbMethod* method, KernelEntry** out) {
    const bool mixed = method->factor_precision == GSB_F32;
    const bool fused = method->arithmetic == GSB_FUSED;
    const bool lm = method->globalization == GSB_LEVENBERG_MARQUARDT;
    KernelEntry* ke = nullptr;
    if (prob->family == GSB_FAMILY_EXPSUM3_LSQ) {
        // the least-squares family: the LevenbergMarquardt step on its stacked QR path
        if (!lm)
            return set_err(GSB_ERR_UNSUPPORTED,
                           "the least-squares batch kernel runs the LevenbergMarquardt step");
        if (method->refinement == GSB_REFINEMENT)
            return set_err(GSB_ERR_UNSUPPORTED,
                           "Newton with a LevenbergMarquardt globalization takes no refinement");
        if (method->threads_per_system > 1)
            return set_err(GSB_ERR_UNSUPPORTED, "one thread per least-squares system");
        if (prob->m != 64) return set_err(GSB_ERR_UNSUPPORTED, "no batch kernel for this m");
        if (!prob->shared) return set_err(GSB_ERR_ARGUMENT, "the abscissae t are missing");
        ke = lm_expsum3_64(fused, mixed);
    } else {
        if (lm)
            return set_err(GSB_ERR_UNSUPPORTED,
                           "LevenbergMarquardt batch kernel only for least-squares families");
        if (method->trial_precision == GSB_F32) {
            // the mixed step with Float32 line-search trials (checked by check_method)
            ke = select_trial32_kernel(prob, fused, method->threads_per_system);
        } else if (method->reuse > 0 || method->globalization == GSB_DOGLEG) {
            // factor reuse and DogLeg: the Float64 LU step without refinement
            if (method->linsolve != GSB_LU || mixed || method->refinement == GSB_REFINEMENT)
                return set_err(GSB_ERR_UNSUPPORTED,
                               "the batch kernels with factor reuse or DogLeg take a Float64 "
                               "LUFactorization and no refinement");
            ke = select_kind_kernel(prob, fused,
                                    method->reuse > 0 ? gsb::kStepReuse : gsb::kStepDogLeg,
                                    method->threads_per_system);
        } else if (method->linsolve == GSB_QR) {
            ke = select_qr_kernel(prob, fused, method->refinement == GSB_REFINEMENT, mixed,
                                  method->threads_per_system);
        } else {
            if (prob->family == GSB_FAMILY_IRK3_HENON_HEILES && !prob->shared)
                return set_err(GSB_ERR_ARGUMENT, "the step h and the tableau A are missing");
            ke = select_kernel(prob, fused, mixed, method->refinement == GSB_REFINEMENT,
                               method->threads_per_system);
        }
    }
    if (!ke) return set_err(GSB_ERR_UNSUPPORTED, "no batch kernel for this family and size");
    *out = ke;
    return 0;
}

// The grid of a launch: one CTA per kernel-sized chunk of systems, or, for a kernel that works
// through ranges of systems, at most the CTAs that are resident on the device at once.
int launch_blocks(const KernelEntry* ke, int64_t nsys, size_t smem, int64_t* blocks) {
    *blocks = (nsys + ke->systems_per_block - 1) / ke->systems_per_block;
    if (!ke->resident) return 0;
    int dev = 0, sms = 0, occ = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (int rc = cuda_err(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                          "cudaDeviceGetAttribute"))
        return rc;
    if (int rc = cuda_err(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                              &occ, reinterpret_cast<const void*>(ke->fn), kThreads, smem),
                          "cudaOccupancyMaxActiveBlocksPerMultiprocessor"))
        return rc;
    const int64_t cap = (int64_t)(sms > 0 ? sms : 1) * (occ > 0 ? occ : 1);
    if (*blocks > cap) *blocks = cap;
    return 0;
}

int launch_solve(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt, double* X,
                 int32_t x_layout, void* S, int32_t s_kind, const double* P, int32_t p_layout,
                 const int64_t* order, int32_t order_base, int64_t nsys, cudaStream_t st,
                 unsigned long long* tally_dev, unsigned* fault) {
    KernelEntry* ke = nullptr;
    if (int rc = select_entry(prob, method, &ke)) return rc;
    int dev = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    size_t smem = (size_t)ke->smem_doubles * sizeof(double);
    if (!ke->attr_set[dev & 63]) {
        if (int rc = cuda_err(cudaFuncSetAttribute(reinterpret_cast<const void*>(ke->fn),
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem),
                              "cudaFuncSetAttribute"))
            return rc;
        ke->attr_set[dev & 63] = true;
    }
    Launch L{X, x_layout, S, s_kind, P, p_layout, order, order_base, nsys, prob->shared, tally_dev};
    L.fault = fault;
    int64_t blocks = 0;
    if (int rc = launch_blocks(ke, nsys, smem, &blocks)) return rc;
    ke->fn<<<(unsigned)blocks, kThreads, smem, st>>>(*method, *opt, L);
    return cuda_err(cudaGetLastError(), "kernel launch");
}

// The argument checks of gsb_solve_batch, for the entry point that allocates nothing.
int check_call(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
               int64_t nsys, int32_t x_layout, int32_t p_layout, int32_t order_base) {
    if (!prob || !method || !opt) return set_err(GSB_ERR_ARGUMENT, "null problem, method or options");
    if (nsys < 0) return set_err(GSB_ERR_DIMENSION, "negative batch length");
    if (int rc = check_options(opt)) return rc;
    if (int rc = check_method(method)) return rc;
    if (param_count(prob) < 0) return set_err(GSB_ERR_ARGUMENT, "unknown family or size");
    if (x_layout != GSB_AOS && x_layout != GSB_SOA) return set_err(GSB_ERR_ARGUMENT, "x_layout");
    if (p_layout != GSB_AOS && p_layout != GSB_SOA) return set_err(GSB_ERR_ARGUMENT, "p_layout");
    if (order_base != 0 && order_base != 1) return set_err(GSB_ERR_ARGUMENT, "order_base");
    return 0;
}

}  // namespace

extern "C" {

int gsb_abi_version(void) { return GSB_ABI_VERSION; }

const char* gsb_last_error(void) { return g_err.c_str(); }

int64_t gsb_param_count(const GsbProblem* prob) {
    if (!prob) return GSB_ERR_ARGUMENT;
    return param_count(prob);
}

void gsb_default_options(GsbOptions* o) {
    std::memset(o, 0, sizeof(*o));
    o->f_abstol = 0.0;
    o->f_reltol = 1.4901161193847656e-08;
    o->x_abstol = 0.0;
    o->x_reltol = 2.0 * 2.220446049250313e-16;
    o->min_iterations = 0;
    o->max_iterations = 100;
    o->max_stalls = 2;
    o->norm = 0;
    o->g_tol = 1.4901161193847656e-08;
    o->kappa = 0.1;
    o->roundoff = 0;
    o->rate_test = 1;
}

void gsb_default_method(GsbMethod* m) {
    std::memset(m, 0, sizeof(*m));
    m->linsolve = GSB_LU;
    m->factor_precision = GSB_F64;
    m->refinement = GSB_NO_REFINEMENT;
    m->refine_maxiter = 5;
    m->refine_eta = 1.4901161193847656e-08;
    m->globalization = GSB_BACKTRACKING;
    m->bt_maxiter = 100;
    m->static_alpha = 1.0;
    m->bt_c1 = 1e-4;
    m->bt_p = 0.5;
    m->lm_mu0 = 1e-6;
    m->lm_mu_min = 1e-15;
    m->lm_mu_max = 1e12;
    m->lm_mu_decrease = 1.0 / 3.0;
    m->lm_mu_increase = 4.0;
    m->lm_rho_accept = 0.0;
    m->regularization = 0.0;
    m->arithmetic = GSB_FUSED;
    m->threads_per_system = 0;
}

// gsb_solve_batch, and with `acc` (device memory, zeroed) the batch summary of the statuses
// accumulated as the kernel closes them.
int solve_batch_impl(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
                     double* X, int32_t x_layout, void* S, int32_t s_kind, const double* P,
                     int32_t p_layout, const int64_t* order, int32_t order_base, int64_t nsys,
                     void* stream, GsbTally* tally, SummaryAcc* acc) {
    if (!prob || !method || !opt) return set_err(GSB_ERR_ARGUMENT, "null problem, method or options");
    if (nsys < 0) return set_err(GSB_ERR_DIMENSION, "negative batch length");
    if (int rc = check_options(opt)) return rc;
    if (int rc = check_method(method)) return rc;
    int64_t np = param_count(prob);
    if (np < 0) return set_err(GSB_ERR_ARGUMENT, "unknown family or size");
    if (x_layout != GSB_AOS && x_layout != GSB_SOA) return set_err(GSB_ERR_ARGUMENT, "x_layout");
    if (p_layout != GSB_AOS && p_layout != GSB_SOA) return set_err(GSB_ERR_ARGUMENT, "p_layout");
    if (s_kind != GSB_STATUS64 && s_kind != GSB_CODES) return set_err(GSB_ERR_ARGUMENT, "s_kind");
    if (order_base != 0 && order_base != 1) return set_err(GSB_ERR_ARGUMENT, "order_base");
    if (tally) std::memset(tally, 0, sizeof(*tally));
    if (nsys == 0) return 0;
    if (!X || !S || !P) return set_err(GSB_ERR_ARGUMENT, "null X, S or P");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (order) {
        // isperm, as the reference checks on the host (src/nonlinear/batched.jl:134-136)
        std::vector<int64_t> h(nsys);
        if (int rc = cuda_err(cudaMemcpyAsync(h.data(), order, nsys * sizeof(int64_t),
                                              cudaMemcpyDeviceToHost, st), "order copy"))
            return rc;
        if (int rc = cuda_err(cudaStreamSynchronize(st), "order copy")) return rc;
        std::vector<char> seen(nsys, 0);
        for (int64_t q = 0; q < nsys; ++q) {
            int64_t v = h[q] - order_base;
            if (v < 0 || v >= nsys || seen[v])
                return set_err(GSB_ERR_ARGUMENT, "order is not a permutation of the batch");
            seen[v] = 1;
        }
    }
    KernelEntry* ke = nullptr;
    if (int rc = select_entry(prob, method, &ke)) return rc;
    Workspace* ws = nullptr;
    if (tally) {
        if (int rc = workspace(&ws)) return rc;
        if (int rc = cuda_err(cudaMemsetAsync(ws->tally, 0, 6 * sizeof(unsigned long long), st),
                              "cudaMemsetAsync"))
            return rc;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    size_t smem = (size_t)ke->smem_doubles * sizeof(double);
    if (!ke->attr_set[dev & 63]) {
        if (int rc = cuda_err(cudaFuncSetAttribute(reinterpret_cast<const void*>(ke->fn),
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem),
                              "cudaFuncSetAttribute"))
            return rc;
        ke->attr_set[dev & 63] = true;
    }
    Launch L{X, x_layout, S, s_kind, P, p_layout, order, order_base, nsys, prob->shared,
             ws ? ws->tally : nullptr};
    L.fault = fault_word();
    L.summary = acc;
    int64_t blocks = 0;
    if (int rc = launch_blocks(ke, nsys, smem, &blocks)) return rc;
    ke->fn<<<(unsigned)blocks, kThreads, smem, st>>>(*method, *opt, L);
    if (int rc = cuda_err(cudaGetLastError(), "kernel launch")) return rc;
    if (tally) {
        unsigned long long h[6];
        if (int rc = cuda_err(cudaMemcpyAsync(h, ws->tally, sizeof(h), cudaMemcpyDeviceToHost, st),
                              "tally copy"))
            return rc;
        if (int rc = cuda_err(cudaStreamSynchronize(st), "tally copy")) return rc;
        if (int rc = check_fault()) return rc;
        for (int c = 0; c < 6; ++c) tally->counts[c] = (int64_t)h[c];
    }
    return 0;
}

int gsb_solve_batch(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
                    double* X, int32_t x_layout, void* S, int32_t s_kind, const double* P,
                    int32_t p_layout, const int64_t* order, int32_t order_base, int64_t nsys,
                    void* stream, GsbTally* tally) {
    g_err.clear();
    return solve_batch_impl(prob, method, opt, X, x_layout, S, s_kind, P, p_layout, order,
                            order_base, nsys, stream, tally, nullptr);
}

// BatchSummary from the partials of a first pass (src/nonlinear/batched.jl:80-89): |F| is the
// 2-norm of the per-system fnorms by rnorm's rule, so when the sum of squares left the normal
// range a second pass over S sums the squares scaled by the largest |fnorm|'s exponent.
int finish_summary(const SummaryAcc& h, const unsigned char* S, int64_t nsys, cudaStream_t st,
                   Workspace* ws, GsbSummary* out) {
    double s = h.sumsq;
    double mx;
    std::memcpy(&mx, &h.maxbits, sizeof(double));
    double fnorm;
    if (h.nan_seen) {
        fnorm = __builtin_nan("");
    } else if (std::isfinite(s) && s >= (double)nsys * 2.2250738585072014e-308) {
        fnorm = std::sqrt(s);
    } else if (mx == 0.0 || !std::isfinite(mx)) {
        fnorm = mx;
    } else {
        int blocks = (int)((nsys + 255) / 256);
        blocks = blocks > 1184 ? 1184 : blocks;
        int e = std::ilogb(mx);
        double zero = 0.0;
        if (int rc = cuda_err(cudaMemcpyAsync(&ws->acc->sumsq, &zero, sizeof(double),
                                              cudaMemcpyHostToDevice, st), "copy"))
            return rc;
        summary_kernel<<<blocks, 256, 0, st>>>(S, nsys, ws->acc, e, 1);
        double s2 = 0;
        if (int rc = cuda_err(cudaMemcpyAsync(&s2, &ws->acc->sumsq, sizeof(double),
                                              cudaMemcpyDeviceToHost, st), "copy"))
            return rc;
        if (int rc = cuda_err(cudaStreamSynchronize(st), "sync")) return rc;
        fnorm = std::ldexp(std::sqrt(s2), e);
    }
    out->fnorm = fnorm;
    out->failure_count = (int64_t)h.failures;
    out->all_converged = h.failures == 0;
    out->max_iterations = h.max_iterations;
    out->total_iterations = (int64_t)h.total_iterations;
    return 0;
}

int gsb_batch_summary(const GsbStatus64* S, int64_t nsys, void* stream, GsbSummary* out) {
    g_err.clear();
    if (!out) return set_err(GSB_ERR_ARGUMENT, "null output");
    std::memset(out, 0, sizeof(*out));
    if (nsys == 0) {
        out->all_converged = 1;
        return 0;
    }
    if (!S) return set_err(GSB_ERR_ARGUMENT, "null statuses");
    Workspace* ws = nullptr;
    if (int rc = workspace(&ws)) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    SummaryAcc h{};
    if (int rc = cuda_err(cudaMemsetAsync(ws->acc, 0, sizeof(SummaryAcc), st), "memset")) return rc;
    int blocks = (int)((nsys + 255) / 256);
    blocks = blocks > 1184 ? 1184 : blocks;
    summary_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<const unsigned char*>(S), nsys, ws->acc,
                                           0, 0);
    if (int rc = cuda_err(cudaMemcpyAsync(&h, ws->acc, sizeof(h), cudaMemcpyDeviceToHost, st), "copy"))
        return rc;
    if (int rc = cuda_err(cudaStreamSynchronize(st), "sync")) return rc;
    return finish_summary(h, reinterpret_cast<const unsigned char*>(S), nsys, st, ws, out);
}

int gsb_solve_batch_summary(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
                            double* X, int32_t x_layout, GsbStatus64* S, const double* P,
                            int32_t p_layout, const int64_t* order, int32_t order_base,
                            int64_t nsys, void* stream, GsbSummary* out) {
    g_err.clear();
    if (!out) return set_err(GSB_ERR_ARGUMENT, "null summary");
    std::memset(out, 0, sizeof(*out));
    if (nsys == 0) {
        if (int rc = solve_batch_impl(prob, method, opt, X, x_layout, S, GSB_STATUS64, P, p_layout,
                                      order, order_base, nsys, stream, nullptr, nullptr))
            return rc;
        out->all_converged = 1;
        return 0;
    }
    Workspace* ws = nullptr;
    if (int rc = workspace(&ws)) return rc;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int rc = cuda_err(cudaMemsetAsync(ws->acc, 0, sizeof(SummaryAcc), st), "memset")) return rc;
    if (int rc = solve_batch_impl(prob, method, opt, X, x_layout, S, GSB_STATUS64, P, p_layout,
                                  order, order_base, nsys, stream, nullptr, ws->acc))
        return rc;
    SummaryAcc h{};
    if (int rc = cuda_err(cudaMemcpyAsync(&h, ws->acc, sizeof(h), cudaMemcpyDeviceToHost, st), "copy"))
        return rc;
    if (int rc = cuda_err(cudaStreamSynchronize(st), "sync")) return rc;
    if (int rc = check_fault()) return rc;
    return finish_summary(h, reinterpret_cast<const unsigned char*>(S), nsys, st, ws, out);
}

int gsb_synchronize(void* stream) {
    if (int rc = cuda_err(cudaStreamSynchronize(reinterpret_cast<cudaStream_t>(stream)),
                          "cudaStreamSynchronize"))
        return rc;
    return check_fault();
}


int gsb_solve_batch_counts_noalloc(const GsbProblem* prob, const GsbMethod* method,
                                   const GsbOptions* opt, double* X, int32_t x_layout,
                                   uint8_t* codes, const double* P, int32_t p_layout,
                                   const int64_t* order, int32_t order_base, int64_t nsys,
                                   void* stream, GsbTally* tally) {
    g_err.clear();
    if (!tally) return set_err(GSB_ERR_ARGUMENT, "the count form needs a host GsbTally");
    std::memset(tally, 0, sizeof(*tally));
    if (int rc = check_call(prob, method, opt, nsys, x_layout, p_layout, order_base)) return rc;
    if (order && nsys > (int64_t)GSB_NOALLOC_MAX_ORDERED)
        return set_err(GSB_ERR_DIMENSION,
                       "with an order, the allocation-free count form takes at most "
                       "16777216 systems (GSB_NOALLOC_MAX_ORDERED)");
    if (nsys == 0) return 0;
    if (!X || !codes || !P) return set_err(GSB_ERR_ARGUMENT, "null X, codes or P");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long* scratch = nullptr;
    if (int rc = noalloc_scratch(&scratch)) return rc;
    const int64_t words = order ? (nsys + 63) / 64 : 0;
    noalloc_clear<<<(unsigned)((kNoallocHead + words + 255) / 256 > 1184 ? 1184 : (kNoallocHead + words + 255) / 256),
                    256, 0, st>>>(scratch, words);
    if (int rc = cuda_err(cudaGetLastError(), "noalloc_clear")) return rc;
    if (order) {
        // isperm on the device (the reference checks it on the host,
        // src/nonlinear/batched.jl:134-136)
        unsigned blocks = (unsigned)((nsys + 255) / 256 > 1184 ? 1184 : (nsys + 255) / 256);
        noalloc_check_order<<<blocks, 256, 0, st>>>(order, order_base, nsys, scratch);
        if (int rc = cuda_err(cudaGetLastError(), "noalloc_check_order")) return rc;
        unsigned long long flags = 0;
        if (int rc = cuda_err(cudaMemcpyAsync(&flags, scratch + 6, sizeof(flags),
                                              cudaMemcpyDeviceToHost, st), "flag copy"))
            return rc;
        if (int rc = cuda_err(cudaStreamSynchronize(st), "flag copy")) return rc;
        if (flags) return set_err(GSB_ERR_ARGUMENT, "order is not a permutation of the batch");
    }
    // word 7 of the array is the kernel's staging-fault word
    if (int rc = launch_solve(prob, method, opt, X, x_layout, codes, GSB_CODES, P, p_layout, order,
                              order_base, nsys, st, scratch, reinterpret_cast<unsigned*>(scratch + 7)))
        return rc;
    unsigned long long h[8];
    if (int rc = cuda_err(cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st),
                          "tally copy"))
        return rc;
    if (int rc = cuda_err(cudaStreamSynchronize(st), "tally copy")) return rc;
    if (h[7] != 0)
        return set_err(GSB_ERR_CUDA,
                       "the batch kernel's wait for its staging copies ran out; systems were left "
                       "unsolved");
    for (int c = 0; c < 6; ++c) tally->counts[c] = (int64_t)h[c];
    return 0;
}

}  // extern "C"

// ─── ragged batches ─────────────────────────────────────────────────────────────────────────
//
// Systems of different sizes, packed back to back. Three small kernels sort the systems into
// size buckets (count, ranges, scatter of the indices), then each bucket's kernel, a persistent
// launch with its own device work queue, solves its bucket through `order` and the ragged
// offsets. The buckets' kernels run on forked streams, so their tails overlap; the whole
// sequence is captured once into a CUDA graph per set of arguments and replayed.

namespace gsb {

constexpr int kUnevenSizes[GSB_UNEVEN_BUCKETS] = {2, 3, 4, 6, 8, 12, 16, 24, 32};

__device__ __forceinline__ int uneven_bucket(int n) {
    switch (n) {
    case 2: return 0;
    case 3: return 1;
    case 4: return 2;
    case 6: return 3;
    case 8: return 4;
    case 12: return 5;
    case 16: return 6;
    case 24: return 7;
    case 32: return 8;
    default: return -1;
    }
}

// The bucketing state of one call, in device memory (zeroed at the start of each run).
struct UnevenWork {
    unsigned long long count[GSB_UNEVEN_BUCKETS];
    unsigned long long range[GSB_UNEVEN_BUCKETS][2];  // {count, first} in the index list
    unsigned long long queue[GSB_UNEVEN_BUCKETS];
    unsigned long long bad;  // systems whose size is outside the set
    unsigned long long tally[6];
};

// The bucketing takes three passes over the sizes, each CTA over its own contiguous range of
// systems (`chunk` each), with no global atomics: its per-bucket counts, then one CTA turns them
// into each CTA's first index per bucket, then each CTA writes its systems' indices in order.
// A bucket's index list is therefore in the order of the batch, so that neighbouring systems of
// a bucket stay neighbours in memory.
constexpr int kBucketThreads = 256;

__device__ __forceinline__ int bucket_slot(int32_t n) {
    const int b = uneven_bucket(n);
    return b < 0 ? GSB_UNEVEN_BUCKETS : b;  // the last slot holds the sizes outside the set
}

// Per-CTA counts of each bucket, cta_count[c * GSB_UNEVEN_BUCKETS + b].
__global__ void __launch_bounds__(kBucketThreads) uneven_count(const int32_t* n, int64_t nsys,
                                                               int64_t chunk, UnevenWork* w,
                                                               unsigned* cta_count) {
    __shared__ unsigned cnt[GSB_UNEVEN_BUCKETS + 1];
    if (threadIdx.x <= GSB_UNEVEN_BUCKETS) cnt[threadIdx.x] = 0u;
    __syncthreads();
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = lo + chunk < nsys ? lo + chunk : nsys;
    const int lane = threadIdx.x & 31;
    for (int64_t s = lo + threadIdx.x; s < hi; s += kBucketThreads) {
        const int slot = bucket_slot(n[s]);
        const unsigned grp = __match_any_sync(__activemask(), slot);
        if (lane == __ffs(grp) - 1) atomicAdd(&cnt[slot], (unsigned)__popc(grp));
    }
    __syncthreads();
    if (threadIdx.x < GSB_UNEVEN_BUCKETS)
        cta_count[(int64_t)blockIdx.x * GSB_UNEVEN_BUCKETS + threadIdx.x] = cnt[threadIdx.x];
    if (threadIdx.x == GSB_UNEVEN_BUCKETS && cnt[GSB_UNEVEN_BUCKETS])
        atomicAdd(&w->bad, (unsigned long long)cnt[GSB_UNEVEN_BUCKETS]);
}

// One CTA of GSB_UNEVEN_BUCKETS warps: warp b scans bucket b's per-CTA counts into each CTA's
// first index (in place), after the indices of the smaller sizes; the bucket ranges go to w.
__global__ void uneven_ranges(UnevenWork* w, unsigned* cta_count, int ctas) {
    __shared__ unsigned long long total[GSB_UNEVEN_BUCKETS];
    const int b = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int per = (ctas + 31) / 32;
    const int c0 = lane * per, c1 = c0 + per < ctas ? c0 + per : ctas;
    unsigned long long sum = 0;
    for (int c = c0; c < c1; ++c) sum += cta_count[(int64_t)c * GSB_UNEVEN_BUCKETS + b];
    unsigned long long incl = sum;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned long long o = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += o;
    }
    if (lane == 31) total[b] = incl;
    __syncthreads();
    unsigned long long first = 0;
    for (int q = 0; q < b; ++q) first += total[q];
    unsigned long long at = first + incl - sum;
    for (int c = c0; c < c1; ++c) {
        unsigned* slot = &cta_count[(int64_t)c * GSB_UNEVEN_BUCKETS + b];
        const unsigned k = *slot;
        *slot = (unsigned)at;
        at += k;
    }
    if (lane == 0) {
        w->count[b] = total[b];
        w->range[b][0] = total[b];
        w->range[b][1] = first;
    }
}

// Each system's index into its bucket's part of the list, tile by tile in the batch's order.
__global__ void __launch_bounds__(kBucketThreads) uneven_scatter(const int32_t* n, int64_t nsys,
                                                                 int64_t chunk,
                                                                 const unsigned* cta_first,
                                                                 int64_t* list) {
    constexpr int W = kBucketThreads / 32, B = GSB_UNEVEN_BUCKETS;
    __shared__ unsigned base[B], tile_total[B];
    __shared__ unsigned warp_first[W][B + 1];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid < B) base[tid] = cta_first[(int64_t)blockIdx.x * B + tid];
    const int64_t lo = (int64_t)blockIdx.x * chunk;
    const int64_t hi = lo + chunk < nsys ? lo + chunk : nsys;
    for (int64_t tile = lo; tile < hi; tile += kBucketThreads) {  // the same count in every thread
        if (tid < W * (B + 1)) warp_first[tid / (B + 1)][tid % (B + 1)] = 0u;
        __syncthreads();
        const int64_t s = tile + tid;
        const int slot = s < hi ? bucket_slot(n[s]) : B;
        const unsigned grp = __match_any_sync(0xffffffffu, slot);
        const unsigned rank = __popc(grp & ((1u << lane) - 1u));
        if (lane == __ffs(grp) - 1) warp_first[warp][slot] = (unsigned)__popc(grp);
        __syncthreads();
        if (tid < B) {
            unsigned run = 0;
            for (int q = 0; q < W; ++q) {
                const unsigned k = warp_first[q][tid];
                warp_first[q][tid] = run;
                run += k;
            }
            tile_total[tid] = run;
        }
        __syncthreads();
        if (slot < B) list[(int64_t)base[slot] + warp_first[warp][slot] + rank] = s;
        __syncthreads();
        if (tid < B) base[tid] += tile_total[tid];
    }
}

}  // namespace gsb

namespace {

struct UnevenKey {
    GsbMethod m;
    GsbOptions o;
    GsbBucketConfig table[GSB_UNEVEN_BUCKETS];
    double* X;
    void* S;
    int32_t s_kind;
    const double* P;
    const int32_t* n;
    const int64_t* x_off;
    const int64_t* p_off;
    int64_t nsys;
    bool operator==(const UnevenKey& k) const { return std::memcmp(this, &k, sizeof(*this)) == 0; }
};

// One device's ragged-batch state: the bucketing workspace, the streams of the buckets' fork,
// and the graph of the last argument set.
struct UnevenPlan {
    bool ready = false;
    UnevenKey key{};
    gsb::UnevenWork* work = nullptr;
    unsigned* cta_count = nullptr;  // the bucketing's per-CTA counts (kBucketCtasPerSm x SMs x 9)
    int64_t* list = nullptr;
    int64_t list_cap = 0;
    cudaStream_t cs = nullptr;
    cudaStream_t side[GSB_UNEVEN_BUCKETS] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[GSB_UNEVEN_BUCKETS] = {};
    cudaGraphExec_t exec = nullptr;
    // Buckets launched as one ordinary grid sized from their count (ctas_per_sm = -1): the
    // graph copies the bucket ranges to pinned host memory and records `counted`; the host then
    // launches those buckets on `ord`, which the caller's stream joins through `ord_done`.
    unsigned long long* h_range = nullptr;  // {count, first} per bucket (pinned)
    cudaStream_t ord = nullptr;
    cudaEvent_t counted = nullptr, ord_done = nullptr;
    bool ordinary[GSB_UNEVEN_BUCKETS] = {};
    bool any_ordinary = false;
    KernelEntry* ke[GSB_UNEVEN_BUCKETS] = {};
    unsigned threads[GSB_UNEVEN_BUCKETS] = {};
    size_t smem[GSB_UNEVEN_BUCKETS] = {};
    int occ[GSB_UNEVEN_BUCKETS] = {};
};
std::mutex g_uneven_mu;
UnevenPlan g_uneven[64];
constexpr int kBucketCtasPerSm = 8;  // CTAs of the bucketing kernels

int uneven_streams(UnevenPlan& p) {
    if (p.cs) return 0;
    if (int rc = cuda_err(cudaStreamCreateWithFlags(&p.cs, cudaStreamNonBlocking), "stream")) return rc;
    if (int rc = cuda_err(cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming), "event")) return rc;
    for (int b = 0; b < GSB_UNEVEN_BUCKETS; ++b) {
        if (int rc = cuda_err(cudaStreamCreateWithFlags(&p.side[b], cudaStreamNonBlocking), "stream"))
            return rc;
        if (int rc = cuda_err(cudaEventCreateWithFlags(&p.join[b], cudaEventDisableTiming), "event"))
            return rc;
    }
    if (int rc = cuda_err(cudaStreamCreateWithFlags(&p.ord, cudaStreamNonBlocking), "stream")) return rc;
    if (int rc = cuda_err(cudaEventCreateWithFlags(&p.counted, cudaEventDisableTiming), "event"))
        return rc;
    if (int rc = cuda_err(cudaEventCreateWithFlags(&p.ord_done, cudaEventDisableTiming), "event"))
        return rc;
    if (int rc = cuda_err(cudaHostAlloc(reinterpret_cast<void**>(&p.h_range),
                                        2 * GSB_UNEVEN_BUCKETS * sizeof(unsigned long long),
                                        cudaHostAllocDefault),
                          "cudaHostAlloc"))
        return rc;
    return 0;
}

// The kernel of bucket b, its persistent grid and its CTA (threads, bytes of shared memory).
// (ctas_per_sm = -1: one ordinary grid, launched by the host once the bucket's count is known;
// `grid` is then 0 and `occ` the resident CTAs per SM of that kernel.)
int uneven_entry(const UnevenKey& k, int b, int sms, KernelEntry** ke, unsigned* grid,
                 unsigned* threads, size_t* smem, int* occ_out) {
    GsbProblem prob{};
    prob.family = GSB_FAMILY_CUBIC_AFFINE;
    prob.n = prob.m = kUnevenSizes[b];
    const bool fused = k.m.arithmetic == GSB_FUSED;
    const bool mixed = k.m.factor_precision == GSB_F32;
    const int T = k.table[b].threads_per_system;
    *ke = select_kernel(&prob, fused, mixed, k.m.refinement == GSB_REFINEMENT,
                        T == 0 ? (kUnevenSizes[b] <= 8 ? 1 : 0) : T);
    if (!*ke) return set_err(GSB_ERR_UNSUPPORTED, "no kernel for bucket n = " +
                                                      std::to_string(kUnevenSizes[b]) +
                                                      " with these threads per system");
    *threads = kThreads;
    *smem = (size_t)(*ke)->smem_doubles * sizeof(double);
    const int spc = k.table[b].systems_per_cta;
    if (spc != 0) {
        // the warp form takes its CTA size at launch; the other forms have theirs fixed
        const int lanes = (*ke)->lanes;
        if (lanes == 0 || spc < 0 || spc * lanes > kThreads || (spc * lanes) % 32 != 0)
            return set_err(GSB_ERR_ARGUMENT,
                           "systems_per_cta of bucket n = " + std::to_string(kUnevenSizes[b]) +
                               ": 0, or (for the warp form, n >= 12) a count whose CTA of "
                               "systems_per_cta x threads_per_system lanes is a multiple of 32 "
                               "and at most " + std::to_string(kThreads));
        *threads = (unsigned)(spc * lanes);
        *smem = (size_t)spc * (*ke)->sys_doubles * sizeof(double);
    }
    const int want = k.table[b].ctas_per_sm;
    if (want < -1)
        return set_err(GSB_ERR_ARGUMENT, "ctas_per_sm of bucket n = " +
                                             std::to_string(kUnevenSizes[b]) +
                                             ": -1 (an ordinary launch), 0 (as many as fit) or more");
    const KernelFn fn = want == -1 ? (*ke)->fn : (*ke)->fn_persistent;
    if (!fn) return set_err(GSB_ERR_UNSUPPORTED, "no persistent bucket kernel");
    // the bucket's kernel (its attribute set once per capture, which is rare); the attribute is
    // the largest CTA the kernel takes, so that every CTA size fits under it
    const size_t smem_max = (size_t)(*ke)->smem_doubles * sizeof(double);
    if (int rc = cuda_err(cudaFuncSetAttribute(reinterpret_cast<const void*>(fn),
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)std::max(smem_max, *smem)),
                          "cudaFuncSetAttribute"))
        return rc;
    int occ = 0;
    if (int rc = cuda_err(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
                              &occ, reinterpret_cast<const void*>(fn), (int)*threads, *smem),
                          "occupancy"))
        return rc;
    if (occ < 1) return set_err(GSB_ERR_UNSUPPORTED, "a bucket kernel does not fit on an SM");
    *occ_out = occ;
    *grid = want == -1 ? 0u : (unsigned)((want > 0 && want < occ ? want : occ) * sms);
    return 0;
}

int uneven_capture(UnevenPlan& p, const UnevenKey& k, bool want_tally) {
    int dev = 0, sms = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (int rc = cuda_err(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "attr"))
        return rc;
    KernelEntry** ke = p.ke;
    unsigned grid[GSB_UNEVEN_BUCKETS];
    unsigned* threads = p.threads;
    size_t* smem = p.smem;
    p.any_ordinary = false;
    for (int b = 0; b < GSB_UNEVEN_BUCKETS; ++b) {
        if (int rc = uneven_entry(k, b, sms, &ke[b], &grid[b], &threads[b], &smem[b], &p.occ[b]))
            return rc;
        p.ordinary[b] = grid[b] == 0;
        p.any_ordinary = p.any_ordinary || p.ordinary[b];
    }
    if (p.exec) {
        cudaGraphExecDestroy(p.exec);
        p.exec = nullptr;
    }
    // the bucketing's CTAs, each over a contiguous range of `chunk` systems
    const unsigned cgrid = (unsigned)std::min<int64_t>(
        (k.nsys + gsb::kBucketThreads - 1) / gsb::kBucketThreads, (int64_t)sms * kBucketCtasPerSm);
    const int64_t chunk = (k.nsys + cgrid - 1) / cgrid;
    unsigned* fault = fault_word();  // allocated (once) before the capture begins
    cudaGraph_t g = nullptr;
    if (int rc = cuda_err(cudaStreamBeginCapture(p.cs, cudaStreamCaptureModeThreadLocal), "capture"))
        return rc;
    cudaMemsetAsync(p.work, 0, sizeof(gsb::UnevenWork), p.cs);
    gsb::uneven_count<<<cgrid, gsb::kBucketThreads, 0, p.cs>>>(k.n, k.nsys, chunk, p.work,
                                                              p.cta_count);
    gsb::uneven_ranges<<<1, 32 * GSB_UNEVEN_BUCKETS, 0, p.cs>>>(p.work, p.cta_count, (int)cgrid);
    gsb::uneven_scatter<<<cgrid, gsb::kBucketThreads, 0, p.cs>>>(k.n, k.nsys, chunk, p.cta_count,
                                                                p.list);
    if (p.any_ordinary) {
        // the bucket ranges for the host, which sizes the ordinary launches from them
        cudaMemcpyAsync(p.h_range, &p.work->range[0][0],
                        2 * GSB_UNEVEN_BUCKETS * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                        p.cs);
        // an event node of the graph (an external record), so that the host can wait on it
        cudaEventRecordWithFlags(p.counted, p.cs, cudaEventRecordExternal);
    }
    cudaEventRecord(p.fork, p.cs);
    // the heaviest buckets (largest n) start first, so that the light ones fill the tail
    for (int b = GSB_UNEVEN_BUCKETS - 1; b >= 0; --b) {
        if (p.ordinary[b]) continue;
        cudaStreamWaitEvent(p.side[b], p.fork, 0);
        Launch L{k.X, GSB_AOS, k.S, k.s_kind, k.P, GSB_AOS, p.list, 0, k.nsys, nullptr,
                 want_tally ? p.work->tally : nullptr, k.x_off, k.p_off, &p.work->queue[b],
                 &p.work->range[b][0], fault};
        ke[b]->fn_persistent<<<grid[b], threads[b], smem[b], p.side[b]>>>(k.m, k.o, L);
        cudaEventRecord(p.join[b], p.side[b]);
        cudaStreamWaitEvent(p.cs, p.join[b], 0);
    }
    cudaError_t e = cudaStreamEndCapture(p.cs, &g);
    if (int rc = cuda_err(e, "end capture")) return rc;
    e = cudaGraphInstantiate(&p.exec, g, 0);
    cudaGraphDestroy(g);
    if (int rc = cuda_err(e, "graph instantiate")) return rc;
    return 0;
}

}  // namespace

extern "C" {

int gsb_uneven_sizes(int32_t* sizes_out) {
    if (!sizes_out) return set_err(GSB_ERR_ARGUMENT, "null sizes_out");
    for (int b = 0; b < GSB_UNEVEN_BUCKETS; ++b) sizes_out[b] = kUnevenSizes[b];
    return 0;
}

int gsb_solve_batch_uneven(const GsbMethod* method, const GsbOptions* opt, double* X, void* S,
                           int32_t s_kind, const double* P, const int32_t* n,
                           const int64_t* x_off, const int64_t* p_off, int64_t nsys,
                           const GsbBucketConfig* table, void* stream, GsbTally* tally) {
    g_err.clear();
    if (!method || !opt) return set_err(GSB_ERR_ARGUMENT, "null method or options");
    if (nsys < 0) return set_err(GSB_ERR_DIMENSION, "negative batch length");
    if (int rc = check_options(opt)) return rc;
    if (int rc = check_method(method)) return rc;
    if (method->globalization == GSB_LEVENBERG_MARQUARDT || method->linsolve != GSB_LU)
        return set_err(GSB_ERR_UNSUPPORTED, "ragged batches run Newton with LUFactorization");
    if (method->reuse > 0 || method->globalization == GSB_DOGLEG)
        return set_err(GSB_ERR_UNSUPPORTED, "ragged batches take no factor reuse and no DogLeg");
    if (method->trial_precision == GSB_F32)
        return set_err(GSB_ERR_UNSUPPORTED, "ragged batches take Float64 line-search trials");
    if (s_kind != GSB_STATUS64 && s_kind != GSB_CODES) return set_err(GSB_ERR_ARGUMENT, "s_kind");
    if (tally) std::memset(tally, 0, sizeof(*tally));
    if (nsys == 0) return 0;
    if (nsys >= (int64_t)1 << 32)
        return set_err(GSB_ERR_DIMENSION, "a ragged batch takes fewer than 2^32 systems");
    if (!X || !S || !P || !n || !x_off || !p_off)
        return set_err(GSB_ERR_ARGUMENT, "null X, S, P, n, x_off or p_off");
    UnevenKey key{};
    key.m = *method;
    key.o = *opt;
    if (table) std::memcpy(key.table, table, sizeof(key.table));
    key.X = X;
    key.S = S;
    key.s_kind = s_kind;
    key.P = P;
    key.n = n;
    key.x_off = x_off;
    key.p_off = p_off;
    key.nsys = nsys;
    int dev = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (dev < 0 || dev >= 64) return set_err(GSB_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_uneven_mu);
    UnevenPlan& p = g_uneven[dev];
    if (int rc = uneven_streams(p)) return rc;
    if (!p.work) {
        if (int rc = cuda_err(cudaMalloc(&p.work, sizeof(gsb::UnevenWork)), "cudaMalloc")) return rc;
    }
    if (!p.cta_count) {
        int sms = 0;
        if (int rc = cuda_err(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                              "attr"))
            return rc;
        const size_t bytes = (size_t)sms * kBucketCtasPerSm * GSB_UNEVEN_BUCKETS * sizeof(unsigned);
        if (int rc = cuda_err(cudaMalloc(&p.cta_count, bytes), "cudaMalloc")) return rc;
    }
    if (p.list_cap < nsys) {
        if (p.list) cudaFree(p.list);
        p.list = nullptr;
        p.list_cap = 0;
        p.ready = false;
        if (int rc = cuda_err(cudaMalloc(&p.list, nsys * sizeof(int64_t)), "cudaMalloc")) return rc;
        p.list_cap = nsys;
    }
    if (!p.ready || !(p.key == key)) {
        p.ready = false;
        if (int rc = uneven_capture(p, key, true)) return rc;
        p.key = key;
        p.ready = true;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (int rc = cuda_err(cudaGraphLaunch(p.exec, st), "graph launch")) return rc;
    if (p.any_ordinary) {
        // the buckets of ordinary launches: one grid each, sized from the count the graph
        // copied out, on their own stream beside the graph's persistent buckets
        if (int rc = cuda_err(cudaEventSynchronize(p.counted), "bucket counts")) return rc;
        if (int rc = cuda_err(cudaStreamWaitEvent(p.ord, p.counted, 0), "stream wait")) return rc;
        int sms = 0;
        if (int rc = cuda_err(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                              "attr"))
            return rc;
        // the ranges tile the index list in bucket order (checked before any launch reads it)
        unsigned long long at = 0;
        for (int b = 0; b < GSB_UNEVEN_BUCKETS; ++b) {
            if (p.h_range[2 * b + 1] != at) return set_err(GSB_ERR_CUDA, "bucket ranges not read");
            at += p.h_range[2 * b];
        }
        if (at > (unsigned long long)key.nsys) return set_err(GSB_ERR_CUDA, "bucket ranges not read");
        for (int b = GSB_UNEVEN_BUCKETS - 1; b >= 0; --b) {
            const unsigned long long count = p.h_range[2 * b], first = p.h_range[2 * b + 1];
            if (!p.ordinary[b] || count == 0) continue;
            KernelEntry* ke = p.ke[b];
            // systems per CTA: the CTA's teams for the warp form (its size chosen at launch),
            // the entry's fixed count otherwise
            const int64_t spb =
                ke->lanes ? (int64_t)p.threads[b] / ke->lanes : (int64_t)ke->systems_per_block;
            int64_t blocks = ((int64_t)count + spb - 1) / spb;
            if (ke->resident && blocks > (int64_t)sms * p.occ[b]) blocks = (int64_t)sms * p.occ[b];
            Launch L{key.X, GSB_AOS, key.S, key.s_kind, key.P, GSB_AOS, p.list + first, 0,
                     (int64_t)count, nullptr, p.work->tally, key.x_off, key.p_off, nullptr,
                     nullptr, fault_word()};
            ke->fn<<<(unsigned)blocks, p.threads[b], p.smem[b], p.ord>>>(key.m, key.o, L);
            if (int rc = cuda_err(cudaGetLastError(), "kernel launch")) return rc;
        }
        if (int rc = cuda_err(cudaEventRecord(p.ord_done, p.ord), "event")) return rc;
        if (int rc = cuda_err(cudaStreamWaitEvent(st, p.ord_done, 0), "stream wait")) return rc;
    }
    unsigned long long h[7];
    if (int rc = cuda_err(cudaMemcpyAsync(h, &p.work->bad, sizeof(h), cudaMemcpyDeviceToHost, st),
                          "tally copy"))
        return rc;
    if (int rc = cuda_err(cudaStreamSynchronize(st), "synchronize")) return rc;
    if (int rc = check_fault()) return rc;
    if (tally)
        for (int c = 0; c < 6; ++c) tally->counts[c] = (int64_t)h[1 + c];
    if (h[0]) return set_err(GSB_ERR_ARGUMENT, std::to_string(h[0]) +
                                                   " systems have a size outside {2, 3, 4, 6, 8, "
                                                   "12, 16, 24, 32}");
    return 0;
}

}  // extern "C"

// ─── batches in host memory ─────────────────────────────────────────────────────────────────
//
// The batch streams through the device in chunks over three streams: while chunk k solves, the
// inputs of chunk k+1 arrive and the results of chunk k-1 leave, so the copies in both
// directions and the solves overlap (page-locked host memory lets the copies run asynchronously).
// Three staging slots per device are kept between calls.

namespace {

constexpr int kSlots = 3;

struct HostPipe {
    double* x[kSlots] = {};
    double* p[kSlots] = {};
    unsigned char* s[kSlots] = {};
    int64_t cap_x = 0, cap_p = 0, cap_s = 0;  // bytes per slot
    unsigned long long* tally = nullptr;
    cudaStream_t h2d = nullptr, comp = nullptr, d2h = nullptr;
    cudaEvent_t in[kSlots] = {}, solved[kSlots] = {}, out[kSlots] = {};
};
std::mutex g_pipe_mu;
HostPipe g_pipe[64];

int pipe_grow(void** buf, int64_t& cap, int64_t bytes) {
    if (cap >= bytes) return 0;
    if (*buf) cudaFree(*buf);
    *buf = nullptr;
    cap = 0;
    if (int rc = cuda_err(cudaMalloc(buf, bytes), "cudaMalloc")) return rc;
    cap = bytes;
    return 0;
}

int pipe_setup(HostPipe& hp, int64_t xb, int64_t pb, int64_t sb) {
    if (!hp.h2d) {
        for (cudaStream_t* st : {&hp.h2d, &hp.comp, &hp.d2h})
            if (int rc = cuda_err(cudaStreamCreateWithFlags(st, cudaStreamNonBlocking), "stream")) return rc;
        for (int k = 0; k < kSlots; ++k)
            for (cudaEvent_t* ev : {&hp.in[k], &hp.solved[k], &hp.out[k]})
                if (int rc = cuda_err(cudaEventCreateWithFlags(ev, cudaEventDisableTiming), "event"))
                    return rc;
        if (int rc = cuda_err(cudaMalloc(&hp.tally, 6 * sizeof(unsigned long long)), "cudaMalloc"))
            return rc;
    }
    int64_t cx = hp.cap_x, cp = hp.cap_p, cs = hp.cap_s;
    for (int k = 0; k < kSlots; ++k) {
        int64_t a = cx, b = cp, c = cs;
        if (int rc = pipe_grow(reinterpret_cast<void**>(&hp.x[k]), a, xb)) return rc;
        if (int rc = pipe_grow(reinterpret_cast<void**>(&hp.p[k]), b, pb)) return rc;
        if (int rc = pipe_grow(reinterpret_cast<void**>(&hp.s[k]), c, sb)) return rc;
        if (k == kSlots - 1) {
            hp.cap_x = a;
            hp.cap_p = b;
            hp.cap_s = c;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int gsb_solve_batch_host(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
                         double* X, void* S, int32_t s_kind, const double* P, int64_t nsys,
                         int64_t chunk, GsbTally* tally) {
    g_err.clear();
    if (!prob || !method || !opt) return set_err(GSB_ERR_ARGUMENT, "null problem, method or options");
    if (nsys < 0) return set_err(GSB_ERR_DIMENSION, "negative batch length");
    if (int rc = check_options(opt)) return rc;
    if (int rc = check_method(method)) return rc;
    const int64_t np = param_count(prob);
    if (np < 0) return set_err(GSB_ERR_ARGUMENT, "unknown family or size");
    if (s_kind != GSB_STATUS64 && s_kind != GSB_CODES) return set_err(GSB_ERR_ARGUMENT, "s_kind");
    if (chunk < 0) return set_err(GSB_ERR_ARGUMENT, "negative chunk");
    if (tally) std::memset(tally, 0, sizeof(*tally));
    if (nsys == 0) return 0;
    if (!X || !S || !P) return set_err(GSB_ERR_ARGUMENT, "null X, S or P");
    const int64_t n = prob->n;
    const int64_t sbytes = s_kind == GSB_STATUS64 ? 72 : 1;
    if (chunk == 0) chunk = 262144;
    if (chunk > nsys) chunk = nsys;
    int dev = 0;
    if (int rc = cuda_err(cudaGetDevice(&dev), "cudaGetDevice")) return rc;
    if (dev < 0 || dev >= 64) return set_err(GSB_ERR_CUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_pipe_mu);
    HostPipe& hp = g_pipe[dev];
    if (int rc = pipe_setup(hp, chunk * n * 8, chunk * np * 8, chunk * sbytes)) return rc;
    if (int rc = cuda_err(cudaMemsetAsync(hp.tally, 0, 6 * sizeof(unsigned long long), hp.comp), "memset"))
        return rc;
    // Every call's return code is checked. On an error after the first copy is queued, the three
    // streams are drained before returning, so that no copy still writes into X or S (or reads
    // the staging slots of a next call) once the caller has been told the call failed.
    auto drain = [&](int rc) {
        cudaStreamSynchronize(hp.h2d);
        cudaStreamSynchronize(hp.comp);
        cudaStreamSynchronize(hp.d2h);
        cudaGetLastError();
        return rc;
    };
    const int64_t nchunks = (nsys + chunk - 1) / chunk;
    unsigned* fault = fault_word();
    for (int64_t c = 0; c < nchunks; ++c) {
        const int k = (int)(c % kSlots);
        const int64_t first = c * chunk;
        const int64_t len = std::min(chunk, nsys - first);
        // the slot's previous results have left before its new inputs arrive
        if (c >= kSlots)
            if (int rc = cuda_err(cudaStreamWaitEvent(hp.h2d, hp.out[k], 0), "wait")) return drain(rc);
        if (int rc = cuda_err(cudaMemcpyAsync(hp.x[k], X + first * n, len * n * 8,
                                              cudaMemcpyHostToDevice, hp.h2d), "copy in"))
            return drain(rc);
        if (int rc = cuda_err(cudaMemcpyAsync(hp.p[k], P + first * np, len * np * 8,
                                              cudaMemcpyHostToDevice, hp.h2d), "copy in"))
            return drain(rc);
        if (int rc = cuda_err(cudaEventRecord(hp.in[k], hp.h2d), "event")) return drain(rc);
        if (int rc = cuda_err(cudaStreamWaitEvent(hp.comp, hp.in[k], 0), "wait")) return drain(rc);
        if (int rc = launch_solve(prob, method, opt, hp.x[k], GSB_AOS, hp.s[k], s_kind, hp.p[k],
                                  GSB_AOS, nullptr, 0, len, hp.comp, tally ? hp.tally : nullptr, fault))
            return drain(rc);
        if (int rc = cuda_err(cudaEventRecord(hp.solved[k], hp.comp), "event")) return drain(rc);
        if (int rc = cuda_err(cudaStreamWaitEvent(hp.d2h, hp.solved[k], 0), "wait")) return drain(rc);
        if (int rc = cuda_err(cudaMemcpyAsync(X + first * n, hp.x[k], len * n * 8,
                                              cudaMemcpyDeviceToHost, hp.d2h), "copy out"))
            return drain(rc);
        if (int rc = cuda_err(cudaMemcpyAsync(static_cast<unsigned char*>(S) + first * sbytes,
                                              hp.s[k], len * sbytes, cudaMemcpyDeviceToHost, hp.d2h),
                              "copy out"))
            return drain(rc);
        if (int rc = cuda_err(cudaEventRecord(hp.out[k], hp.d2h), "event")) return drain(rc);
    }
    unsigned long long h[6] = {};
    if (tally)
        if (int rc = cuda_err(cudaMemcpyAsync(h, hp.tally, sizeof(h), cudaMemcpyDeviceToHost, hp.comp),
                              "tally copy"))
            return drain(rc);
    cudaError_t e = cudaStreamSynchronize(hp.comp);
    if (e == cudaSuccess) e = cudaStreamSynchronize(hp.d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(hp.h2d);
    if (int rc = cuda_err(e, "host batch")) return drain(rc);
    if (int rc = check_fault()) return rc;
    if (tally)
        for (int c = 0; c < 6; ++c) tally->counts[c] = (int64_t)h[c];
    return 0;
}

}  // extern "C"
