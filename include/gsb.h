/*
 * gsb.h — the C-ABI of libgsb, a B200 (sm_100a) implementation of the R2 batched regime of
 * GeometricSolvers.jl: many small independent nonlinear systems, one work item per system, one
 * status per system.
 *
 * Reference interface replaced (paths are within the GeometricSolvers.jl project):
 *   solve_batch!(X, S, prob, method, p; order, options, workgroupsize, kwargs...) -> S
 *       src/nonlinear/batched.jl:257-287   -> gsb_solve_batch(..., s_kind = GSB_STATUS64)
 *   solve_batch!(X, prob, method, p; ...) -> NamedTuple of the six ReturnCode counts
 *       src/nonlinear/batched.jl:289-307   -> gsb_solve_batch(..., s_kind = GSB_CODES, tally)
 *   batch_summary(S) -> BatchSummary
 *       src/nonlinear/batched.jl:80-89     -> gsb_batch_summary
 *   SolverStatus{Float64}   src/base/status.jl:101-117     -> GsbStatus64 (same byte layout)
 *   Options{Float64}        src/base/options.jl:58-71      -> GsbOptions
 *   ReturnCode              src/base/returncodes.jl:14     -> GsbReturnCode
 *
 * Conventions. Every call returns 0 on success and a negative GsbError otherwise; nothing aborts.
 * Argument errors are detected on the host before any launch, as the reference's host checks
 * (src/nonlinear/batched.jl:113-150, 270-283) are. Numerical failures are never errors: each is
 * a GsbReturnCode in the status of its system. All array pointers are caller-owned DEVICE memory
 * (CuArray, torch tensor, cudaMalloc) of the current device; `stream` is a cudaStream_t (NULL =
 * the legacy default stream). Launches are stream-ordered; gsb_synchronize(stream) gives the
 * blocking behaviour of the reference's `_launch!` (src/nonlinear/batched.jl:193).
 */
#ifndef GSB_H
#define GSB_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GSB_ABI_VERSION 2

#if defined(__GNUC__)
#define GSB_API __attribute__((visibility("default")))
#else
#define GSB_API
#endif

/* ReturnCode, src/base/returncodes.jl:14 (UInt8, values 0..5 in this order). */
typedef enum {
    GSB_SUCCESS = 0,
    GSB_STALLED = 1,
    GSB_MAXITERS = 2,
    GSB_SINGULAR = 3,
    GSB_NONFINITE = 4,
    GSB_LINESEARCH_FAILED = 5
} GsbReturnCode;

/* Host-side errors. They mirror the reference's ArgumentError / DimensionMismatch. */
typedef enum {
    GSB_OK = 0,
    GSB_ERR_DIMENSION = -1,   /* DimensionMismatch: lengths that disagree */
    GSB_ERR_ARGUMENT = -2,    /* ArgumentError: an invalid value or option */
    GSB_ERR_UNSUPPORTED = -3, /* a combination the reference refuses or this build lacks */
    GSB_ERR_CUDA = -4         /* a CUDA runtime error; gsb_last_error() has the text */
} GsbError;

/*
 * SolverStatus{Float64} (src/base/status.jl:101-117) with Julia's field layout: offsets
 * code 0, f_calls 2, iterations 4, fnorm 8, stepnorm 16, step_failures 24, promoted 28,
 * stationary 29, jvp_calls 30, rank 32, nullnorm 40, gradratio 48, rate 56, contracted 64,
 * reused 65; size 72, alignment 8. A Vector{SolverStatus{Float64}} is passed by pointer.
 */
typedef struct {
    uint8_t code;
    uint8_t pad0_;
    int16_t f_calls;
    int32_t iterations;
    double fnorm;
    double stepnorm;
    int32_t step_failures;
    uint8_t promoted;
    uint8_t stationary;
    int16_t jvp_calls;
    int32_t rank;
    uint32_t pad1_;
    double nullnorm;
    double gradratio;
    double rate;
    uint8_t contracted;
    uint8_t reused;
    uint8_t pad2_[6];
} GsbStatus64;

/* Options{Float64}, src/base/options.jl:58-71, field for field. Defaults :207-236. */
typedef struct {
    double f_abstol;
    double f_reltol;
    double x_abstol;
    double x_reltol;
    int32_t min_iterations;
    int32_t max_iterations;
    int32_t max_stalls;
    int32_t norm; /* 0 = L2Norm, 1 = MaxNorm */
    double g_tol;
    double kappa;
    uint8_t roundoff;
    uint8_t rate_test;
    uint8_t pad_[6];
} GsbOptions;

/* Residual families: device functions selected by this tag. */
typedef enum {
    /* F(x, p) = A x + 0.1 x.^3 - b, p = (A column-major n*n, b n); n in 1..32.
     * BatchParams form (src/nonlinear/batched.jl:34-47, parameters (shared, per_system[i])):
     * with shared = A column-major and shared_len = n*n, every system shares A and its block
     * p is b alone (n doubles); n in {2, 3, 4, 6, 8} (one thread per system) and {12, 16,
     * 24, 32} (the warp form, A staged once per CTA at the family's column stride). */
    GSB_FAMILY_CUBIC_AFFINE = 1,
    /* Least squares r_i = sum_j a_j exp(-b_j t_i) - y_i, i = 1..m; x = (a1, b1, a2, b2, a3, b3),
     * p = y (m values); the m abscissae t are the problem's shared constants. n = 6. */
    GSB_FAMILY_EXPSUM3_LSQ = 2,
    /* Gauss-Legendre 3-stage stage equations of the Henon-Heiles field: Z - h (A (x) I) f(y + Z)
     * with x = Z the 12 stacked stage increments, p = y_n (q1, q2, p1, p2). Shared constants:
     * h, then the 3x3 tableau A column-major. n = 12. */
    GSB_FAMILY_IRK3_HENON_HEILES = 3,
    /* Test families of the reference's batch tests, with analytic Jacobians (prob.J). */
    GSB_FAMILY_HETERO6 = 100,  /* test/nonlinear/batched.jl:54-90; p = outcome 1..6; n = 2 */
    GSB_FAMILY_COUPLED2 = 101, /* test/nonlinear/batched.jl:92-104; p = (p1, p2); n = 2 */
    /* Families given by their residual alone, their Jacobian and JVP from forward-mode dual
     * passes on the device (src/ad/forwarddiff_static.jl:50-65, src/ad/jvp.jl:96-107):
     * Wood's function (problem 4 of test/helpers/standard_problems.jl) with the coupling weight
     * of its second and fourth residuals (20.2 there) as the one parameter, p = (w), n = 4; and
     * the cubic-affine family of GSB_FAMILY_CUBIC_AFFINE (same p) with the dual pass in place of
     * its written-out Jacobian, n in {2, 3, 4}. */
    GSB_FAMILY_WOOD = 102,
    GSB_FAMILY_CUBIC_AFFINE_DUAL = 103
} GsbFamily;

typedef struct {
    int32_t family;       /* GsbFamily */
    int32_t n;            /* unknowns */
    int32_t m;            /* residuals (m == n for a NonlinearProblem) */
    int32_t pad_;
    const double* shared; /* device pointer to the family's shared constants, or NULL */
    int64_t shared_len;
} GsbProblem;

/* The factor of a Newton step: partial-pivot LU (src/linear/static/lu.jl) or Householder QR
 * without pivoting (src/linear/static/qr.jl). For a square family GSB_QR runs with a Float64
 * factor (with or without Refinement) or a Float32 one (the mixed step), one thread per system,
 * n <= 8; a least-squares family's LevenbergMarquardt step takes its stacked QR. */
typedef enum { GSB_LU = 0, GSB_QR = 1 } GsbLinsolve;
typedef enum { GSB_F64 = 0, GSB_F32 = 1 } GsbPrecision;
typedef enum { GSB_NO_REFINEMENT = 0, GSB_REFINEMENT = 1 } GsbRefinementKind;
/* The rounding of the linear algebra (factorisation, solves, norms, products with the Jacobian).
 * GSB_FUSED contracts each product-and-sum into one fused multiply-add and divides by a pivot
 * through its reciprocal (the fast default; results agree with the reference to rounding);
 * GSB_UNFUSED rounds every product and every sum on its own, as Julia evaluates `a * b + c`, so
 * that a batch reproduces a CPU restatement of the reference bit for bit. Residual families fix
 * their own operation order and are the same under both. */
typedef enum { GSB_FUSED = 0, GSB_UNFUSED = 1 } GsbArithmetic;

typedef enum {
    GSB_STATIC = 0,
    GSB_BACKTRACKING = 1,
    GSB_LEVENBERG_MARQUARDT = 2,
    GSB_DOGLEG = 3
} GsbGlobalization;

/*
 * Newton (src/nonlinear/newton.jl:138-250) with the fields the batch path reads:
 *   linsolve + factor_precision  = LUFactorization{TF}() / QRFactorization{TF}()
 *   refinement                   = NoRefinement() / Refinement(eta, maxiter)
 *   globalization                = Static(alpha) / Backtracking(c1, p, maxiter) /
 *                                  LevenbergMarquardt(mu0, mu_min, mu_max, mu_decrease,
 *                                                     mu_increase, rho_accept; scaling = :none) /
 *                                  DogLeg(radius)
 *   reuse                        = Newton(reuse = k)
 * regularization must be 0 (the default); the matrix-free methods are not part of this ABI.
 * reuse >= 1 and DogLeg run with a Float64 LU factor, no refinement and one thread per system
 * (n <= 8); other combinations return GSB_ERR_UNSUPPORTED. `arithmetic` and
 * `threads_per_system` have no counterpart in the reference: they choose the device arithmetic
 * (GsbArithmetic) and how many lanes solve one system.
 */
typedef struct {
    int32_t linsolve;         /* GsbLinsolve */
    int32_t factor_precision; /* GsbPrecision */
    int32_t refinement;       /* GsbRefinementKind */
    int32_t refine_maxiter;
    double refine_eta;
    int32_t globalization;    /* GsbGlobalization */
    int32_t bt_maxiter;
    double static_alpha;
    double bt_c1;
    double bt_p;
    double lm_mu0;
    double lm_mu_min;
    double lm_mu_max;
    double lm_mu_decrease;
    double lm_mu_increase;
    double lm_rho_accept;
    double regularization;
    int32_t arithmetic;         /* GsbArithmetic */
    int32_t threads_per_system; /* lanes of a warp that share one system: 1, 2, 4, 8, 16 or 32;
                                   0 = the library's tuned choice for the family and size */
    int32_t reuse;              /* Newton(reuse = k): k >= 1; 0 = nothing (a fresh factor at
                                   every step) */
    int32_t trial_precision;    /* GsbPrecision of the line-search trials; no counterpart in the
                                   reference, whose trials are Float64 (GSB_F64, 0). GSB_F32 (with
                                   a Float32 LUFactorization, no reuse, Backtracking or Static,
                                   one thread per system, cubic-affine n in {2, 3, 4, 6, 8}) forms
                                   each trial's increment alpha d in Float32, added to the
                                   Float64 iterate, and takes the measured slope from the
                                   residual the step holds with a Float32 fold; the residual,
                                   its norm and every convergence test stay Float64. */
    double dogleg_radius;       /* DogLeg(radius): the initial trust radius, > 0; 0 = nothing
                                   (the first step sets it) */
} GsbMethod;

/* The six counts of the count form, src/nonlinear/batched.jl:197-199, by GsbReturnCode. */
typedef struct {
    int64_t counts[6];
} GsbTally;

/* BatchSummary{Float64} (src/nonlinear/batched.jl:63-69) with Julia's field layout: offsets
 * fnorm 0, all_converged 8 (Bool), failure_count 16, max_iterations 24 (Int32),
 * total_iterations 32; size 40, alignment 8. A Ref{BatchSummary{Float64}} is passed by pointer. */
typedef struct {
    double fnorm;
    uint8_t all_converged;
    uint8_t pad0_[7];
    int64_t failure_count;
    int32_t max_iterations;
    int32_t pad1_;
    int64_t total_iterations;
} GsbSummary;

/* Layouts of X (nsys iterates of n values) and P (nsys parameter blocks). */
typedef enum {
    GSB_AOS = 0, /* entry k of system s at base[s * len + k]: Julia's Vector{SVector} */
    GSB_SOA = 1  /* entry k of system s at base[k * nsys + s]: coalesced on the device */
} GsbLayout;

/* Forms of S. */
typedef enum {
    GSB_STATUS64 = 0, /* S is GsbStatus64[nsys] */
    GSB_CODES = 1     /* S is uint8_t[nsys] ReturnCodes; the count form */
} GsbStatusKind;

/* ABI version and the sm_100a device code of this build (1 when compiled for sm_100a). */
GSB_API int gsb_abi_version(void);

/* The last CUDA or argument error message of this thread, or "". */
GSB_API const char* gsb_last_error(void);

/* Number of parameters per system of `prob` (n*n+n for GSB_FAMILY_CUBIC_AFFINE, ...), or a
 * negative GsbError for an unknown family or size. */
GSB_API int64_t gsb_param_count(const GsbProblem* prob);

/* Options(Float64) defaults, src/base/options.jl:207-236. */
GSB_API void gsb_default_options(GsbOptions* opt);

/* Newton(; linsolve = LUFactorization(), globalization = Backtracking()) with the reference's
 * defaults for every field (Backtracking c1 = 1e-4, p = 0.5, maxiter = 100; Static alpha = 1;
 * Refinement eta = sqrt(eps), maxiter = 5; LevenbergMarquardt mu0 = 1e-6, mu_min = 1e-15,
 * mu_max = 1e12, mu_decrease = 1/3, mu_increase = 4, rho_accept = 0). */
GSB_API void gsb_default_method(GsbMethod* method);

/*
 * Solve every system in place: X[idx] is the start of system idx and becomes its final iterate;
 * S[idx] receives its status (s_kind GSB_STATUS64) or its code (GSB_CODES). P holds the
 * per-system parameter blocks (PerSystem), in p_layout. When `order` is not NULL it is a
 * permutation of 0..nsys-1 (order_base 0) or 1..nsys (order_base 1), and work item i solves
 * system order[i] (src/nonlinear/batched.jl:91-92, 171-179); a non-permutation is
 * GSB_ERR_ARGUMENT. When `tally` is not NULL (a host pointer) the call also returns the six
 * counts, which synchronises `stream`. An empty batch returns at once (batched.jl:285, 303).
 * Replaces solve_batch! (src/nonlinear/batched.jl:257-307).
 */
GSB_API int gsb_solve_batch(const GsbProblem* prob, const GsbMethod* method, const GsbOptions* opt,
                    double* X, int32_t x_layout, void* S, int32_t s_kind, const double* P,
                    int32_t p_layout, const int64_t* order, int32_t order_base, int64_t nsys,
                    void* stream, GsbTally* tally);

/* batch_summary(S) of nsys device statuses into *out (host), src/nonlinear/batched.jl:80-89.
 * Synchronises `stream`. */
GSB_API int gsb_batch_summary(const GsbStatus64* S, int64_t nsys, void* stream, GsbSummary* out);

/* solve_batch!(X, S, prob, method, p; order, options) followed by batch_summary(S) (src/nonlinear/
 * batched.jl:257-287 and 80-89), with the summary's reduction fused into the solve: each warp
 * adds up the statuses it closes (the sum of fnorm^2, the largest |fnorm|, the failures, the
 * largest and the total iteration count) and adds its part to the call's accumulator once, so
 * the statuses are not read back; only when the sum of squares leaves the normal range does a
 * second pass over S take rnorm's scaled sum. S is GsbStatus64[nsys] (device); *out (host) is
 * written; the call synchronises `stream`. Arguments and errors as gsb_solve_batch. */
GSB_API int gsb_solve_batch_summary(const GsbProblem* prob, const GsbMethod* method,
                                    const GsbOptions* opt, double* X, int32_t x_layout,
                                    GsbStatus64* S, const double* P, int32_t p_layout,
                                    const int64_t* order, int32_t order_base, int64_t nsys,
                                    void* stream, GsbSummary* out);

/* Wait for the work queued on `stream`. Returns GSB_ERR_CUDA if a batch kernel reported that a
 * bounded wait for its parameter staging copies ran out (its systems were then left unsolved; no
 * such wait is expected to run out). */
GSB_API int gsb_synchronize(void* stream);

/*
 * The count form of gsb_solve_batch for callers that cannot allocate device memory: a host whose
 * memory manager has reserved the whole device heap for its own pool, or a loop that cannot take
 * the device-wide synchronisation of cudaMalloc. It has no counterpart in the reference: it is
 * the count form with its working memory in a static device array of this library instead of
 * the allocator.
 *
 * It solves in place like gsb_solve_batch with s_kind GSB_CODES: X receives the iterates, `codes`
 * (uint8_t[nsys], device) the ReturnCodes, and *tally (host, required) the six counts. The six
 * counters, the permutation check of `order` and the kernel's staging-fault word live in one
 * static device array of this library (2 MiB, held by every device that loads the library until
 * the process exits), so a successful call allocates nothing: no cudaMalloc, no host heap (an
 * error's message text may allocate). Limit: with `order`, nsys may be at most
 * GSB_NOALLOC_MAX_ORDERED (16,777,216); beyond it the call returns GSB_ERR_DIMENSION before any
 * launch. Without `order` there is no limit. The first call on a device also looks up the
 * array's device address; make that first call before any stream capture on that device. Every
 * call reuses the same array (each call clears what it needs first), so calls that overlap on
 * the device race: issue them on one stream, or wait between them. The call returns after its
 * counts have reached the host.
 */
#define GSB_NOALLOC_MAX_ORDERED 16777216
GSB_API int gsb_solve_batch_counts_noalloc(const GsbProblem* prob, const GsbMethod* method,
                                           const GsbOptions* opt, double* X, int32_t x_layout,
                                           uint8_t* codes, const double* P, int32_t p_layout,
                                           const int64_t* order, int32_t order_base,
                                           int64_t nsys, void* stream, GsbTally* tally);

/* A batch whose X, S and P live in host memory (AoS layouts; page-locked memory lets the copies
 * overlap). No counterpart in the reference's device path: the call streams the batch through
 * the device in chunks of `chunk` systems (0: 262,144), on three streams, so that the copy of
 * chunk k+1's inputs, the solve of chunk k and the copy back of chunk k-1's iterates and statuses
 * overlap. `prob->shared` must still be a device pointer. Three device staging slots are
 * allocated on the first call on a device and kept. The call returns when every result is in
 * host memory; tally as in gsb_solve_batch. */
GSB_API int gsb_solve_batch_host(const GsbProblem* prob, const GsbMethod* method,
                                 const GsbOptions* opt, double* X, void* S, int32_t s_kind,
                                 const double* P, int64_t nsys, int64_t chunk, GsbTally* tally);

/* ─── ragged batches: systems of different sizes in one call ───────────────────────────────
 *
 * No counterpart in the reference, whose solve_batch! takes one size per call: a batch of
 * cubic-affine systems (GSB_FAMILY_CUBIC_AFFINE) whose sizes n[s] are drawn from the set
 * {2, 3, 4, 6, 8, 12, 16, 24, 32}, packed back to back: system s's iterate is X[x_off[s] ..
 * x_off[s] + n[s]) and its parameter block (A column-major, then b) is P[p_off[s] .. p_off[s] +
 * n[s]^2 + n[s]); its status is S[s] (72-byte status or 1-byte code, s_kind). The call buckets
 * the systems by size on the device, then runs one persistent kernel per bucket, each taking
 * CTA-sized chunks of its bucket from a device work queue; all of it is one CUDA graph, built
 * on the first call with a given set of arguments and replayed after. `table` (nullable) gives,
 * per bucket in the order of the sizes above, the threads per system (0: the default of the
 * size; 1 up to n = 8, or 2, 4, 8 lanes for n = 6 and 8 under fused arithmetic; 16 or 32 lanes
 * for n = 12 and 16; 32 for n = 24 and 32), the persistent CTAs per SM (0: as many as fit; -1:
 * no persistent kernel for the bucket but one ordinary grid, which the call launches from the
 * host once the bucketing has counted the bucket's systems, beside the graph) and the systems
 * per CTA of the warp form (n >= 12: a CTA of systems_per_cta x threads_per_system
 * lanes, a multiple of 32 and at most 128; 0: 128 lanes; the other forms take 0). The call
 * returns after the batch is solved; a size outside the set returns GSB_ERR_ARGUMENT (its
 * systems are left untouched). All pointers are device pointers.
 */
#define GSB_UNEVEN_BUCKETS 9
typedef struct {
    int32_t threads_per_system;
    int32_t ctas_per_sm;
    int32_t systems_per_cta;
    int32_t pad_;
} GsbBucketConfig;

GSB_API int gsb_uneven_sizes(int32_t* sizes_out /* GSB_UNEVEN_BUCKETS entries */);
GSB_API int gsb_solve_batch_uneven(const GsbMethod* method, const GsbOptions* opt, double* X,
                                   void* S, int32_t s_kind, const double* P, const int32_t* n,
                                   const int64_t* x_off, const int64_t* p_off, int64_t nsys,
                                   const GsbBucketConfig* table, void* stream, GsbTally* tally);

/* ─── the learned warm start of the stage systems (no counterpart in the reference) ────────── */

/* Self-test of the tensor-core tile product the warm-start network is built on: D (128 x N,
 * FP32, row-major) = A B^T for BF16 operands, A 128 x K and B N x K row-major (mode 0), or A
 * given as its K x 128 transpose and B as its K x N transpose (mode 1). 16 <= K <= 128 and
 * 16 <= N <= 256, multiples of 16. Device pointers; returns after the product is written. */
GSB_API int gsb_umma_selftest(const uint16_t* A, const uint16_t* B, float* D, int32_t K, int32_t N,
                              int32_t mode, void* stream);

/* The network: a 4 -> 128 -> 128 -> 12 MLP (GELU, BF16 weights and activations in the
 * tensor-core products, FP32 accumulation) giving the start Z0 = g(y) + scale * net((y - mean)
 * * inv_dev) of the Gauss-3 stage equations of a Hénon–Heiles state y, where g(y)_j = h c_j f(y)
 * is the explicit stage guess. theta holds gsb_mlp_sizes' theta_floats FP32 parameters: W1
 * [128][4], b1 [128], W2 [128][128] (in, out), b2 [128], W3 [128][16] (in, out; outputs 12..15
 * zero), b3 [16]; pack holds its BF16 copies (pack_halves), written by gsb_mlp_pack and
 * gsb_mlp_adam; norm holds mean (4), inv_dev (4), scale (12). `shared` is the stage family's
 * (h, A column-major). err_scratch is one device int. All pointers are device pointers. */
GSB_API int gsb_mlp_sizes(int64_t* theta_floats, int64_t* pack_halves);
GSB_API int gsb_mlp_pack(const float* theta, uint16_t* pack, void* stream);
/* Z0 (n x 12) for the states (n x 4); returns after Z0 is written. */
GSB_API int gsb_mlp_predict(const float* theta, const uint16_t* pack, const float* norm,
                            const double* shared, const double* states, double* Z0, int64_t n,
                            int* err_scratch, void* stream);
/* The gradient of the mean squared error of the network's output against `targets` (n x 12,
 * the scaled corrections (Z - g(y)) / scale) into grad (theta_floats), and the sum of squared
 * errors into loss; stream-ordered. */
GSB_API int gsb_mlp_grad(const float* theta, const uint16_t* pack, const float* norm,
                         const double* states, const float* targets, int64_t n, float* grad,
                         float* loss, int* err_scratch, void* stream);
/* One bias-corrected Adam step (step >= 1) on theta with moments m, v; refreshes pack. */
GSB_API int gsb_mlp_adam(float* theta, float* m, float* v, const float* grad, uint16_t* pack,
                         float lr, float beta1, float beta2, float eps, int32_t step, void* stream);
/* The accept-if-better gate: per system, X = the start (Z0 or Xdefault, n x 12) whose FP64
 * residual norm of the stage equations is smaller (Xdefault on ties and non-finite Z0), and
 * accepted = 1 where Z0 was taken. */
GSB_API int gsb_warm_start_select(const double* shared, const double* states, const double* Z0,
                                  const double* Xdefault, double* X, uint8_t* accepted, int64_t n,
                                  void* stream);

#ifdef __cplusplus
}
#endif

#endif /* GSB_H */
