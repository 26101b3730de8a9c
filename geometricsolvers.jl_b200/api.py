"""The host interface of the batch solver, mirroring GeometricSolvers.jl's R2 API.

Names, argument meaning and error behaviour follow the reference:
  solve_batch(X, S, prob, method, p; order, options, **kwargs) -> S      src/nonlinear/batched.jl:257-287
  solve_batch(X, prob, method, p; ...) -> counts                          src/nonlinear/batched.jl:289-307
  batch_summary(S) -> BatchSummary                                        src/nonlinear/batched.jl:80-89
  PerSystem(data)                                                         src/nonlinear/batched.jl:8-21
  Options(...)                                                            src/base/options.jl:207-236
  Newton / GaussNewton, LUFactorization(TF), QRFactorization(TF),
  Static, Backtracking, LevenbergMarquardt, Refinement, NoRefinement      (constructor checks cited)
Every solve runs on the device through libgsb (``abi.load_library``); there is no host fallback.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from decimal import Decimal, getcontext
from typing import NamedTuple, Optional

import numpy as np

from . import abi

EPS = float(np.finfo(np.float64).eps)
SQRT_EPS = math.sqrt(EPS)


class ArgumentError(ValueError):
    """The reference's ArgumentError: an invalid argument, refused on the host."""


class DimensionMismatch(ValueError):
    """The reference's DimensionMismatch: lengths that disagree."""


def _raise_for(rc: int, lib=None):
    if rc == 0:
        return
    msg = ""
    if lib is not None:
        raw = lib.gsb_last_error()
        msg = raw.decode() if raw else ""
    if rc == -1:
        raise DimensionMismatch(msg or "dimension mismatch")
    if rc == -2:
        raise ArgumentError(msg or "invalid argument")
    if rc == -3:
        raise ArgumentError(msg or "unsupported combination")
    raise RuntimeError(f"libgsb error {rc}: {msg}")


# ─── Options, src/base/options.jl:58-71 and 207-245 ─────────────────────────────────────────


def _nonnegative(name, tol):
    if not (tol >= 0):  # NaN fails
        raise ArgumentError(f"{name} must be non-negative, got {tol}")


@dataclass(frozen=True)
class Options:
    f_abstol: float = 0.0
    f_reltol: float = SQRT_EPS
    x_abstol: float = 0.0
    x_reltol: float = 2 * EPS
    min_iterations: int = 0
    max_iterations: int = 100
    max_stalls: int = 2
    g_tol: float = SQRT_EPS
    norm: str = "l2"
    kappa: float = 0.1
    roundoff: bool = False
    rate_test: bool = True

    def __post_init__(self):
        for name in ("f_abstol", "f_reltol", "x_abstol", "x_reltol", "g_tol"):
            _nonnegative(name, getattr(self, name))
        if self.min_iterations < 0:
            raise ArgumentError(f"min_iterations must be non-negative, got {self.min_iterations}")
        if self.max_iterations < self.min_iterations:
            raise ArgumentError(
                f"max_iterations = {self.max_iterations} is below min_iterations = {self.min_iterations}"
            )
        if self.max_stalls < 1:
            raise ArgumentError(f"max_stalls must be at least 1, got {self.max_stalls}")
        if not (0.0 < self.kappa < 1.0):
            raise ArgumentError("kappa must be finite and in (0, 1)")
        if self.norm not in ("l2", "max"):
            raise ArgumentError(f"norm must be 'l2' or 'max', got {self.norm!r}")

    def to_abi(self) -> abi.GsbOptions:
        o = abi.GsbOptions()
        o.f_abstol, o.f_reltol = self.f_abstol, self.f_reltol
        o.x_abstol, o.x_reltol = self.x_abstol, self.x_reltol
        o.min_iterations, o.max_iterations = self.min_iterations, self.max_iterations
        o.max_stalls = self.max_stalls
        o.norm = 0 if self.norm == "l2" else 1
        o.g_tol, o.kappa = self.g_tol, self.kappa
        o.roundoff, o.rate_test = int(self.roundoff), int(self.rate_test)
        return o


# ─── linear methods, src/linear/methods.jl:37-258 ───────────────────────────────────────────


def _precision(TF):
    if TF is None or TF in ("float64", np.float64, "Float64"):
        return abi.GSB_F64
    if TF in ("float32", np.float32, "Float32"):
        return abi.GSB_F32
    raise ArgumentError(f"factor precision must be None, 'float64' or 'float32', got {TF!r}")


@dataclass(frozen=True)
class LUFactorization:
    TF: Optional[str] = None


@dataclass(frozen=True)
class QRFactorization:
    TF: Optional[str] = None


# ─── globalizations ─────────────────────────────────────────────────────────────────────────


@dataclass(frozen=True)
class Static:
    """Static(α = 1.0), src/globalization/static.jl:8-20."""

    alpha: float = 1.0

    def __post_init__(self):
        if not (self.alpha > 0 and math.isfinite(self.alpha)):
            raise ArgumentError("the step of Static must be positive and finite")


@dataclass(frozen=True)
class Backtracking:
    """Backtracking(; c₁ = 1e-4, p = 0.5, maxiter = 100), src/globalization/backtracking.jl:28-48."""

    c1: float = 1e-4
    p: float = 0.5
    maxiter: int = 100

    def __post_init__(self):
        if not (0 < self.c1 < 1):
            raise ArgumentError("Backtracking needs 0 < c₁ < 1")
        if not (0 < self.p < 1):
            raise ArgumentError("Backtracking needs 0 < p < 1")
        if not (1 <= self.maxiter <= 2**31 - 1):
            raise ArgumentError("Backtracking needs 1 ≤ maxiter ≤ typemax(Int32)")


@dataclass(frozen=True)
class DogLeg:
    """DogLeg(; radius = nothing), src/globalization/dogleg.jl:1-60: the trust-region
    globalization on the dogleg curve (Procedure 4.1 of Pawlowski, Simonis, Walker and Shadid
    2008). `radius` is the initial trust radius, positive and finite, clamped to [1e-6, 1e10];
    None lets the first step set it from the first Newton (or Cauchy) step."""

    radius: Optional[float] = None

    def __post_init__(self):
        if self.radius is not None:
            if not (self.radius > 0 and math.isfinite(self.radius)):
                raise ArgumentError("the radius of DogLeg must be positive and finite")
            object.__setattr__(self, "radius", min(max(float(self.radius), 1e-6), 1e10))


@dataclass(frozen=True)
class LevenbergMarquardt:
    """LevenbergMarquardt(; μ₀, μ_min, μ_max, μ_decrease, μ_increase, ρ_accept, scaling),
    src/globalization/levenbergmarquardt.jl:48-98 (the stacked QR path, scaling = :none)."""

    mu0: float = 1e-6
    mu_min: float = max(1e-15, 4 * EPS)
    mu_max: float = 1e12
    mu_decrease: float = 1.0 / 3.0
    mu_increase: float = 4.0
    rho_accept: float = 0.0
    scaling: str = "none"

    def __post_init__(self):
        fin = all(math.isfinite(v) for v in (self.mu0, self.mu_min, self.mu_max))
        if not (fin and 0 < self.mu_min <= self.mu0 <= self.mu_max):
            raise ArgumentError(
                "LevenbergMarquardt requires finite damping bounds 0 < μ_min ≤ μ₀ ≤ μ_max < Inf"
            )
        if not (math.isfinite(self.mu_decrease) and 0 < self.mu_decrease < 1):
            raise ArgumentError("LevenbergMarquardt requires 0 < μ_decrease < 1")
        if not (math.isfinite(self.mu_increase) and self.mu_increase > 1):
            raise ArgumentError("LevenbergMarquardt requires μ_increase > 1")
        if not (math.isfinite(self.rho_accept) and 0 <= self.rho_accept < 1):
            raise ArgumentError("LevenbergMarquardt requires 0 ≤ ρ_accept < 1")
        if self.scaling not in ("none", "diagonal"):
            raise ArgumentError("LevenbergMarquardt requires scaling ∈ (:none, :diagonal)")


# ─── refinement, src/nonlinear/refinement.jl:1-47 ───────────────────────────────────────────


@dataclass(frozen=True)
class NoRefinement:
    pass


@dataclass(frozen=True)
class Refinement:
    eta: float = SQRT_EPS
    maxiter: int = 5

    def __post_init__(self):
        if self.maxiter < 1:
            raise ArgumentError("Refinement maxiter must be ≥ 1")
        if not (math.isfinite(self.eta) and 0 < self.eta < 1):
            raise ArgumentError("Refinement η must be finite and in (0, 1)")


# ─── Newton, src/nonlinear/newton.jl:138-250 ────────────────────────────────────────────────


@dataclass(frozen=True)
class Newton:
    linsolve: object = LUFactorization()
    globalization: object = Static()
    refinement: object = NoRefinement()
    regularization: float = 0.0
    reuse: Optional[int] = None
    # The rounding of the linear algebra on the device: "fused" (FMA, the default) or
    # "unfused" (every product and sum rounded alone, as Julia evaluates); no reference field.
    arithmetic: str = "fused"
    # Lanes of a warp that share one system on the device (1, 2, 4, 8, 16, 32), or None for the
    # library's tuned choice; no reference field.
    threads_per_system: Optional[int] = None
    # The precision of the line-search trials: None (Float64, the reference's) or "float32" (a
    # departure with no reference field: each trial's increment alpha d in Float32 and the
    # measured slope from the held residual; residuals, norms and tests stay Float64). Takes a
    # Float32 LUFactorization, no reuse, Backtracking or Static.
    trial: Optional[str] = None

    def __post_init__(self):
        if self.arithmetic not in ("fused", "unfused"):
            raise ArgumentError("arithmetic must be 'fused' or 'unfused'")
        if self.trial not in (None, "float64", "float32"):
            raise ArgumentError("trial must be None, 'float64' or 'float32'")
        if self.trial == "float32":
            if not (isinstance(self.linsolve, LUFactorization)
                    and _precision(self.linsolve.TF) == abi.GSB_F32):
                raise ArgumentError("Float32 line-search trials go with LUFactorization('float32')")
            if self.reuse is not None or not isinstance(self.globalization, (Backtracking, Static)):
                raise ArgumentError("Float32 line-search trials take no reuse and Backtracking "
                                    "or Static")
        if self.threads_per_system not in (None, 1, 2, 4, 8, 16, 32):
            raise ArgumentError("threads_per_system must be None or one of 1, 2, 4, 8, 16, 32")
        if isinstance(self.refinement, bool):
            object.__setattr__(self, "refinement", Refinement() if self.refinement else NoRefinement())
        if not (self.regularization >= 0 and math.isfinite(self.regularization)):
            raise ArgumentError("Newton regularization must be finite and ≥ 0")
        if self.reuse is not None:
            if self.reuse < 1:
                raise ArgumentError("Newton reuse must be ≥ 1 or nothing")
            if isinstance(self.globalization, LevenbergMarquardt):
                raise ArgumentError("Newton with a LevenbergMarquardt globalization takes no reuse")
            if isinstance(self.globalization, DogLeg):
                raise ArgumentError("DogLeg takes no factor reuse")
        if isinstance(self.globalization, LevenbergMarquardt) and isinstance(self.refinement, Refinement):
            raise ArgumentError(
                "Newton with a LevenbergMarquardt globalization takes no refinement: a refinement "
                "corrects the solve of J d = -F, which the damped step does not take; use "
                "refinement = NoRefinement()"
            )

    def to_abi(self) -> abi.GsbMethod:
        m = abi.GsbMethod()
        ls = self.linsolve
        if isinstance(ls, LUFactorization):
            m.linsolve = abi.GSB_LU
        elif isinstance(ls, QRFactorization):
            m.linsolve = abi.GSB_QR
        else:
            raise ArgumentError(f"unsupported linear method {ls!r}: LUFactorization or QRFactorization")
        m.factor_precision = _precision(ls.TF)
        ref = self.refinement
        if isinstance(ref, Refinement):
            m.refinement, m.refine_eta, m.refine_maxiter = abi.GSB_REFINEMENT, ref.eta, ref.maxiter
        else:
            m.refinement, m.refine_eta, m.refine_maxiter = abi.GSB_NO_REFINEMENT, SQRT_EPS, 5
        g = self.globalization
        m.static_alpha, m.bt_c1, m.bt_p, m.bt_maxiter = 1.0, 1e-4, 0.5, 100
        lm = LevenbergMarquardt()
        if isinstance(g, Static):
            m.globalization, m.static_alpha = abi.GSB_STATIC, g.alpha
        elif isinstance(g, Backtracking):
            m.globalization = abi.GSB_BACKTRACKING
            m.bt_c1, m.bt_p, m.bt_maxiter = g.c1, g.p, g.maxiter
        elif isinstance(g, LevenbergMarquardt):
            m.globalization = abi.GSB_LEVENBERG_MARQUARDT
            if g.scaling != "none":
                raise ArgumentError("the batch LevenbergMarquardt step takes scaling = :none")
            lm = g
        elif isinstance(g, DogLeg):
            m.globalization = abi.GSB_DOGLEG
        else:
            raise ArgumentError(f"unsupported globalization {g!r}")
        m.lm_mu0, m.lm_mu_min, m.lm_mu_max = lm.mu0, lm.mu_min, lm.mu_max
        m.lm_mu_decrease, m.lm_mu_increase, m.lm_rho_accept = lm.mu_decrease, lm.mu_increase, lm.rho_accept
        if self.regularization != 0.0:
            raise ArgumentError("the batch path takes regularization = 0")
        m.reuse = 0 if self.reuse is None else int(self.reuse)
        m.dogleg_radius = (g.radius or 0.0) if isinstance(g, DogLeg) else 0.0
        m.trial_precision = abi.GSB_F32 if self.trial == "float32" else abi.GSB_F64
        m.regularization = 0.0
        m.arithmetic = abi.GSB_FUSED if self.arithmetic == "fused" else abi.GSB_UNFUSED
        m.threads_per_system = 0 if self.threads_per_system is None else self.threads_per_system
        return m


def GaussNewton(linsolve=QRFactorization(), globalization=Static(), refinement=NoRefinement()):
    """GaussNewton(; linsolve = QRFactorization(), ...), src/nonlinear/leastsquares.jl:72-90."""
    return Newton(linsolve=linsolve, globalization=globalization, refinement=refinement)


# ─── residual families and problems ─────────────────────────────────────────────────────────


def gauss3_tableau() -> np.ndarray:
    """The 3-stage Gauss–Legendre collocation matrix, from the closed form with c = 1/2 ∓ √15/10,
    1/2, evaluated in 50-digit decimals and rounded once to Float64 (as the reference's
    test/helpers/stage_problems.jl:152-168 computes A in BigFloat and rounds once)."""
    getcontext().prec = 50
    r = Decimal(15).sqrt()
    f = Decimal
    A = [
        [f(5) / 36, f(2) / 9 - r / 15, f(5) / 36 - r / 30],
        [f(5) / 36 + r / 24, f(2) / 9, f(5) / 36 - r / 24],
        [f(5) / 36 + r / 30, f(2) / 9 + r / 15, f(5) / 36],
    ]
    return np.array([[float(v) for v in row] for row in A], dtype=np.float64)


class Family:
    family: int
    n: int
    m: int
    lsq = False

    def shared(self) -> Optional[np.ndarray]:
        return None

    @property
    def param_count(self) -> int:
        raise NotImplementedError


class CubicAffine(Family):
    """F(x, p) = A x + 0.1 x.^3 - b with p = (A column-major n×n, b). jacobian = "rule" (the
    default) takes the family's written-out Jacobian; jacobian = "dual" takes the device's
    generic forward-mode dual pass over the residual (n in 2, 3, 4), the same bits."""

    family = abi.Family.CUBIC_AFFINE

    def __init__(self, n: int, jacobian: str = "rule"):
        if not (1 <= n <= 32):
            raise ArgumentError(f"CubicAffine takes 1 ≤ n ≤ 32, got {n}")
        if jacobian not in ("rule", "dual"):
            raise ArgumentError("jacobian must be 'rule' or 'dual'")
        if jacobian == "dual":
            if not (2 <= n <= 4):
                raise ArgumentError("the dual-pass CubicAffine takes n in 2, 3, 4")
            self.family = abi.Family.CUBIC_AFFINE_DUAL
        self.n = self.m = n

    @property
    def param_count(self):
        return self.n * self.n + self.n


class ExpSum3(Family):
    """r_i = Σ_j a_j exp(-b_j t_i) - y_i, x = (a1, b1, a2, b2, a3, b3), p = y."""

    family = abi.Family.EXPSUM3_LSQ
    lsq = True

    def __init__(self, t=None):
        self.t = np.linspace(0.0, 4.0, 64) if t is None else np.asarray(t, dtype=np.float64)
        if self.t.shape != (64,):
            raise ArgumentError("ExpSum3 takes 64 abscissae")
        self.n, self.m = 6, 64

    def shared(self):
        return self.t

    @property
    def param_count(self):
        return self.m


class IrkHenonHeiles(Family):
    """Gauss–Legendre 3-stage stage equations Z - h (A ⊗ I) f(y + Z) of the Hénon–Heiles field,
    x = Z (12), p = y (4)."""

    family = abi.Family.IRK3_HENON_HEILES

    def __init__(self, h: float = 0.1):
        self.h = float(h)
        self.A = gauss3_tableau()
        self.n = self.m = 12

    def shared(self):
        return np.concatenate([[self.h], self.A.flatten(order="F")])

    @property
    def param_count(self):
        return 4


class Hetero6(Family):
    """The six-outcome residual of test/nonlinear/batched.jl:54-90; p = outcome 1..6."""

    family = abi.Family.HETERO6

    def __init__(self):
        self.n = self.m = 2

    @property
    def param_count(self):
        return 1


class Coupled2(Family):
    """The coupled residual of test/nonlinear/batched.jl:92-104; p = (p1, p2)."""

    family = abi.Family.COUPLED2

    def __init__(self):
        self.n = self.m = 2

    @property
    def param_count(self):
        return 2


class Wood(Family):
    """Wood's function (problem 4 of test/helpers/standard_problems.jl) with the coupling weight
    w of its second and fourth residuals (20.2 in the standard problem) per system, p = (w,). A
    family given by its residual alone: the device takes its Jacobian and JVP from dual passes."""

    family = abi.Family.WOOD

    def __init__(self):
        self.n = self.m = 4

    @property
    def param_count(self):
        return 1


class NonlinearProblem:
    """NonlinearProblem(F), src/nonlinear/problem.jl:81-110, with F a residual family."""

    def __init__(self, family: Family):
        if family.lsq:
            raise ArgumentError("a least-squares family is a LeastSquaresProblem")
        self.family = family
        self._shared_dev = {}

    def to_abi(self, shared_ptr=None) -> abi.GsbProblem:
        p = abi.GsbProblem()
        p.family, p.n, p.m = int(self.family.family), self.family.n, self.family.m
        sh = self.family.shared()
        p.shared = shared_ptr
        p.shared_len = 0 if sh is None else len(sh)
        return p

    def shared_device(self, device):
        """The family's shared constants as a float64 tensor on `device` (None for a family
        without them). Cached per device and per value of the constants, so a family whose
        constants change (a new step h, a new grid t) gets a fresh copy."""
        import torch

        sh = self.family.shared()
        if sh is None:
            return None
        sh = np.ascontiguousarray(np.asarray(sh, dtype=np.float64))
        dkey = (device.type, device.index) if isinstance(device, torch.device) else str(device)
        key = (dkey, sh.tobytes())
        v = self._shared_dev.get(key)
        if v is None:
            if len(self._shared_dev) > 64:
                self._shared_dev.clear()
            v = self._shared_dev[key] = torch.tensor(sh, dtype=torch.float64, device=device)
        return v


class LeastSquaresProblem(NonlinearProblem):
    """LeastSquaresProblem(F, m), src/nonlinear/leastsquares.jl:19-60."""

    def __init__(self, family: Family):
        if not family.lsq:
            raise ArgumentError("LeastSquaresProblem takes a least-squares family")
        self.family = family
        self._shared_dev = {}


# ─── batch containers ───────────────────────────────────────────────────────────────────────


class SoA:
    """A batch stored entry-major: `data[k, s]` is entry k of system s (coalesced on the device)."""

    def __init__(self, data):
        self.data = data


class PerSystem:
    """PerSystem(data), src/nonlinear/batched.jl:8-21: system i receives data[i]. `data` is a
    (nsys, np) tensor, or SoA of an (np, nsys) tensor."""

    def __init__(self, data):
        self.data = data


class BatchParams:
    """BatchParams(shared, per_system), src/nonlinear/batched.jl:34-47: system i receives
    (shared, per_system[i]). For CubicAffine, `shared` is the batch's n×n matrix A (a float64
    tensor on the device of X, or anything numpy takes) and `per_system` the right-hand sides b,
    an (nsys, n) tensor or SoA of an (n, nsys) tensor."""

    def __init__(self, shared, per_system):
        self.shared = shared
        self.per_system = per_system


class ReturnCodeCounts(NamedTuple):
    SUCCESS: int
    STALLED: int
    MAXITERS: int
    SINGULAR: int
    NONFINITE: int
    LINESEARCH_FAILED: int


def isconverged(counts: ReturnCodeCounts) -> bool:
    """isconverged(counts), src/base/status.jl:276-277."""
    return counts.SUCCESS == sum(counts)


class BatchSummary(NamedTuple):
    """BatchSummary{Float64}, src/nonlinear/batched.jl:63-69."""

    fnorm: float
    all_converged: bool
    failure_count: int
    max_iterations: int
    total_iterations: int


def status_buffer(nsys: int, device="cuda"):
    """An uninitialised Vector{SolverStatus{Float64}} of nsys entries: a (nsys, 72) uint8 tensor."""
    import torch

    return torch.empty((nsys, 72), dtype=torch.uint8, device=device)


def statuses(S) -> np.ndarray:
    """The statuses S (a (nsys, 72) uint8 tensor or array) as a numpy structured array."""
    arr = S.detach().cpu().numpy() if hasattr(S, "detach") else np.asarray(S)
    return np.ascontiguousarray(arr).view(abi.SOLVER_STATUS_DTYPE).reshape(-1)
