"""gsb200 — B200-native batched nonlinear solves (the R2 regime of GeometricSolvers.jl).

Import it as ``import gsb200`` (the shim at the repository root). The solves run in libgsb.so,
CUDA kernels for sm_100a behind the C-ABI of include/gsb.h.
"""

from . import abi
from .abi import ReturnCode, SOLVER_STATUS_DTYPE, load_library
from .api import (
    ArgumentError,
    Backtracking,
    BatchParams,
    BatchSummary,
    CubicAffine,
    Coupled2,
    DimensionMismatch,
    DogLeg,
    ExpSum3,
    GaussNewton,
    Hetero6,
    IrkHenonHeiles,
    LeastSquaresProblem,
    LevenbergMarquardt,
    LUFactorization,
    Newton,
    NoRefinement,
    NonlinearProblem,
    Options,
    PerSystem,
    QRFactorization,
    Refinement,
    ReturnCodeCounts,
    SoA,
    Static,
    Wood,
    gauss3_tableau,
    isconverged,
    status_buffer,
    statuses,
)
from .batch import (batch_summary, ragged_offsets, solve_batch, solve_batch_host,
                    solve_batch_summary,
                    solve_batch_uneven)
from . import tune, warmstart
from .warmstart import MlpWarmStart

__all__ = [name for name in dir() if not name.startswith("_")]
