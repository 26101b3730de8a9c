"""The C-ABI library: it loads, exports every symbol include/gsb.h declares, and its structs have
the reference's layouts (CPU only: no call here touches a device)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    with open(os.path.join(ROOT, "include", "gsb.h")) as fh:
        return re.findall(r"GSB_API\s+[\w\s\*]+?\b(gsb_\w+)\s*\(", fh.read())


def test_header_and_exports(gsb):
    names = _declared()
    assert set(names) == set(gsb.abi.EXPORTED_SYMBOLS)
    lib = gsb.load_library()
    for name in names:
        assert hasattr(lib, name), name
    assert lib.gsb_abi_version() == 2


def test_status_layout(gsb):
    # SolverStatus{Float64}, src/base/status.jl:101-117
    S = gsb.abi.GsbStatus64
    offsets = {f: getattr(S, f).offset for f, _ in S._fields_}
    assert ctypes.sizeof(S) == 72
    assert [offsets[f] for f in ("code", "f_calls", "iterations", "fnorm", "stepnorm",
                                 "step_failures", "promoted", "stationary", "jvp_calls", "rank",
                                 "nullnorm", "gradratio", "rate", "contracted", "reused")] == \
        [0, 2, 4, 8, 16, 24, 28, 29, 30, 32, 40, 48, 56, 64, 65]
    assert gsb.SOLVER_STATUS_DTYPE.itemsize == 72


def test_summary_layout(gsb):
    # BatchSummary{Float64}, src/nonlinear/batched.jl:63-69: fnorm::Float64, all_converged::Bool,
    # failure_count::Int, max_iterations::Int32, total_iterations::Int (Julia's C layout)
    S = gsb.abi.GsbSummary
    offsets = {f: getattr(S, f).offset for f, _ in S._fields_}
    assert ctypes.sizeof(S) == 40
    assert [offsets[f] for f in ("fnorm", "all_converged", "failure_count", "max_iterations",
                                 "total_iterations")] == [0, 8, 16, 24, 32]


def test_defaults_match_reference(gsb):
    lib = gsb.load_library()
    o = gsb.abi.GsbOptions()
    lib.gsb_default_options(ctypes.byref(o))
    ref = gsb.Options().to_abi()
    for f, _ in o._fields_:
        if f != "pad_":
            assert getattr(o, f) == getattr(ref, f), f
    m = gsb.abi.GsbMethod()
    lib.gsb_default_method(ctypes.byref(m))
    mr = gsb.Newton(globalization=gsb.Backtracking()).to_abi()
    for f, _ in m._fields_:
        if f != "pad_":
            assert getattr(m, f) == pytest.approx(getattr(mr, f)), f


def test_param_counts(gsb):
    lib = gsb.load_library()
    for fam, expect in ((gsb.CubicAffine(8), 72), (gsb.CubicAffine(3), 12), (gsb.Hetero6(), 1),
                        (gsb.Coupled2(), 2), (gsb.IrkHenonHeiles(), 4)):
        p = gsb.NonlinearProblem(fam).to_abi()
        assert lib.gsb_param_count(ctypes.byref(p)) == expect == fam.param_count


def test_batch_params_form(gsb):
    # BatchParams of the cubic family (src/nonlinear/batched.jl:34-47): with the shared A in
    # `shared` (n^2 doubles) a system's block is b alone; other shared lengths keep (A, b)
    import numpy as np
    import torch

    _shared_matrix = gsb.batch._shared_matrix
    lib = gsb.load_library()
    A = torch.arange(64, dtype=torch.float64).reshape(8, 8)
    p = gsb.NonlinearProblem(gsb.CubicAffine(8)).to_abi()
    p.shared, p.shared_len = A.data_ptr(), 64
    assert lib.gsb_param_count(ctypes.byref(p)) == 8
    p.shared_len = 63
    assert lib.gsb_param_count(ctypes.byref(p)) == 72
    col = _shared_matrix(gsb.CubicAffine(8), A, torch.device("cpu"))
    assert np.array_equal(col.numpy(), A.numpy().flatten(order="F"))
    with pytest.raises(gsb.DimensionMismatch):
        _shared_matrix(gsb.CubicAffine(8), A[:4], torch.device("cpu"))
    with pytest.raises(gsb.ArgumentError):
        _shared_matrix(gsb.Coupled2(), A, torch.device("cpu"))
    with pytest.raises(gsb.ArgumentError):
        gsb.solve_batch_host(torch.zeros(4, 2, dtype=torch.float64), None,
                             gsb.NonlinearProblem(gsb.Coupled2()), gsb.Newton(),
                             gsb.BatchParams(A, torch.zeros(4, 2, dtype=torch.float64)))


def test_host_checks_refuse_before_any_launch(gsb):
    # constructor checks of the reference (src/base/options.jl:207-236, backtracking.jl:34-40,
    # newton.jl:160-176); a host tensor is refused (the solver has no host path)
    import torch

    with pytest.raises(gsb.ArgumentError):
        gsb.Options(f_abstol=-1.0)
    with pytest.raises(gsb.ArgumentError):
        gsb.Options(max_iterations=2, min_iterations=3)
    with pytest.raises(gsb.ArgumentError):
        gsb.Backtracking(c1=1.5)
    with pytest.raises(gsb.ArgumentError):
        gsb.Newton(globalization=gsb.LevenbergMarquardt(), refinement=gsb.Refinement())
    prob = gsb.NonlinearProblem(gsb.CubicAffine(3))
    X = torch.zeros(4, 3, dtype=torch.float64)
    P = gsb.PerSystem(torch.zeros(4, 12, dtype=torch.float64))
    with pytest.raises(gsb.ArgumentError):
        gsb.solve_batch(X, prob, gsb.Newton(), P)
