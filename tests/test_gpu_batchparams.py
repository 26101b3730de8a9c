"""BatchParams(shared, per_system) (src/nonlinear/batched.jl:34-47): the cubic-affine batch with
one matrix A shared by every system and a right-hand side b per system, n = 2 … 8 (one thread per
system) and 12 … 32 (the warp form).

The device stages A once per CTA and streams only b; the oracle solves the same batch with A
replicated into every system's (A, b) block, so the two must agree exactly as the per-system
form does: bit for bit under the unfused arithmetic, codes, iteration counts and 1e-10 under the
fused one.
"""

import numpy as np
import pytest

from test_gpu_parity import OPTS, _dev, check_parity
from workloads import rng

pytestmark = pytest.mark.gpu


def shared_batch(n, nsys, diag, config_id, illcond=False):
    """(X0, A (n, n), B (nsys, n), P (nsys, n*n + n) with A replicated column-major)."""
    g = rng(config_id, 7)
    A = g.standard_normal((n, n)) * 0.5
    A[np.arange(n), np.arange(n)] += diag
    if illcond:  # a graded spectrum: the FP32 factor needs refinement, some systems promote
        U, _, Vt = np.linalg.svd(A)
        A = (U * np.logspace(0, -7, n)) @ Vt
    B = g.uniform(-1.0, 1.0, (nsys, n)) * (1.0 + 3.0 * g.uniform(0.0, 1.0, (nsys, 1)))
    P = np.concatenate([np.broadcast_to(A.T.reshape(1, n * n), (nsys, n * n)), B], axis=1)
    return np.zeros((nsys, n)), A, np.ascontiguousarray(B), np.ascontiguousarray(P)


def run_shared(gsb, prob, method, X0, A, B, options, soa=False, host=False):
    import torch

    if host:
        X = torch.tensor(X0, dtype=torch.float64)
        S = torch.zeros((X0.shape[0], 72), dtype=torch.uint8)
        gsb.solve_batch_host(X, S, prob, method, gsb.BatchParams(A, torch.tensor(B)),
                             chunk=X0.shape[0] // 3 + 1, options=options)
        return X.numpy(), gsb.statuses(S)
    X = _dev(X0.T if soa else X0)
    Bd = _dev(B.T if soa else B)
    S = gsb.status_buffer(X0.shape[0])
    gsb.solve_batch(gsb.SoA(X) if soa else X, S, prob, method,
                    gsb.BatchParams(_dev(A), gsb.SoA(Bd) if soa else Bd), options=options)
    x = X.cpu().numpy()
    return (x.T if soa else x), gsb.statuses(S)


@pytest.mark.parametrize("arith", ["fused", "unfused"])
@pytest.mark.parametrize("n", [2, 3, 4, 6, 8, 12, 16, 24, 32])
def test_shared_matrix_parity(gsb, oracle, n, arith):
    X0, A, B, P = shared_batch(n, 40000 if n <= 8 else 4096, n + 1.0, 10 + n)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic=arith)
    opts = gsb.Options(**OPTS)
    xg, sg = run_shared(gsb, prob, m, X0, A, B, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xg, sg, xo, so, bitwise=(arith == "unfused"))
    assert np.all(so["code"] == 0)


@pytest.mark.parametrize("n", [4, 8, 12, 32])
def test_shared_matrix_mixed_refinement(gsb, oracle, n):
    # FP32 factor + FP64 refinement with the shared A, on a graded spectrum that promotes
    X0, A, B, P = shared_batch(n, 20000 if n <= 8 else 2048, 0.0, 20 + n, illcond=True)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(linsolve=gsb.LUFactorization("float32"), refinement=gsb.Refinement(),
                   globalization=gsb.Backtracking(), arithmetic="unfused")
    opts = gsb.Options(**OPTS)
    xg, sg = run_shared(gsb, prob, m, X0, A, B, opts)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    check_parity(xg, sg, xo, so, bitwise=True)


def test_shared_matrix_soa_and_host(gsb, oracle):
    n = 8
    X0, A, B, P = shared_batch(n, 30001, 6.0, 31)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(n))
    m = gsb.Newton(globalization=gsb.Backtracking(), arithmetic="unfused")
    opts = gsb.Options(**OPTS)
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    for kw in (dict(soa=True), dict(host=True)):
        xg, sg = run_shared(gsb, prob, m, X0, A, B, opts, **kw)
        check_parity(xg, sg, xo, so, bitwise=True)


def test_shared_matrix_unsupported_and_mismatch(gsb):
    import torch

    # a size without a kernel of its own (n = 10) is refused with a shared A as without one
    prob = gsb.NonlinearProblem(gsb.CubicAffine(10))
    X = torch.zeros((64, 10), dtype=torch.float64, device="cuda")
    S = gsb.status_buffer(64)
    A = torch.eye(10, dtype=torch.float64, device="cuda")
    B = torch.ones((64, 10), dtype=torch.float64, device="cuda")
    with pytest.raises(Exception, match="no batch kernel"):
        gsb.solve_batch(X, S, prob, gsb.Newton(), gsb.BatchParams(A, B))
    prob8 = gsb.NonlinearProblem(gsb.CubicAffine(8))
    X8 = torch.zeros((64, 8), dtype=torch.float64, device="cuda")
    with pytest.raises(gsb.DimensionMismatch):
        gsb.solve_batch(X8, S, prob8, gsb.Newton(), gsb.BatchParams(A, B[:, :8]))
    with pytest.raises(gsb.DimensionMismatch):
        gsb.solve_batch(X8, S, prob8, gsb.Newton(), gsb.BatchParams(A[:8, :8], B))
    # a team of threads per system reads whole (A, b) blocks: refused with a shared A
    with pytest.raises(Exception, match="no batch kernel"):
        gsb.solve_batch(X8, S, prob8, gsb.Newton(threads_per_system=4),
                        gsb.BatchParams(A[:8, :8].contiguous(), B[:, :8].contiguous()))
