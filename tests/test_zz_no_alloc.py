"""The allocation-free count form, gsb_solve_batch_counts_noalloc, called through the C-ABI.

Some callers cannot allocate device memory: a host whose memory manager has reserved the whole
device heap for its own pool, or a loop that cannot take cudaMalloc's device-wide
synchronisation. This entry point keeps its counters and its check of `order` in a static
device array of the library instead. Each check here compares it with the count form of
gsb_solve_batch on the same inputs, on two calls in a row (the second call must not see what the
first one left in the shared array).
"""

import ctypes

import numpy as np
import pytest

from workloads import c1

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10


def _dev(a):
    import torch

    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")


def _call(gsb, fn, prob, method, opts, X, codes, P, order=None, noalloc=True):
    import torch

    lib = gsb.load_library()
    gp = prob.to_abi(None)
    gm = method.to_abi()
    go = opts.to_abi()
    tally = gsb.abi.GsbTally()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    order_ptr = None if order is None else order.data_ptr()
    if noalloc:
        rc = lib.gsb_solve_batch_counts_noalloc(
            ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), X.data_ptr(), gsb.abi.GSB_AOS,
            codes.data_ptr(), P.data_ptr(), gsb.abi.GSB_AOS, order_ptr, 0, X.shape[0], stream,
            ctypes.byref(tally))
    else:
        rc = lib.gsb_solve_batch(
            ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), X.data_ptr(), gsb.abi.GSB_AOS,
            codes.data_ptr(), gsb.abi.GSB_CODES, P.data_ptr(), gsb.abi.GSB_AOS, order_ptr, 0,
            X.shape[0], stream, ctypes.byref(tally))
    torch.cuda.synchronize()
    return rc, [int(c) for c in tally.counts]


def _rel_err(x, xr):
    num = np.max(np.abs(x - xr), axis=1)
    den = np.max(np.abs(xr), axis=1)
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(den > 0, num / den, num)


def _compare(gsb, prob, method, opts, X0, P, order=None):
    import torch

    Pd = _dev(P)
    X_ref = _dev(X0)
    c_ref = torch.empty(X0.shape[0], dtype=torch.uint8, device="cuda")
    rc, counts_ref = _call(gsb, None, prob, method, opts, X_ref, c_ref, Pd, order, noalloc=False)
    assert rc == 0
    for _ in range(2):  # two calls in a row
        X = _dev(X0)
        codes = torch.full((X0.shape[0],), 255, dtype=torch.uint8, device="cuda")
        rc, counts = _call(gsb, None, prob, method, opts, X, codes, Pd, order)
        assert rc == 0, gsb.load_library().gsb_last_error()
        assert counts == counts_ref
        assert sum(counts) == X0.shape[0]
        assert torch.equal(codes, c_ref)
        x, xr = X.cpu().numpy(), X_ref.cpu().numpy()
        ok = c_ref.cpu().numpy() == 0
        assert np.all(_rel_err(x[ok], xr[ok]) <= REL_TOL)


def test_noalloc_counts_match_count_form(gsb):
    X0, P = c1(50000)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(8))
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    for method in (gsb.Newton(globalization=gsb.Backtracking()),
                   gsb.Newton(linsolve=gsb.LUFactorization("float32"),
                              refinement=gsb.Refinement(), globalization=gsb.Backtracking())):
        _compare(gsb, prob, method, opts, X0, P)


def test_noalloc_six_outcomes_and_order(gsb):
    import torch

    codes = [1, 2, 3, 4, 5, 6, 1, 3] * 64
    X0 = np.array([[2.5, 3.5]] * len(codes))
    P = np.array(codes, float)[:, None]
    prob = gsb.NonlinearProblem(gsb.Hetero6())
    method = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(max_iterations=3)
    _compare(gsb, prob, method, opts, X0, P)
    perm = torch.tensor(np.random.default_rng(3).permutation(len(codes)), dtype=torch.int64,
                        device="cuda")
    _compare(gsb, prob, method, opts, X0, P, order=perm)


def test_noalloc_rejections(gsb):
    import torch

    prob = gsb.NonlinearProblem(gsb.Coupled2())
    method = gsb.Newton()
    opts = gsb.Options()
    X = _dev(np.zeros((4, 2)))
    P = _dev(np.ones((4, 2)))
    codes = torch.zeros(4, dtype=torch.uint8, device="cuda")
    dup = torch.tensor([0, 1, 1, 3], dtype=torch.int64, device="cuda")
    rc, _ = _call(gsb, None, prob, method, opts, X, codes, P, dup)
    assert rc == -2
    # an ordered batch above the limit is refused before anything is read or launched
    lib = gsb.load_library()
    gp, gm, go = prob.to_abi(None), method.to_abi(), opts.to_abi()
    tally = gsb.abi.GsbTally()
    rc = lib.gsb_solve_batch_counts_noalloc(
        ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), X.data_ptr(), 0, codes.data_ptr(),
        P.data_ptr(), 0, dup.data_ptr(), 0, 16777217, None, ctypes.byref(tally))
    assert rc == -1
    # after a refused call the next one starts clean
    good = torch.tensor([3, 2, 1, 0], dtype=torch.int64, device="cuda")
    rc, counts = _call(gsb, None, prob, method, opts, X, codes, P, good)
    assert rc == 0 and sum(counts) == 4
