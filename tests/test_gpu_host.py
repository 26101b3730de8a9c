"""Batches in host memory (gsb_solve_batch_host): chunked, with the copies overlapping the
solves. The results must equal those of the device-resident call byte for byte (the same
kernels on the same inputs), for ragged chunk tails, the count form and a family with shared
constants."""

import numpy as np
import pytest

from workloads import c1, c2

pytestmark = pytest.mark.gpu


def _device_solve(gsb, prob, m, X0, P, opts):
    import torch

    X = torch.tensor(X0, device="cuda")
    S = gsb.status_buffer(X0.shape[0])
    gsb.solve_batch(X, S, prob, m, gsb.PerSystem(torch.tensor(P, device="cuda")), options=opts)
    return X.cpu().numpy(), S.cpu().numpy()


@pytest.mark.parametrize("chunk", [0, 65536, 100000, 10 ** 7])
def test_host_batch_equals_device_batch(gsb, chunk):
    import torch

    X0, P = c1(300000)
    prob = gsb.NonlinearProblem(gsb.CubicAffine(8))
    m = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    xd, sd = _device_solve(gsb, prob, m, X0, P, opts)
    Xh = torch.tensor(X0).pin_memory()
    Ph = torch.tensor(P).pin_memory()
    Sh = torch.empty((300000, 72), dtype=torch.uint8).pin_memory()
    gsb.solve_batch_host(Xh, Sh, prob, m, gsb.PerSystem(Ph), chunk=chunk, options=opts)
    assert Xh.numpy().tobytes() == xd.tobytes()
    assert Sh.numpy().tobytes() == sd.tobytes()
    # the count form, from unpinned host memory
    counts = gsb.solve_batch_host(torch.tensor(X0), None, prob, m, gsb.PerSystem(torch.tensor(P)),
                                  chunk=chunk, options=opts)
    assert list(counts) == np.bincount(gsb.statuses(torch.tensor(sd))["code"], minlength=6).tolist()


def test_host_batch_least_squares(gsb):
    import torch

    X0, Y, t = c2(20000)
    prob = gsb.LeastSquaresProblem(gsb.ExpSum3(t))
    m = gsb.Newton(linsolve=gsb.QRFactorization(), globalization=gsb.LevenbergMarquardt())
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    xd, sd = _device_solve(gsb, prob, m, X0, Y, opts)
    Xh = torch.tensor(X0)
    Sh = torch.empty((20000, 72), dtype=torch.uint8)
    gsb.solve_batch_host(Xh, Sh, prob, m, gsb.PerSystem(torch.tensor(Y)), chunk=6000, options=opts)
    assert Xh.numpy().tobytes() == xd.tobytes()
    assert Sh.numpy().tobytes() == sd.tobytes()
