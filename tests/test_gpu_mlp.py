"""The tensor-core tile product under the warm-start network (tcgen05, BF16 operands from
shared memory, FP32 accumulation in tensor memory), against a float64 product of the same
BF16-rounded operands: K-major operands (the forward and input-gradient products) and
MN-major operands (the weight-gradient products, which read activation tiles transposed)."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _selftest(gsb, K, N, mode, seed):
    import torch

    lib = gsb.load_library()
    g = torch.Generator().manual_seed(seed)
    if mode == 0:
        A = torch.randn(128, K, generator=g).to(torch.bfloat16)
        B = torch.randn(N, K, generator=g).to(torch.bfloat16)
        ref = A.double() @ B.double().T
    else:
        A = torch.randn(K, 128, generator=g).to(torch.bfloat16)   # A^T
        B = torch.randn(K, N, generator=g).to(torch.bfloat16)     # B^T
        ref = A.double().T @ B.double()
    Ad, Bd = A.cuda().contiguous(), B.cuda().contiguous()
    D = torch.empty(128, N, dtype=torch.float32, device="cuda")
    rc = lib.gsb_umma_selftest(ctypes.c_void_p(Ad.data_ptr()), ctypes.c_void_p(Bd.data_ptr()),
                               ctypes.c_void_p(D.data_ptr()), K, N, mode,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    return D.double().cpu().numpy(), ref.numpy()


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("K,N", [(16, 16), (128, 128), (128, 16), (64, 256), (32, 48)])
def test_umma_tile_product(gsb, K, N, mode):
    d, ref = _selftest(gsb, K, N, mode, seed=K * 1000 + N + mode)
    err = np.abs(d - ref).max() / max(1.0, np.abs(ref).max())
    assert err < 1e-5, err


def _net(gsb, seed=0):
    return gsb.MlpWarmStart(gsb.IrkHenonHeiles(0.1), seed=seed)


def test_mlp_gradient_matches_cpu(gsb):
    """The device gradient (forward and backward on the tensor cores, weight gradients
    accumulated in tensor memory across a CTA's tiles) against the float64 CPU restatement."""
    import torch
    from oracle import mlp_reference as R
    from workloads import c3_states

    net = _net(gsb, seed=3)
    states = c3_states(40000, stream=5)          # 313 tiles: most CTAs take more than one
    g = np.random.default_rng(4)
    Z = net.stage_guess(states) * (1 + 0.01 * g.standard_normal((40000, 12)))
    t = net.set_normalisation(states, Z)
    S = torch.tensor(states, device="cuda")
    T = torch.tensor(t, dtype=torch.float32, device="cuda")
    grad, loss = net.gradient(S, T)
    torch.cuda.synchronize()
    assert int(net.err.item()) == 0
    gd = grad.double().cpu().numpy()
    sse, gr = R.loss_and_grad(net.theta.cpu().numpy(), net.norm.cpu().numpy(), states, t)
    assert abs(float(loss.item()) * 40000 * 12 - sse) <= 1e-3 * sse
    blocks = {"W1": (R.W1, R.B1), "b1": (R.B1, R.W2), "W2": (R.W2, R.B2), "b2": (R.B2, R.W3),
              "W3": (R.W3, R.B3), "b3": (R.B3, R.NTHETA)}
    for name, (a, b) in blocks.items():
        rel = np.linalg.norm(gd[a:b] - gr[a:b]) / np.linalg.norm(gr[a:b])
        assert rel < 2e-2, (name, rel)


def test_mlp_predict_and_gate(gsb):
    import torch
    from oracle import mlp_reference as R
    from workloads import c3_states

    net = _net(gsb, seed=5)
    states = c3_states(1000, stream=6)
    net.set_normalisation(states, net.stage_guess(states))
    S = torch.tensor(states, device="cuda")
    Z0 = net.predict(S).cpu().numpy()
    # the CPU forward of the same network
    w1, b1, w2, b2, w3, b3 = R.unpack(net.theta.cpu().numpy())
    nm = net.norm.cpu().numpy().astype(np.float64)
    xh = ((states.astype(np.float32) - nm[:4].astype(np.float32)) * nm[4:8].astype(np.float32)).astype(np.float64)
    out = (R.bf16(R.gelu(R.bf16(R.gelu(xh @ w1.T + b1)) @ R.bf16(w2) + b2)) @ R.bf16(w3) + b3)[:, :12]
    ref = net.stage_guess(states) + nm[8:20] * out
    assert np.abs(Z0 - ref).max() <= 2e-2 * np.abs(nm[8:20] * out).max() + 1e-12
    # the gate: the exact solution beats zero; a non-finite prediction is refused
    X0 = torch.zeros(1000, 12, dtype=torch.float64, device="cuda")
    Zt = torch.tensor(Z0, device="cuda")
    Zt[0] = float("nan")
    X, acc = net.select(S, Zt, X0)
    acc = acc.cpu().numpy()
    assert acc[0] == 0 and np.all(X[0].cpu().numpy() == 0.0)
    assert acc[1:].sum() > 0


def test_warm_start_gain(gsb, oracle):
    """Trained on the plain solver's solutions of a disjoint draw, the network's starts take
    fewer Newton iterations than the default start Z = 0, and every system still converges to
    the oracle's solution; the fallback rate (predictions the gate refused) is reported."""
    import torch
    from workloads import c3, c3_states

    fam = gsb.IrkHenonHeiles(0.1)
    prob = gsb.NonlinearProblem(fam)
    m = gsb.Newton(globalization=gsb.Backtracking())
    opts = gsb.Options(f_abstol=1e-12, f_reltol=0.0, max_iterations=50)
    # training data: the plain solver's solutions from a disjoint seed stream
    ntr = 2097152
    tr = c3_states(ntr, stream=1)
    Ztr = torch.zeros(ntr, 12, dtype=torch.float64, device="cuda")
    gsb.solve_batch(Ztr, gsb.status_buffer(ntr), prob, m,
                    gsb.PerSystem(torch.tensor(tr, device="cuda")), options=opts)
    net = gsb.MlpWarmStart(fam, seed=0)
    hist = net.train(tr, Ztr.cpu().numpy(), epochs=80, batch=8192, lr=5e-3)
    assert hist[-1] < 1e-2 * hist[0]
    X0, P = c3(16384)
    Pd = torch.tensor(P, device="cuda")
    Xd = torch.tensor(X0, device="cuda")
    Xw, acc = net.warm_start(Pd, Xd)
    S0, Sw = gsb.status_buffer(16384), gsb.status_buffer(16384)
    gsb.solve_batch(Xd, S0, prob, m, gsb.PerSystem(Pd), options=opts)
    gsb.solve_batch(Xw, Sw, prob, m, gsb.PerSystem(Pd), options=opts)
    s0, sw = gsb.statuses(S0), gsb.statuses(Sw)
    assert np.all(s0["code"] == 0) and np.all(sw["code"] == 0)
    # from Z = 0 every system takes two steps; most warm starts converge in one
    assert s0["iterations"].mean() == 2.0
    assert sw["iterations"].mean() < 1.2
    xo, so = oracle.solve_batch(prob, m, X0.copy(), P, opts)
    xw = Xw.cpu().numpy()
    err = np.max(np.abs(xw - xo), axis=1) / np.max(np.abs(xo), axis=1)
    assert np.all(err <= 1e-10)
    print(f"iterations {s0['iterations'].mean():.3f} -> {sw['iterations'].mean():.3f}; "
          f"fallback {1 - acc.float().mean().item():.4f}")
