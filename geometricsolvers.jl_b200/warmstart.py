"""The learned warm start of the Gauss-3 stage systems (the IRK batch of the Hénon–Heiles field).

A 4 -> 128 -> 128 -> 12 MLP (GELU; BF16 weights and activations in the tensor-core products,
FP32 accumulation; the kernels are libgsb's `gsb_mlp_*`) maps a state y to a start

    Z0 = g(y) + scale * net((y - mean) * inv_dev),     g(y)_j = h c_j f(y),

the explicit stage guess plus a learned correction. It is trained on the device, with the
project's own forward and backward kernels and Adam, on solutions that the plain Newton solver
produced. At solve time the prediction is kept for a system only where its FP64 residual norm
beats the default start's (``gsb_warm_start_select``), so plain Newton stays both the fallback
and the arbiter of every prediction.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import abi
from .api import ArgumentError, _raise_for


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class MlpWarmStart:
    """The network, its Adam state and its normalisation, on one CUDA device."""

    def __init__(self, family, device="cuda", seed=0):
        import torch

        self.family = family  # an api.IrkHenonHeiles (h and its tableau)
        self.device = torch.device(device)
        lib = abi.load_library()
        nt, npk = ctypes.c_int64(), ctypes.c_int64()
        lib.gsb_mlp_sizes(ctypes.byref(nt), ctypes.byref(npk))
        self.n_theta, self.n_pack = nt.value, npk.value
        g = torch.Generator().manual_seed(seed)
        theta = torch.zeros(self.n_theta, dtype=torch.float32)
        # He-style initialisation: W1 [128][4], W2 [128][128], W3 [128][12 of 16]
        theta[0:512] = torch.randn(512, generator=g) * math.sqrt(2.0 / 4)
        theta[640:17024] = torch.randn(16384, generator=g) * math.sqrt(2.0 / 128)
        w3 = torch.zeros(128, 16)
        w3[:, :12] = torch.randn(128, 12, generator=g) * math.sqrt(1.0 / 128)
        theta[17152:19200] = w3.reshape(-1)
        self.theta = theta.to(self.device)
        self.m = torch.zeros_like(self.theta)
        self.v = torch.zeros_like(self.theta)
        self.grad = torch.zeros_like(self.theta)
        self.pack = torch.zeros(self.n_pack, dtype=torch.int16, device=self.device)
        self.norm = torch.zeros(20, dtype=torch.float32, device=self.device)
        self.loss_buf = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.shared = torch.tensor(family.shared(), dtype=torch.float64, device=self.device)
        self.step = 0
        self._lib = lib
        self._stream = lambda: ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)
        _raise_for(lib.gsb_mlp_pack(_ptr(self.theta), _ptr(self.pack), self._stream()), lib)

    # the explicit stage guess g(y), on the host (float64)
    def stage_guess(self, states):
        h = self.family.h
        A = self.family.A
        c = A.sum(axis=1)
        y = np.asarray(states, dtype=np.float64)
        f = np.stack([y[:, 2], y[:, 3], -y[:, 0] - 2.0 * y[:, 0] * y[:, 1],
                      -y[:, 1] - y[:, 0] ** 2 + y[:, 1] ** 2], axis=1)
        return np.concatenate([h * c[j] * f for j in range(3)], axis=1)

    def set_normalisation(self, states, Z):
        import torch

        s = np.asarray(states, dtype=np.float64)
        mean = s.mean(axis=0)
        inv = 1.0 / np.maximum(s.std(axis=0), 1e-12)
        corr = np.asarray(Z, dtype=np.float64) - self.stage_guess(s)
        scale = np.maximum(corr.std(axis=0), 1e-30)
        self.norm.copy_(torch.tensor(np.concatenate([mean, inv, scale]), dtype=torch.float32))
        return corr / scale

    def gradient(self, states_dev, targets_dev):
        """The gradient and the mean loss on one batch (no update)."""
        n = states_dev.shape[0]
        _raise_for(self._lib.gsb_mlp_grad(
            _ptr(self.theta), _ptr(self.pack), _ptr(self.norm), _ptr(states_dev),
            _ptr(targets_dev), n, _ptr(self.grad), _ptr(self.loss_buf), _ptr(self.err),
            self._stream()), self._lib)
        return self.grad, self.loss_buf / (n * 12)

    def train(self, states, Z, epochs=20, batch=32768, lr=2e-3, seed=1, log=None):
        """Fit the network to the solutions Z (n x 12) of the states (n x 4)."""
        import torch

        t = self.set_normalisation(states, Z)
        S = torch.tensor(np.ascontiguousarray(states), dtype=torch.float64, device=self.device)
        T = torch.tensor(t, dtype=torch.float32, device=self.device)
        n = S.shape[0]
        g = torch.Generator(device=self.device).manual_seed(seed)
        history = []
        for ep in range(epochs):
            perm = torch.randperm(n, device=self.device, generator=g)
            lr_ep = lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs))  # cosine decay
            total = torch.zeros((), device=self.device)
            for b0 in range(0, n - batch + 1, batch):
                idx = perm[b0:b0 + batch]
                xs, ts = S[idx].contiguous(), T[idx].contiguous()
                _, loss = self.gradient(xs, ts)
                total += loss[0]
                self.step += 1
                _raise_for(self._lib.gsb_mlp_adam(
                    _ptr(self.theta), _ptr(self.m), _ptr(self.v), _ptr(self.grad), _ptr(self.pack),
                    lr_ep, 0.9, 0.999, 1e-8, self.step, self._stream()), self._lib)
            if int(self.err.item()):
                raise RuntimeError("a training tile timed out waiting for the tensor cores")
            history.append(float(total.item()) / max(1, n // batch))
            if log:
                log(ep, history[-1])
        return history

    def predict(self, states_dev):
        import torch

        n = states_dev.shape[0]
        Z0 = torch.empty((n, 12), dtype=torch.float64, device=self.device)
        _raise_for(self._lib.gsb_mlp_predict(
            _ptr(self.theta), _ptr(self.pack), _ptr(self.norm), _ptr(self.shared),
            _ptr(states_dev), _ptr(Z0), n, _ptr(self.err), self._stream()), self._lib)
        return Z0

    def select(self, states_dev, Z0, X_default):
        """The accept-if-better gate: (X, accepted)."""
        import torch

        n = states_dev.shape[0]
        if Z0.shape != (n, 12) or X_default.shape != (n, 12):
            raise ArgumentError("Z0 and X_default must be (n, 12)")
        X = torch.empty_like(X_default)
        acc = torch.empty(n, dtype=torch.uint8, device=self.device)
        _raise_for(self._lib.gsb_warm_start_select(
            _ptr(self.shared), _ptr(states_dev), _ptr(Z0), _ptr(X_default), _ptr(X), _ptr(acc), n,
            self._stream()), self._lib)
        return X, acc

    def warm_start(self, states_dev, X_default):
        """The start of each system: the network's where it beats X_default, else X_default."""
        return self.select(states_dev, self.predict(states_dev), X_default)
