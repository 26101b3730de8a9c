"""ORACLE — test infrastructure only. A float64 CPU restatement of the warm-start network's forward
pass, loss and gradient (libgsb's gsb_mlp_grad), rounding to BF16 at the points where the device
rounds (the tensor-core operands: W2, W3, the activations H1, H2 and the output and hidden
gradients), so that the device gradient can be checked against it."""

import numpy as np

W1, B1, W2, B2, W3, B3, NTHETA = 0, 512, 640, 17024, 17152, 19200, 19216


def bf16(x):
    """Round float64 values to BF16 (nearest even) through float32, as the device does."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def _erf(x):
    from math import erf

    return np.vectorize(erf)(x)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def unpack(theta):
    t = np.asarray(theta, dtype=np.float64)
    return (t[W1:B1].reshape(128, 4), t[B1:W2], t[W2:B2].reshape(128, 128), t[B2:W3],
            t[W3:B3].reshape(128, 16), t[B3:NTHETA])


def loss_and_grad(theta, norm, states, targets):
    """(sum of squared errors, gradient of the mean squared error) for n samples."""
    w1, b1, w2, b2, w3, b3 = unpack(theta)
    norm = np.asarray(norm, dtype=np.float64)
    xh = ((np.asarray(states, dtype=np.float32) - norm[0:4].astype(np.float32)) *
          norm[4:8].astype(np.float32)).astype(np.float64)
    n = xh.shape[0]
    z1 = xh @ w1.T + b1
    h1 = bf16(gelu(z1))
    z2 = h1 @ bf16(w2) + b2
    h2 = bf16(gelu(z2))
    out = (h2 @ bf16(w3) + b3)[:, :12]
    d = out - np.asarray(targets, dtype=np.float64)
    sse = float(np.sum(d * d))
    g = np.zeros((n, 16))
    g[:, :12] = 2.0 / (n * 12) * d
    g3 = bf16(g)
    grad = np.zeros(NTHETA)
    grad[B3:B3 + 12] = g[:, :12].sum(axis=0)
    dw3 = h2.T @ g3
    grad[W3:B3] = np.concatenate([dw3[:, :12], np.zeros((128, 4))], axis=1).reshape(-1)
    dh2 = g3 @ bf16(w3).T
    dz2 = dh2 * gelu_grad(z2)
    g2 = bf16(dz2)
    grad[B2:W3] = dz2.sum(axis=0)
    grad[W2:B2] = (h1.T @ g2).reshape(-1)
    dh1 = g2 @ bf16(w2).T
    dz1 = dh1 * gelu_grad(z1)
    grad[B1:W2] = dz1.sum(axis=0)
    grad[W1:B1] = (dz1.T @ xh).reshape(-1)
    return sse, grad
