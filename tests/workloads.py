"""Seeded synthetic inputs of the batch configurations (shared by the tests and bench.py).

Counter-based generation with numpy's Philox bit generator, seed 20261203 + config id, so
every rank and every run draws the same systems.
"""

import numpy as np

SEED = 20261203


def rng(config_id, stream=0):
    return np.random.Generator(np.random.Philox(key=SEED + config_id, counter=stream))


def cubic_affine(n, nsys, diag, config_id, stream=0):
    """F(x) = A x + 0.1 x.^3 - b: A = diag I + 0.5 N(0,1), b ~ U(-1, 1)^n, x0 = 0.
    Returns (X0 (nsys, n), P (nsys, n*n + n)) with A column-major in each parameter block."""
    g = rng(config_id, stream)
    A = g.standard_normal((nsys, n, n)) * 0.5
    A[:, np.arange(n), np.arange(n)] += diag
    b = g.uniform(-1.0, 1.0, (nsys, n))
    P = np.concatenate([A.transpose(0, 2, 1).reshape(nsys, n * n), b], axis=1)
    return np.zeros((nsys, n)), np.ascontiguousarray(P)


def c0(nsys=65536):
    return cubic_affine(3, nsys, 4.0, 0)


def c1(nsys=1048576):
    return cubic_affine(8, nsys, 6.0, 1)


def cubic_affine_pivoting(n, nsys, diag, config_id):
    """The cubic-affine batch with the rows of each A in a random order (b permuted alike), so
    that partial pivoting exchanges rows in nearly every factorisation."""
    X0, P = cubic_affine(n, nsys, diag, config_id)
    g = rng(config_id, stream=7)
    A = P[:, : n * n].reshape(nsys, n, n).transpose(0, 2, 1)  # back to row-major (nsys, n, n)
    b = P[:, n * n:]
    perm = np.argsort(g.random((nsys, n)), axis=1)
    A = np.take_along_axis(A, perm[:, :, None], axis=1)
    b = np.take_along_axis(b, perm, axis=1)
    P = np.concatenate([A.transpose(0, 2, 1).reshape(nsys, n * n), b], axis=1)
    return X0, np.ascontiguousarray(P)


def cubic_affine_illcond(n, nsys, config_id, log10_cond=(3.0, 9.0)):
    """Cubic-affine systems whose A = Q1 diag(s) Q2 has a condition number drawn log-uniformly
    from 10^log10_cond, so that the Float32 factor of the mixed form needs its refinement passes
    and, on the ill-conditioned end, is promoted to Float64. b ~ 1e-3 U(-1, 1)^n, x0 = 0."""
    g = rng(config_id, stream=11)
    q1, _ = np.linalg.qr(g.standard_normal((nsys, n, n)))
    q2, _ = np.linalg.qr(g.standard_normal((nsys, n, n)))
    lc = g.uniform(log10_cond[0], log10_cond[1], nsys)
    s = 10.0 ** (-lc[:, None] * np.linspace(0.0, 1.0, n)[None, :])
    A = np.einsum("sij,sj,sjk->sik", q1, s, q2) * (n + 1.0)
    b = g.uniform(-1.0, 1.0, (nsys, n)) * 1e-3
    P = np.concatenate([A.transpose(0, 2, 1).reshape(nsys, n * n), b], axis=1)
    return np.zeros((nsys, n)), np.ascontiguousarray(P)


def c2(nsys=524288, m=64):
    """Exp-sum least squares: t = linspace(0, 4, m) (shared), true a_j ~ U(0.5, 2) and b_j ~
    U(0.1, 3) sorted ascending, y = sum_j a_j exp(-b_j t) + N(0, 1e-3^2), x0 = truth (1 + U(-0.2,
    0.2)). x = (a1, b1, a2, b2, a3, b3). Returns (X0 (nsys, 6), Y (nsys, m), t (m,))."""
    g = rng(2)
    t = np.linspace(0.0, 4.0, m)
    a = g.uniform(0.5, 2.0, (nsys, 3))
    b = np.sort(g.uniform(0.1, 3.0, (nsys, 3)), axis=1)
    y = np.einsum("sj,sji->si", a, np.exp(-b[:, :, None] * t[None, None, :]))
    y += g.standard_normal((nsys, m)) * 1e-3
    truth = np.stack([a[:, 0], b[:, 0], a[:, 1], b[:, 1], a[:, 2], b[:, 2]], axis=1)
    X0 = truth * (1.0 + g.uniform(-0.2, 0.2, (nsys, 6)))
    return np.ascontiguousarray(X0), np.ascontiguousarray(y), t


C4_SIZES = (2, 3, 4, 6, 8, 12, 16, 24, 32)


def c4(nsys=4194304):
    """The ragged batch: sizes n from {2, 3, 4, 6, 8, 12, 16, 24, 32} with probability ∝ 1/n,
    each system cubic-affine with A = (n+1) I + 0.5 N(0,1), b ~ U(-1, 1)^n, x0 = 0, packed back
    to back. Returns (sizes (nsys,) int32, X0 (sum n,), P (sum n^2 + n,))."""
    g = rng(4)
    w = np.array([1.0 / n for n in C4_SIZES])
    sizes = np.array(C4_SIZES, dtype=np.int32)[g.choice(len(C4_SIZES), nsys, p=w / w.sum())]
    n64 = sizes.astype(np.int64)
    p_len = n64 * n64 + n64
    p_off = np.cumsum(p_len) - p_len
    P = np.empty(int(p_len.sum()), dtype=np.float64)
    for b, n in enumerate(C4_SIZES):
        sel = np.flatnonzero(sizes == n)
        if sel.size == 0:
            continue
        _, Pb = cubic_affine(n, sel.size, n + 1.0, 4, stream=b + 1)
        idx = p_off[sel][:, None] + np.arange(n * n + n)[None, :]
        P[idx] = Pb
    return sizes, np.zeros(int(n64.sum()), dtype=np.float64), P


def henon_heiles_energy(s):
    q1, q2, p1, p2 = s[:, 0], s[:, 1], s[:, 2], s[:, 3]
    return 0.5 * (p1 * p1 + p2 * p2) + 0.5 * (q1 * q1 + q2 * q2) + q1 * q1 * q2 - q2 ** 3 / 3.0


def c3_states(nsys, config_id=3, stream=0, box=0.6):
    """Hénon–Heiles states (q1, q2, p1, p2) uniform in [-box, box]^4, rejection-sampled to energy
    H in [0.01, 0.16]. The training set of the warm start draws from its own stream."""
    g = rng(config_id, stream)
    out = np.empty((0, 4))
    while out.shape[0] < nsys:
        s = g.uniform(-box, box, (2 * (nsys - out.shape[0]) + 1024, 4))
        H = henon_heiles_energy(s)
        out = np.concatenate([out, s[(H >= 0.01) & (H <= 0.16)]])
    return np.ascontiguousarray(out[:nsys])


def c3(nsys=262144):
    """The Gauss-3 stage systems of one h = 0.1 step from each state: Z0 = 0 (12 unknowns) and
    P = the state (4 per system)."""
    P = c3_states(nsys)
    return np.zeros((nsys, 12)), P
