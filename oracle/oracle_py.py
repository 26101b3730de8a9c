"""ORACLE — test infrastructure only. ctypes bindings of oracle/liboracle.so, the CPU
restatement of GeometricSolvers.jl's R2 batch. Used by tests/, the smoke check and bench.py's
CPU-baseline leg as the checker; never by the product."""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

import gsb200
from gsb200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

FAM_QUADMOD2 = 200
FAM_CUBICDIAG2 = 201

_lib = None


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    L = ctypes.CDLL(LIB)
    P = ctypes.POINTER
    vp = ctypes.c_void_p
    L.oracle_solve_batch.argtypes = [
        P(abi.GsbProblem), P(abi.GsbMethod), P(abi.GsbOptions),
        vp, ctypes.c_int32, vp, ctypes.c_int32, vp, ctypes.c_int32, vp, ctypes.c_int32,
        ctypes.c_int64, ctypes.c_int32,
    ]
    L.oracle_solve_batch.restype = ctypes.c_int
    L.oracle_max_threads.restype = ctypes.c_int
    L.oracle_standard_cell.argtypes = [
        ctypes.c_int32, vp, ctypes.c_int32, ctypes.c_int32, vp, P(abi.GsbStatus64),
        P(ctypes.c_int64), P(ctypes.c_int64),
    ]
    L.oracle_standard_cell.restype = ctypes.c_int
    L.oracle_standard_residual.argtypes = [ctypes.c_int32, vp, vp]
    L.oracle_standard_residual.restype = ctypes.c_int
    L.oracle_backtrack_step.argtypes = [ctypes.c_double] * 7
    L.oracle_backtrack_step.restype = ctypes.c_double
    L.oracle_ldexp2.argtypes = [ctypes.c_double, ctypes.c_int64]
    L.oracle_ldexp2.restype = ctypes.c_double
    L.oracle_ldexp2f.argtypes = [ctypes.c_float, ctypes.c_int64]
    L.oracle_ldexp2f.restype = ctypes.c_float
    L.oracle_rnorm.argtypes = [vp, ctypes.c_int32]
    L.oracle_rnorm.restype = ctypes.c_double
    L.oracle_matrix_exponent.argtypes = [vp, ctypes.c_int32]
    L.oracle_matrix_exponent.restype = ctypes.c_int32
    L.oracle_rhs_exponent.argtypes = [vp, ctypes.c_int32, ctypes.c_int32]
    L.oracle_rhs_exponent.restype = ctypes.c_int32
    L.oracle_factor_solve.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, vp, vp,
                                      P(ctypes.c_int32)]
    L.oracle_factor_solve.restype = ctypes.c_int32
    L.oracle_givens.argtypes = [ctypes.c_double, ctypes.c_double, P(ctypes.c_double),
                                P(ctypes.c_double), P(ctypes.c_double)]
    L.oracle_givens.restype = None
    L.oracle_family_eval.argtypes = [P(abi.GsbProblem), vp, vp, vp, vp]
    L.oracle_family_eval.restype = ctypes.c_int
    _lib = L
    return L


LINE_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_void_p)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def max_threads() -> int:
    return lib().oracle_max_threads()


def solve_batch(prob, method, X, P, options=None, *, order=None, order_base=0, s_kind="status",
                x_layout="aos", p_layout="aos", nthreads=0, family_code=None, n=None, m=None,
                shared=None):
    """Run the CPU batch on host arrays in place; returns the statuses (structured array) or the
    codes. `prob` is a gsb200 problem, or None with `family_code`, `n`, `m` for the
    oracle-only test families."""
    L = lib()
    X = np.ascontiguousarray(X, dtype=np.float64)
    P = np.ascontiguousarray(P, dtype=np.float64)
    nsys = X.shape[0] if x_layout == "aos" else X.shape[1]
    if prob is not None:
        sh = prob.family.shared()
        gp = prob.to_abi()
    else:
        sh = shared
        gp = abi.GsbProblem()
        gp.family, gp.n, gp.m = family_code, n, m
    sh_arr = None if sh is None else np.ascontiguousarray(sh, dtype=np.float64)
    gp.shared = None if sh_arr is None else sh_arr.ctypes.data
    gm = method.to_abi()
    go = (options or gsb200.Options()).to_abi()
    if s_kind == "status":
        S = np.zeros(nsys, dtype=abi.SOLVER_STATUS_DTYPE)
        sk = abi.GSB_STATUS64
    else:
        S = np.zeros(nsys, dtype=np.uint8)
        sk = abi.GSB_CODES
    order_arr = None if order is None else np.ascontiguousarray(order, dtype=np.int64)
    rc = L.oracle_solve_batch(
        ctypes.byref(gp), ctypes.byref(gm), ctypes.byref(go), _ptr(X),
        abi.GSB_AOS if x_layout == "aos" else abi.GSB_SOA, _ptr(S), sk, _ptr(P),
        abi.GSB_AOS if p_layout == "aos" else abi.GSB_SOA, _ptr(order_arr), order_base, nsys,
        nthreads,
    )
    if rc != 0:
        raise RuntimeError(f"oracle_solve_batch returned {rc}")
    return X, S


def standard_cell(number, x0, column, max_iterations=200):
    L = lib()
    x0 = np.ascontiguousarray(x0, dtype=np.float64)
    x = np.zeros_like(x0)
    st = abi.GsbStatus64()
    fe = ctypes.c_int64()
    de = ctypes.c_int64()
    n = L.oracle_standard_cell(number, _ptr(x0), column, max_iterations, _ptr(x),
                               ctypes.byref(st), ctypes.byref(fe), ctypes.byref(de))
    if n < 0:
        raise ValueError(number)
    return x, st, fe.value, de.value


def standard_residual(number, x):
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros_like(x)
    lib().oracle_standard_residual(number, _ptr(x), _ptr(out))
    return out


def backtracking(phi, dphi, phi0, *, exact=True, c1=1e-4, p=0.5, maxiter=100, alpha=1.0):
    """The Backtracking search along a line φ(α), φ′(α) given as Python callables."""
    trials = []

    def _phi(a, _):
        trials.append(a)
        return float(phi(a))

    def _dphi(a, _):
        return float(dphi(a))

    f1, f2 = LINE_FN(_phi), LINE_FN(_dphi)
    ao, po, ev = ctypes.c_double(), ctypes.c_double(), ctypes.c_int32()
    code = lib().oracle_backtracking(
        c1, p, maxiter, f1, f2, None, int(exact), phi0, alpha, ctypes.byref(ao), ctypes.byref(po),
        ctypes.byref(ev))
    return code, ao.value, po.value, ev.value, trials


def _setup_backtracking():
    L = lib()
    L.oracle_backtracking.argtypes = [
        ctypes.c_double, ctypes.c_double, ctypes.c_int32, LINE_FN, LINE_FN, ctypes.c_void_p,
        ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int32),
    ]
    L.oracle_backtracking.restype = ctypes.c_int


def factor_solve(J, r, qr=False, f32=False):
    J = np.asfortranarray(J, dtype=np.float64)
    n = J.shape[0]
    Jc = np.ascontiguousarray(J.flatten(order="F"))
    r = np.ascontiguousarray(r, dtype=np.float64)
    d = np.zeros(n)
    e = ctypes.c_int32()
    info = lib().oracle_factor_solve(_ptr(Jc), n, int(qr), int(f32), _ptr(r), _ptr(d), ctypes.byref(e))
    return info, d, e.value


def family_eval(prob, x, p):
    gp = prob.to_abi()
    sh = prob.family.shared()
    sh_arr = None if sh is None else np.ascontiguousarray(sh, dtype=np.float64)
    gp.shared = None if sh_arr is None else sh_arr.ctypes.data
    x = np.ascontiguousarray(x, dtype=np.float64)
    p = np.ascontiguousarray(p, dtype=np.float64)
    F = np.zeros(prob.family.m)
    J = np.zeros(prob.family.m * prob.family.n)
    rc = lib().oracle_family_eval(ctypes.byref(gp), _ptr(x), _ptr(p), _ptr(F), _ptr(J))
    if rc != 0:
        raise RuntimeError(rc)
    return F, J.reshape(prob.family.n, prob.family.m).T


def ldexp2(x, e):
    return lib().oracle_ldexp2(x, e)


def rnorm(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return lib().oracle_rnorm(_ptr(a), len(a))


def givens(f, g):
    c, s, r = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().oracle_givens(f, g, ctypes.byref(c), ctypes.byref(s), ctypes.byref(r))
    return c.value, s.value, r.value


lib()
_setup_backtracking()
