"""ctypes binding of the oracle (oracle/liboracle.so) for the tests.

The oracle is the checker: a CPU restatement of the reference algorithm,
pinned to the reference's regression goldens (test_oracle_golden.py).
"""
import ctypes as C
import os

import numpy as np

import helpers

_lib = None


def lib():
    global _lib
    if _lib is None:
        helpers.build_oracle()
        L = C.CDLL(os.path.join(helpers.ORACLE_DIR, "liboracle.so"))
        dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        L.orc_batch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_int, dp, dp, ip, dp, ip]
        L.orc_setup_dims.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, ip, ip]
        L.orc_setup_copy.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, ip, ip, dp]
        L.orc_solver_open.restype = vp
        L.orc_solver_open.argtypes = [C.c_char_p]
        L.orc_solver_dims.argtypes = [vp, ip, ip, ip, dp, dp, dp]
        L.orc_solver_steps.argtypes = [vp, C.c_int]
        L.orc_solver_step_dt.argtypes = [vp, C.c_double]
        L.orc_solver_state.argtypes = [vp, dp, dp]
        L.orc_solver_set_state.argtypes = [vp, dp, dp]
        L.orc_solver_stats.argtypes = [vp, ip, dp, C.POINTER(C.c_longlong), ip]
        L.orc_solver_close.argtypes = [vp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def setup(order, Q, use_gaunt):
    n, n2, nq, nnz = C.c_int(), C.c_int(), C.c_int(), C.c_int()
    st = lib().orc_setup_dims(order, Q, int(use_gaunt), C.byref(n), C.byref(n2), C.byref(nq),
                              C.byref(nnz))
    assert st == 0
    n, n2, nq, nnz = n.value, n2.value, nq.value, nnz.value
    w, xi, eta = np.empty(nq), np.empty(nq), np.empty(nq)
    p = np.empty((nq, n2))
    off = np.zeros(n * n + 1, np.int32)
    idx = np.zeros(max(nnz, 1), np.int32)
    val = np.zeros(max(nnz, 1))
    lib().orc_setup_copy(order, Q, int(use_gaunt), _dp(w), _dp(xi), _dp(eta), _dp(p), _ip(off),
                         _ip(idx), _dp(val))
    return {"n": n, "n2": n2, "nq": nq, "w": w, "xi": xi, "eta": eta, "p": p,
            "off": off, "idx": idx[:nnz], "val": val[:nnz]}


def opt_batch(order, Q, use_gaunt, u, alpha, moment_type=0, max_iter=100, tol=1e-8,
              cond_h_max=1e10, delta_ppn=1e-10, tol_gamma=0.0):
    """opt() on each row of u/alpha in place; returns iters, regs, status."""
    count = u.shape[0]
    iters = np.zeros(count, np.int32)
    regs = np.zeros(count)
    status = np.zeros(count, np.int32)
    lib().orc_batch(order, Q, int(use_gaunt), moment_type, max_iter, tol, cond_h_max, delta_ppn,
                    tol_gamma, count, _dp(u), _dp(alpha), _ip(iters), _dp(regs), _ip(status))
    return iters, regs, status


class GridSolver:
    def __init__(self, deck_path):
        self.h = lib().orc_solver_open(deck_path.encode())
        assert self.h, "oracle rejected the deck"
        NX, NY, n = C.c_int(), C.c_int(), C.c_int()
        md, dx, dy = C.c_double(), C.c_double(), C.c_double()
        lib().orc_solver_dims(self.h, C.byref(NX), C.byref(NY), C.byref(n), C.byref(md),
                              C.byref(dx), C.byref(dy))
        self.NX, self.NY, self.n = NX.value, NY.value, n.value
        self.max_dt, self.dx, self.dy = md.value, dx.value, dy.value

    def steps(self, k):
        st = lib().orc_solver_steps(self.h, k)
        assert st == 0, "oracle error %d" % st

    def state(self):
        m = np.empty((self.NX, self.NY, self.n))
        a = np.empty((self.NX, self.NY, self.n))
        lib().orc_solver_state(self.h, _dp(m), _dp(a))
        return m, a

    def set_state(self, m, a):
        m = np.ascontiguousarray(m, dtype=np.float64)
        a = np.ascontiguousarray(a, dtype=np.float64)
        lib().orc_solver_set_state(self.h, _dp(m), _dp(a))

    def stats(self):
        mi, im, ns = C.c_int(), C.c_double(), C.c_longlong()
        hist = np.zeros(5, np.int32)
        lib().orc_solver_stats(self.h, C.byref(mi), C.byref(im), C.byref(ns), _ip(hist))
        return {"max_iter": mi.value, "iter_mean": im.value, "num_solves": ns.value,
                "hist_reg": hist.tolist()}

    def close(self):
        if self.h:
            lib().orc_solver_close(self.h)
            self.h = None

    def __del__(self):
        self.close()
