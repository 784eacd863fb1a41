"""ctypes binding of the oracle (liboracle.so in this directory).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline / reference arm of bench.py.  The oracle is the checker, a CPU
restatement of the reference algorithm pinned to the reference's regression
goldens (tests/test_oracle_golden.py).
"""
import ctypes as C
import os
import subprocess
import threading

import numpy as np

ORACLE_DIR = os.path.dirname(os.path.abspath(__file__))
_build_lock = threading.Lock()
_built = False


def build():
    """Builds the oracle libraries and driver once per process."""
    global _built
    with _build_lock:
        if not _built:
            subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)
            _built = True
    return os.path.join(ORACLE_DIR, "oracle_momopt")

_lib = None
_lib_fma = None


def lib(fma=False):
    """The oracle; fma=True gives the same code compiled with FMA contraction."""
    global _lib, _lib_fma
    if fma:
        if _lib_fma is None:
            build()
            _lib_fma = _bind(C.CDLL(os.path.join(ORACLE_DIR, "liboracle_fma.so")))
        return _lib_fma
    if _lib is None:
        build()
        _lib = _bind(C.CDLL(os.path.join(ORACLE_DIR, "liboracle.so")))
    return _lib


def _bind(L):
    if True:
        dp, ip, vp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
        L.orc_batch.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                C.c_double, C.c_double, C.c_int, dp, dp, ip, dp, ip]
        L.orc_setup_dims.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, ip, ip]
        L.orc_setup_copy.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, ip, ip, dp]
        L.orc_solver_open.restype = vp
        L.orc_solver_open.argtypes = [C.c_char_p]
        L.orc_solver_open_node.restype = vp
        L.orc_solver_open_node.argtypes = [C.c_char_p, C.c_int, C.c_int]
        L.orc_solver_node_info.argtypes = [vp, ip, dp]
        L.orc_solver_save_old_h.argtypes = [vp]
        L.orc_solver_pre_exchange_h.argtypes = [vp]
        L.orc_solver_run_h.argtypes = [vp, C.c_char_p, C.c_int]
        L.orc_solver_stage_exchanged_h.argtypes = [vp, C.c_double]
        L.orc_solver_average_h.argtypes = [vp]
        L.orc_solver_halo_count_h.argtypes = [vp, C.c_int]
        L.orc_solver_halo_count_h.restype = C.c_longlong
        L.orc_solver_halo_h.argtypes = [vp, C.c_int, C.c_int, dp]
        L.orc_solver_output_h.argtypes = [vp, C.c_double, C.c_char_p]
        L.orc_solver_dims.argtypes = [vp, ip, ip, ip, dp, dp, dp]
        L.orc_solver_steps.argtypes = [vp, C.c_int]
        L.orc_solver_step_dt.argtypes = [vp, C.c_double]
        L.orc_solver_state.argtypes = [vp, dp, dp]
        L.orc_solver_set_state.argtypes = [vp, dp, dp]
        L.orc_solver_stats.argtypes = [vp, ip, dp, C.POINTER(C.c_longlong), ip]
        L.orc_solver_close.argtypes = [vp]
        L.orc_solver_last_iters.argtypes = [vp, ip]
        L.orc_batch_cb.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double,
                                   C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, dp, dp, dp,
                                   dp, ip, dp, ip]
        L.orc_cb_init.argtypes = [C.c_int, C.c_int, C.c_double, C.c_int, dp, dp]
        L.orc_cb_init.restype = None
    return L


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
              cond_h_max=1e10, delta_ppn=1e-10, tol_gamma=0.0, fma=False):
    """opt() on each row of u/alpha in place; returns iters, regs, status."""
    count = u.shape[0]
    iters = np.zeros(count, np.int32)
    regs = np.zeros(count)
    status = np.zeros(count, np.int32)
    lib(fma).orc_batch(order, Q, int(use_gaunt), moment_type, max_iter, tol, cond_h_max, delta_ppn,
                    tol_gamma, count, _dp(u), _dp(alpha), _ip(iters), _dp(regs), _ip(status))
    return iters, regs, status


def cb_init(n, count, moment_type=0, delta_ppn=1e-10):
    """The reference's initial change-of-basis state (P2M [count][n][n]
    row-major lower triangular, alphaP [count][n])."""
    P2M = np.zeros((count, n, n))
    alphaP = np.zeros((count, n))
    lib().orc_cb_init(n, moment_type, delta_ppn, count, _dp(P2M), _dp(alphaP))
    return P2M, alphaP


def optcb_batch(order, Q, u, P2M, alphaP, alpha, moment_type=0, max_iter=100, tol=1e-8,
                cond_h_max=1e10, delta_ppn=1e-10, fma=False, opt_type=1, max_bfgs_iter=5,
                cond_h_max_bfgs=20.0):
    """Change-of-basis opt (opt_type 1: optcb.cpp, 2: optbfgs.cpp) on each
    row in place: u, P2M, alphaP updated, alpha receives the multipliers.
    Returns iters, regs, status."""
    count = u.shape[0]
    iters = np.zeros(count, np.int32)
    regs = np.zeros(count)
    status = np.zeros(count, np.int32)
    lib(fma).orc_batch_cb(order, Q, moment_type, opt_type, max_iter, tol, cond_h_max, delta_ppn,
                          max_bfgs_iter, cond_h_max_bfgs, count, _dp(u), _dp(P2M), _dp(alphaP),
                          _dp(alpha), _ip(iters), _dp(regs), _ip(status))
    return iters, regs, status


class GridSolver:
    """The oracle's solver of a deck: the whole grid (one node), or node
    `node` of the deck's NUM_MPI_PARTITIONS_X x _Y partition on num_nodes."""

    def __init__(self, deck_path, fma=False, node=0, num_nodes=1):
        self.L = lib(fma)
        self.h = self.L.orc_solver_open_node(deck_path.encode(), node, num_nodes)
        assert self.h, "oracle rejected the deck"
        NX, NY, n = C.c_int(), C.c_int(), C.c_int()
        md, dx, dy = C.c_double(), C.c_double(), C.c_double()
        self.L.orc_solver_dims(self.h, C.byref(NX), C.byref(NY), C.byref(n), C.byref(md),
                              C.byref(dx), C.byref(dy))
        self.NX, self.NY, self.n = NX.value, NY.value, n.value
        self.max_dt, self.dx, self.dy = md.value, dx.value, dy.value

    def steps(self, k):
        st = self.L.orc_solver_steps(self.h, k)
        assert st == 0, "oracle error %d" % st

    def state(self):
        m = np.empty((self.NX, self.NY, self.n))
        a = np.empty((self.NX, self.NY, self.n))
        self.L.orc_solver_state(self.h, _dp(m), _dp(a))
        return m, a

    def set_state(self, m, a):
        m = np.ascontiguousarray(m, dtype=np.float64)
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.L.orc_solver_set_state(self.h, _dp(m), _dp(a))

    def node_info(self):
        info = np.zeros(7, np.int32)
        origin = np.zeros(2)
        self.L.orc_solver_node_info(self.h, _ip(info), _dp(origin))
        keys = ("node", "nodes_x", "nodes_y", "node_x", "node_y", "size_x", "size_y")
        d = dict(zip(keys, info.tolist()))
        d["init_x"], d["init_y"] = origin.tolist()
        return d

    # a node's RK2 step with the halo exchanged between the stages
    def save_old(self):
        self.L.orc_solver_save_old_h(self.h)

    def pre_exchange(self):
        """The stage's work before its halo exchange (the moment filter of
        SOLVER moment, moment_update.cpp:178-179; nothing for momopt)."""
        self.L.orc_solver_pre_exchange_h(self.h)

    def run(self, out_dir, max_steps=-1):
        """main.cpp:204-230 with outputs into out_dir."""
        st = self.L.orc_solver_run_h(self.h, out_dir.encode(), max_steps)
        assert st == 0, "oracle error %d" % st

    def stage_exchanged(self, dt):
        st = self.L.orc_solver_stage_exchanged_h(self.h, dt)
        assert st == 0, "oracle error %d" % st

    def average(self):
        self.L.orc_solver_average_h(self.h)

    def halo_counts(self):
        return [self.L.orc_solver_halo_count_h(self.h, side) for side in range(4)]

    def halo_pack(self, side):
        buf = np.empty(self.L.orc_solver_halo_count_h(self.h, side))
        self.L.orc_solver_halo_h(self.h, side, 1, _dp(buf))
        return buf

    def halo_unpack(self, side, buf):
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        self.L.orc_solver_halo_h(self.h, side, 0, _dp(buf))

    def output(self, time, out_dir):
        st = self.L.orc_solver_output_h(self.h, time, out_dir.encode())
        assert st == 0, "oracle output error %d" % st

    def last_iterations(self):
        it = np.empty(self.NX * self.NY, np.int32)
        self.L.orc_solver_last_iters(self.h, _ip(it))
        return it.reshape(self.NX, self.NY)

    def stats(self):
        mi, im, ns = C.c_int(), C.c_double(), C.c_longlong()
        hist = np.zeros(5, np.int32)
        self.L.orc_solver_stats(self.h, C.byref(mi), C.byref(im), C.byref(ns), _ip(hist))
        return {"max_iter": mi.value, "iter_mean": im.value, "num_solves": ns.value,
                "hist_reg": hist.tolist()}

    def close(self):
        if self.h:
            self.L.orc_solver_close(self.h)
            self.h = None

    def __del__(self):
        self.close()
