"""Python binding of libclosures_gpu.so (include/closures_gpu.h) via ctypes.

Mirrors the reference's interfaces for the Mn/PPn path:
  * ``Solver`` -- MomOptSolver behind the Solver interface (src/solver.h:15-61):
    built from an input.deck, ``update(dt)`` (momopt_update.cpp:283-382),
    ``output_data(time)`` (momopt_output.cpp:21-77);
  * ``Context.solve_batch`` -- the per-vector operator
    ``opt(n, n2, nq, u, alpha, options, w, p, &outs)`` (opt/opt.cpp:82-148),
    batched, in place on u and alpha;
  * ``angular`` -- MomOptSolver::init's quadrature / basis / Gaunt set-up
    (momopt_init.cpp:88-259).
Every call goes to the CUDA library; there is no Python or CPU fallback and
a missing library or device raises ``ClosuresError``.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libclosures_gpu.so")

CL_OK, CL_ERR_ARG, CL_ERR_CUDA, CL_ERR_U0, CL_ERR_MAXREG, CL_ERR_TIMEOUT, CL_ERR_STATE = (
    0, -1, -2, -3, -4, -5, -6)
CL_MN, CL_PPN = 0, 1
CL_FP64, CL_MIXED = 0, 1
CL_SOLVER_MOMOPT, CL_SOLVER_MOMENT = 0, 1
CL_CONTRACT_PAIRS, CL_CONTRACT_SINGLE = 0, 1
REGULARIZATIONS = (0.0, 1e-3, 1e-2, 1e-1, 5e-1)


class ClosuresError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("closures_gpu error %d: %s" % (code, msg))
        self.code = code


class cl_angular(C.Structure):
    _fields_ = [("order", C.c_int), ("quad_order", C.c_int), ("use_gaunt", C.c_int),
                ("n", C.c_int), ("n2", C.c_int), ("nq", C.c_int),
                ("w", C.POINTER(C.c_double)), ("xi", C.POINTER(C.c_double)),
                ("eta", C.POINTER(C.c_double)), ("p", C.POINTER(C.c_double)),
                ("gaunt_nnz", C.c_int), ("gaunt_off", C.POINTER(C.c_int)),
                ("gaunt_idx", C.POINTER(C.c_int)), ("gaunt_val", C.POINTER(C.c_double))]


class cl_options(C.Structure):
    _fields_ = [("moment_type", C.c_int), ("opt_type", C.c_int), ("max_iter", C.c_int),
                ("tol", C.c_double), ("cond_h_max", C.c_double), ("delta_ppn", C.c_double),
                ("tol_gamma", C.c_double), ("precision", C.c_int), ("max_bfgs_iter", C.c_int),
                ("cond_h_max_bfgs", C.c_double), ("contraction", C.c_int)]


class cl_grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("ghost", C.c_int), ("init_cond", C.c_int),
                ("init_x", C.c_double), ("init_y", C.c_double), ("theta", C.c_double)]


class cl_node(C.Structure):
    _fields_ = [("node", C.c_int), ("nodes_x", C.c_int), ("nodes_y", C.c_int), ("node_x", C.c_int),
                ("node_y", C.c_int), ("size_x", C.c_int), ("size_y", C.c_int),
                ("init_x", C.c_double), ("init_y", C.c_double)]


class cl_stats(C.Structure):
    _fields_ = [("max_iter", C.c_int), ("iter_mean", C.c_double), ("num_solves", C.c_int64),
                ("hist_reg", C.c_int64 * 5), ("total_iter", C.c_int64),
                ("total_trials", C.c_int64), ("fallbacks", C.c_int64), ("screened", C.c_int64),
                ("screen_evals", C.c_int64), ("flux_tiles", C.c_int64)]


class cl_tuning(C.Structure):
    _fields_ = [("newton_warps", C.c_int), ("newton_ctas", C.c_int), ("newton_contraction", C.c_int),
                ("flux_contraction", C.c_int), ("from_cache", C.c_int), ("ncand", C.c_int),
                ("cand_kernel", C.c_int * 8), ("cand_warps", C.c_int * 8),
                ("cand_contraction", C.c_int * 8), ("cand_ms", C.c_float * 8), ("screen_ctas", C.c_int)]


_CONTRACTION_NAMES = {0: "pairs", 1: "single"}


def _tuning_dict(t):
    cands = []
    for i in range(t.ncand):
        cands.append({"kernel": "newton" if t.cand_kernel[i] == 1 else "flux",
                      "warps": t.cand_warps[i],
                      "contraction": _CONTRACTION_NAMES.get(t.cand_contraction[i]),
                      "ms": float(t.cand_ms[i])})
    return {"newton_warps": t.newton_warps, "newton_cells_per_cta": 4 * t.newton_warps,
            "newton_ctas": t.newton_ctas,
            "newton_contraction": _CONTRACTION_NAMES.get(t.newton_contraction),
            "flux_contraction": _CONTRACTION_NAMES.get(t.flux_contraction),
            "from_cache": bool(t.from_cache), "candidates": cands, "screen_ctas": t.screen_ctas}


_lib = None


def lib():
    """Loads the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ClosuresError(CL_ERR_STATE, "%s is missing: build it with make -C %s"
                                % (LIB_PATH, HERE))
        L = C.CDLL(LIB_PATH)
        vp, ip, dp = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double)
        sig = {
            "cl_angular_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(cl_angular)]),
            "cl_angular_free": (None, [C.POINTER(cl_angular)]),
            "cl_create": (C.c_int, [C.POINTER(cl_grid), C.POINTER(cl_options),
                                    C.POINTER(cl_angular), dp, dp, dp, dp, C.POINTER(vp)]),
            "cl_destroy": (None, [vp]),
            "cl_last_error": (C.c_char_p, [vp]),
            "cl_global_error": (C.c_char_p, []),
            "cl_error_text": (C.c_char_p, [C.c_int]),
            "cl_step": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
            "cl_step_async": (C.c_int, [vp, C.c_double, C.c_double, C.c_double]),
            "cl_step_timed": (C.c_int, [vp, C.c_double, C.c_double, C.c_double,
                                        C.POINTER(C.c_float)]),
            "cl_sync": (C.c_int, [vp]),
            "cl_get_state": (C.c_int, [vp, dp, dp]),
            "cl_set_state": (C.c_int, [vp, dp, dp]),
            "cl_step_host": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, dp, dp]),
            "cl_get_stats": (C.c_int, [vp, C.POINTER(cl_stats)]),
            "cl_tune": (C.c_int, [vp, C.c_int, C.POINTER(cl_tuning)]),
            "cl_get_tuning": (C.c_int, [vp, C.POINTER(cl_tuning)]),
            "cl_set_launch_shape": (C.c_int, [vp, C.c_int, C.c_int, C.c_int]),
            "cl_set_range_test": (C.c_int, [vp, C.c_int]),
            "cl_set_uniform_flux_skip": (C.c_int, [vp, C.c_int]),
            "cl_get_last_iterations": (C.c_int, [vp, ip]),
            "cl_solve_batch": (C.c_int, [vp, C.c_int, dp, dp, ip, dp, ip]),
            "cl_solve_batch_device": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp]),
            "cl_solve_batch_device_start": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, vp]),
            "cl_solve_batch_cb_device": (C.c_int, [vp, C.c_int, vp, vp, vp, vp, vp, vp, vp]),
            "cl_device_state": (C.c_int, [vp, C.POINTER(vp), C.POINTER(vp)]),
            "cl_multi_create": (C.c_int, [C.c_int, ip, C.c_int, C.c_int, C.POINTER(cl_options),
                                          C.POINTER(vp)]),
            "cl_multi_destroy": (None, [vp]),
            "cl_multi_last_error": (C.c_char_p, [vp]),
            "cl_multi_solve_device": (C.c_int, [vp, ip, C.POINTER(vp), C.POINTER(vp),
                                                C.POINTER(vp), C.POINTER(vp), C.POINTER(vp)]),
            "cl_multi_solve_device_start": (C.c_int, [vp, ip, C.POINTER(vp), C.POINTER(vp),
                                                      C.POINTER(vp), C.POINTER(vp), C.POINTER(vp),
                                                      C.POINTER(vp)]),
            "cl_launch_count": (C.c_int64, []),
            "cl_selftest": (C.c_int, []),
            "cl_fp64_peak": (C.c_int, [C.POINTER(C.c_double)]),
            "cl_exp_check": (C.c_int, [dp, C.c_int, dp, dp]),
            "cl_solver_create": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(vp), dp]),
            "cl_solver_geometry": (C.c_int, [vp, ip, ip, ip, dp, dp, dp, dp]),
            "cl_solver_update": (C.c_int, [vp, C.c_double]),
            "cl_solver_output": (C.c_int, [vp, C.c_double]),
            "cl_solver_context": (vp, [vp]),
            "cl_solver_last_error": (C.c_char_p, [vp]),
            "cl_solver_destroy": (None, [vp]),
            "cl_run_deck": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int]),
            "cl_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_ulonglong,
                                        C.POINTER(vp)]),
            "cl_mlp_destroy": (None, [vp]),
            "cl_mlp_last_error": (C.c_char_p, [vp]),
            "cl_mlp_set_output_scaling": (C.c_int, [vp, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
            "cl_mlp_train": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, C.c_int, C.c_float,
                                       C.c_ulonglong, C.POINTER(C.c_float)]),
            "cl_mlp_predict": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, ip, vp]),
            "cl_mlp_loss_and_grads": (C.c_int, [vp, dp, dp, C.c_int, C.POINTER(C.c_float),
                                                C.POINTER(C.POINTER(C.c_float)),
                                                C.POINTER(C.POINTER(C.c_float))]),
            "cl_mlp_get_params": (C.c_int, [vp, C.POINTER(C.POINTER(C.c_float)),
                                            C.POINTER(C.POINTER(C.c_float))]),
            "cl_mlp_set_params": (C.c_int, [vp, C.POINTER(C.POINTER(C.c_float)),
                                            C.POINTER(C.POINTER(C.c_float))]),
            "cl_set_warm_start": (C.c_int, [vp, vp]),
            "cl_set_warm_start_selective": (C.c_int, [vp, vp, C.c_int]),
            "cl_tc_gemm_bf16": (C.c_int, [vp, vp, C.c_int, C.c_int, C.c_int, vp]),
            "cl_set_last_iterations": (C.c_int, [vp, vp]),
            "cl_mlp_predict_selected": (C.c_int, [vp, vp, vp, C.c_int, vp, C.c_int, vp]),
            "cl_solve_batch_noalloc": (C.c_int, [C.POINTER(cl_angular), C.POINTER(cl_options),
                                                 C.c_int, vp, vp, vp, vp, vp, vp]),
            "cl_noalloc_last_error": (C.c_char_p, []),
            "cl_stage": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_double]),
            "cl_stage_timed": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_double,
                                         C.POINTER(C.c_float)]),
            "cl_stream": (C.c_int, [vp, C.POINTER(vp)]),
            "cl_halo_counts": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
            "cl_halo_pack": (C.c_int, [vp, C.POINTER(vp)]),
            "cl_halo_unpack": (C.c_int, [vp, C.POINTER(vp)]),
            "cl_partition": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                       C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.POINTER(cl_node)]),
            "cl_solver_create_node": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.c_int,
                                                C.POINTER(vp), dp]),
            "cl_solver_node": (C.c_int, [vp, C.POINTER(cl_node)]),
            "cl_solver_stage": (C.c_int, [vp, C.c_int, C.c_double]),
            "cl_solver_kind": (C.c_int, [vp]),
            "cl_solver_get_state": (C.c_int, [vp, dp]),
            "cl_solver_set_state": (C.c_int, [vp, dp]),
            "cl_solver_pn": (vp, [vp]),
            "cl_solver_halo_counts": (C.c_int, [vp, C.POINTER(C.c_longlong)]),
            "cl_solver_halo_pack": (C.c_int, [vp, C.POINTER(vp)]),
            "cl_solver_halo_unpack": (C.c_int, [vp, C.POINTER(vp)]),
            "cl_solver_stream": (C.c_int, [vp, C.POINTER(vp)]),
            "cl_solver_sync": (C.c_int, [vp]),
            "cl_solver_set_exchanged_sides": (C.c_int, [vp, C.c_int]),
            "cl_pn_stage_timed": (C.c_int, [vp, C.c_int, C.c_double, C.c_double, C.c_double,
                                            C.POINTER(C.c_float)]),
            "cl_pn_last_error": (C.c_char_p, [vp]),
            "cl_pn_step_host": (C.c_int, [vp, C.c_double, C.c_double, C.c_double, dp]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _check(rc, msg_fn):
    if rc != CL_OK:
        m = msg_fn()
        raise ClosuresError(rc, m.decode() if isinstance(m, bytes) else str(m))


def global_error():
    return lib().cl_global_error().decode()


def error_text(code):
    """The library's message for a return code (cl_error_text)."""
    return lib().cl_error_text(int(code)).decode()


def launch_count():
    return int(lib().cl_launch_count())


def selftest():
    _check(lib().cl_selftest(), lib().cl_global_error)


def exp_check(x):
    """(table-driven exp, CUDA exp) of the points x, both evaluated on the device."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    fast, ref = np.empty_like(x), np.empty_like(x)
    _check(lib().cl_exp_check(_dp(x), x.size, _dp(fast), _dp(ref)), lib().cl_global_error)
    return fast, ref


def fp64_peak_tflops():
    """Measured FP64 tensor-core throughput of the current device."""
    v = C.c_double()
    _check(lib().cl_fp64_peak(C.byref(v)), lib().cl_global_error)
    return v.value


class Angular:
    """Quadrature, basis and Gaunt table (momopt_init.cpp:88-259) as numpy arrays."""

    def __init__(self, order, quad_order, use_gaunt):
        self._a = cl_angular()
        _check(lib().cl_angular_create(order, quad_order, int(use_gaunt), C.byref(self._a)),
               lib().cl_global_error)
        a = self._a
        self.order, self.quad_order, self.use_gaunt = a.order, a.quad_order, a.use_gaunt
        self.n, self.n2, self.nq = a.n, a.n2, a.nq
        cp = lambda ptr, k: np.ctypeslib.as_array(ptr, shape=(k,)).copy()
        self.w = cp(a.w, a.nq)
        self.xi = cp(a.xi, a.nq)
        self.eta = cp(a.eta, a.nq)
        self.p = cp(a.p, a.nq * a.n2).reshape(a.nq, a.n2)
        if a.use_gaunt:
            self.gaunt_off = cp(a.gaunt_off, a.n * a.n + 1)
            self.gaunt_idx = cp(a.gaunt_idx, a.gaunt_nnz) if a.gaunt_nnz else np.zeros(0, np.int32)
            self.gaunt_val = cp(a.gaunt_val, a.gaunt_nnz) if a.gaunt_nnz else np.zeros(0)
        else:
            self.gaunt_off = self.gaunt_idx = self.gaunt_val = None

    def __del__(self):
        if _lib is not None and hasattr(self, "_a"):
            _lib.cl_angular_free(C.byref(self._a))


def make_options(moment_type=CL_MN, max_iter=100, tol=1e-8, cond_h_max=1e10, delta_ppn=1e-10,
                 tol_gamma=0.0, precision=CL_FP64, opt_type=0, max_bfgs_iter=5, cond_h_max_bfgs=20.0,
                 contraction=0):
    return cl_options(moment_type, opt_type, max_iter, tol, cond_h_max, delta_ppn, tol_gamma,
                      precision, max_bfgs_iter, cond_h_max_bfgs, contraction)


class Context:
    """A grid state on the device (cl_create); also serves batched solves."""

    def __init__(self, grid, options, angular, sigma_t, sigma_s, moments, alpha):
        self._ctx = C.c_void_p()
        self.n = angular.n
        self.NX, self.NY = grid.nx + 4, grid.ny + 4
        st = np.ascontiguousarray(sigma_t, dtype=np.float64)
        ss = np.ascontiguousarray(sigma_s, dtype=np.float64)
        m = np.ascontiguousarray(moments, dtype=np.float64)
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        _check(lib().cl_create(C.byref(grid), C.byref(options), C.byref(angular._a), _dp(st),
                               _dp(ss), _dp(m), _dp(a), C.byref(self._ctx)),
               lib().cl_global_error)

    @classmethod
    def for_batches(cls, angular, options):
        """A minimal 1x1 grid context used only for batched opt() solves."""
        g = cl_grid(1, 1, 2, 0, 0.0, 0.0, 2.0)
        C_ = 25
        n = angular.n
        m = np.zeros((C_, n))
        m[:, 0] = 1.0
        a = np.zeros((C_, n))
        return cls(g, options, angular, np.ones(C_), np.ones(C_), m, a)

    def close(self):
        if self._ctx and not getattr(self, "_borrowed", False):
            lib().cl_destroy(self._ctx)
        self._ctx = C.c_void_p()

    def __del__(self):
        if _lib is not None and getattr(self, "_ctx", None):
            self.close()

    def _err(self):
        return lib().cl_last_error(self._ctx)

    def step(self, dt, dx, dy):
        _check(lib().cl_step(self._ctx, dt, dx, dy), self._err)

    def step_timed(self, dt, dx, dy):
        """One RK2 step kernel by kernel; returns the four kernel durations (ms)."""
        ms = (C.c_float * 4)()
        _check(lib().cl_step_timed(self._ctx, dt, dx, dy, ms), self._err)
        return list(ms)

    def step_async(self, dt, dx, dy):
        _check(lib().cl_step_async(self._ctx, dt, dx, dy), self._err)

    def sync(self):
        _check(lib().cl_sync(self._ctx), self._err)

    def get_state(self):
        m = np.empty((self.NX * self.NY, self.n))
        a = np.empty((self.NX * self.NY, self.n))
        _check(lib().cl_get_state(self._ctx, _dp(m), _dp(a)), self._err)
        return m.reshape(self.NX, self.NY, self.n), a.reshape(self.NX, self.NY, self.n)

    def set_state(self, moments, alpha):
        m = np.ascontiguousarray(moments, dtype=np.float64)
        a = np.ascontiguousarray(alpha, dtype=np.float64)
        _check(lib().cl_set_state(self._ctx, _dp(m), _dp(a)), self._err)

    def step_host(self, dt, dx, dy, moments, alpha):
        """One RK2 step on host arrays ([NX*NY][n] float64, C-contiguous),
        updated in place; page-locked arrays let the copies overlap the
        kernels."""
        for x in (moments, alpha):
            if x.dtype != np.float64 or not x.flags.c_contiguous or x.size != self.NX * self.NY * self.n:
                raise ValueError("step_host needs C-contiguous float64 arrays of NX*NY*n values")
        _check(lib().cl_step_host(self._ctx, dt, dx, dy, _dp(moments), _dp(alpha)), self._err)

    def last_iterations(self):
        it = np.empty(self.NX * self.NY, np.int32)
        _check(lib().cl_get_last_iterations(self._ctx, _ip(it)), self._err)
        return it.reshape(self.NX, self.NY)

    def set_last_iterations(self, iters):
        it = np.ascontiguousarray(iters, dtype=np.int32).reshape(-1)
        assert it.size == self.NX * self.NY
        _check(lib().cl_set_last_iterations(self._ctx, _ip(it)), self._err)

    def stats(self):
        s = cl_stats()
        _check(lib().cl_get_stats(self._ctx, C.byref(s)), self._err)
        return {"max_iter": s.max_iter, "iter_mean": s.iter_mean, "num_solves": s.num_solves,
                "hist_reg": list(s.hist_reg), "total_iter": s.total_iter,
                "total_trials": s.total_trials, "fallbacks": s.fallbacks,
                "screened": s.screened, "screen_evals": s.screen_evals,
                "flux_tiles": s.flux_tiles}

    def solve_batch(self, u, alpha, check=True):
        """opt() on every row of u/alpha (in place).  Returns iters, reg, status."""
        count = u.shape[0]
        assert u.dtype == np.float64 and alpha.dtype == np.float64
        assert u.flags.c_contiguous and alpha.flags.c_contiguous
        iters = np.zeros(count, np.int32)
        reg = np.zeros(count)
        status = np.zeros(count, np.int32)
        rc = lib().cl_solve_batch(self._ctx, count, _dp(u), _dp(alpha), _ip(iters), _dp(reg),
                                  _ip(status))
        if check:
            _check(rc, self._err)
        return iters, reg, status

    def solve_batch_device(self, d_u, d_alpha, d_iters=None, d_reg=None, d_status=None, count=None,
                           d_alpha_start=None):
        """Device-pointer form (torch tensors or raw addresses); with
        d_alpha_start the solve starts there and d_alpha is the fallback start."""
        ptr = lambda t: None if t is None else (t.data_ptr() if hasattr(t, "data_ptr") else int(t))
        _check(lib().cl_solve_batch_device_start(self._ctx, count, ptr(d_u), ptr(d_alpha),
                                                 ptr(d_alpha_start), ptr(d_iters), ptr(d_reg),
                                                 ptr(d_status)), self._err)

    def solve_batch_cb_device(self, d_u, d_P2M, d_alphaP, d_alpha, d_iters=None, d_reg=None,
                              d_status=None, count=None):
        """Change-of-basis solve (opt_type 1 or 2 contexts): per-vector basis and
        alphaP state in/out, alpha out (moment basis)."""
        ptr = lambda t: None if t is None else (t.data_ptr() if hasattr(t, "data_ptr") else int(t))
        _check(lib().cl_solve_batch_cb_device(self._ctx, count, ptr(d_u), ptr(d_P2M), ptr(d_alphaP),
                                              ptr(d_alpha), ptr(d_iters), ptr(d_reg), ptr(d_status)),
               self._err)

    def set_warm_start(self, mlp, min_prev_iters=0):
        """Predict alpha with `mlp` before every optimisation stage (None: off);
        with min_prev_iters > 0 only for the cells whose previous stage took at
        least that many iterations.  The context borrows the network's device
        buffers, so it keeps a reference to `mlp` until the warm start is
        replaced or removed."""
        _check(lib().cl_set_warm_start_selective(self._ctx, mlp._m if mlp is not None else None,
                                                 int(min_prev_iters)), self._err)
        self._warm = mlp

    def tune(self, use_cache=False):
        """Runs the launch-shape autotuner on the current state (cl_tune) and
        returns what it chose and timed (with use_cache, a cached choice for
        this configuration is applied without timing)."""
        t = cl_tuning()
        _check(lib().cl_tune(self._ctx, int(bool(use_cache)), C.byref(t)), self._err)
        return _tuning_dict(t)

    def tuning(self):
        """The launch shapes in use (cl_get_tuning)."""
        t = cl_tuning()
        _check(lib().cl_get_tuning(self._ctx, C.byref(t)), self._err)
        return _tuning_dict(t)

    def set_launch_shape(self, newton_warps=8, newton_contraction=0, flux_contraction=0):
        _check(lib().cl_set_launch_shape(self._ctx, newton_warps, newton_contraction, flux_contraction),
               self._err)

    def set_range_test(self, enable=True):
        """K1's exponent-range convergence test on or off (cl_set_range_test);
        results are the same either way."""
        _check(lib().cl_set_range_test(self._ctx, 1 if enable else 0), self._err)

    def set_uniform_flux_skip(self, enable=True):
        """K2+K3's uniform-tile shortcut on or off (cl_set_uniform_flux_skip);
        results are the same either way, up to the sign of zero."""
        _check(lib().cl_set_uniform_flux_skip(self._ctx, 1 if enable else 0), self._err)

    def stream(self):
        """The context's CUDA stream as a torch.cuda.ExternalStream (for
        events and stream ordering with torch work)."""
        import torch
        st = C.c_void_p()
        _check(lib().cl_stream(self._ctx, C.byref(st)), self._err)
        return torch.cuda.ExternalStream(st.value, device=torch.device("cuda", torch.cuda.current_device()))

    def device_state(self):
        m, a = C.c_void_p(), C.c_void_p()
        _check(lib().cl_device_state(self._ctx, C.byref(m), C.byref(a)), self._err)
        return m.value, a.value


class MultiSolver:
    """Several moment orders at one quadrature order, one persistent launch."""

    def __init__(self, orders, quad_order, use_gaunt, options):
        self._m = C.c_void_p()
        self.orders = list(orders)
        arr = (C.c_int * len(orders))(*orders)
        _check(lib().cl_multi_create(len(orders), arr, quad_order, int(use_gaunt),
                                     C.byref(options), C.byref(self._m)), lib().cl_global_error)

    def solve_device(self, counts, d_u, d_alpha, d_iters=None, d_reg=None, d_status=None,
                     d_alpha_start=None):
        k = len(self.orders)
        ptr = lambda t: None if t is None else (t.data_ptr() if hasattr(t, "data_ptr") else int(t))
        arr = lambda ts: None if ts is None else (C.c_void_p * k)(*[ptr(t) for t in ts])
        cnt = (C.c_int * k)(*counts)
        _check(lib().cl_multi_solve_device_start(self._m, cnt, arr(d_u), arr(d_alpha),
                                                 arr(d_alpha_start), arr(d_iters), arr(d_reg),
                                                 arr(d_status)),
               lambda: lib().cl_multi_last_error(self._m))

    def close(self):
        if self._m:
            lib().cl_multi_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        if _lib is not None and getattr(self, "_m", None):
            self.close()


class Solver:
    """MomOptSolver on the B200, driven like the reference's Solver."""

    def __init__(self, deck_path, out_dir="."):
        self._s = C.c_void_p()
        md = C.c_double()
        _check(lib().cl_solver_create(deck_path.encode(), out_dir.encode(), C.byref(self._s),
                                      C.byref(md)), lib().cl_global_error)
        self._geometry(md.value)

    def _geometry(self, max_dt):
        self.max_dt = max_dt
        nx, ny, n = C.c_int(), C.c_int(), C.c_int()
        dx, dy, tf, odt = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        lib().cl_solver_geometry(self._s, C.byref(nx), C.byref(ny), C.byref(n), C.byref(dx),
                                 C.byref(dy), C.byref(tf), C.byref(odt))
        self.nx, self.ny, self.n = nx.value, ny.value, n.value
        self.dx, self.dy, self.t_final, self.out_delta_t = dx.value, dy.value, tf.value, odt.value
        self.NX, self.NY = self.nx + 4, self.ny + 4

    def _err(self):
        return lib().cl_solver_last_error(self._s)

    def update(self, dt):
        _check(lib().cl_solver_update(self._s, dt), self._err)

    def output_data(self, time):
        _check(lib().cl_solver_output(self._s, time), self._err)

    def context(self):
        """The device context (shares the solver's state; one wrapper per
        solver, so a warm start set through it lives as long as the solver)."""
        c = getattr(self, "_cctx", None)
        if c is None:
            c = Context.__new__(Context)
            c._ctx = C.c_void_p(lib().cl_solver_context(self._s))
            c._borrowed = True
            c.n, c.NX, c.NY = self.n, self.NX, self.NY
            self._cctx = c
        return c

    @property
    def kind(self):
        """CL_SOLVER_MOMOPT or CL_SOLVER_MOMENT (the deck's SOLVER)."""
        return lib().cl_solver_kind(self._s)

    def moments(self):
        """The state (ghosts included) as [NX][NY][n]."""
        m = np.empty((self.NX * self.NY, self.n))
        _check(lib().cl_solver_get_state(self._s, _dp(m)), self._err)
        return m.reshape(self.NX, self.NY, self.n)

    def set_moments(self, m):
        m = np.ascontiguousarray(m, dtype=np.float64)
        _check(lib().cl_solver_set_state(self._s, _dp(m)), self._err)

    def step_host(self, dt, moments):
        """SOLVER moment: one RK2 step on a host state ([NX*NY][n] float64,
        C-contiguous), updated in place; page-locked arrays let the copies
        overlap the stages."""
        pn = lib().cl_solver_pn(self._s)
        if not pn:
            raise ValueError("step_host on a solver without a linear moment stage (use Context.step_host)")
        if moments.dtype != np.float64 or not moments.flags.c_contiguous or \
                moments.size != self.NX * self.NY * self.n:
            raise ValueError("step_host needs a C-contiguous float64 array of NX*NY*n values")
        _check(lib().cl_pn_step_host(pn, dt, self.dx, self.dy, _dp(moments)),
               lambda: lib().cl_pn_last_error(pn))

    def context_state(self):
        """Moments and multipliers (momopt; zeros for the multipliers of the
        linear moment solver, which has none)."""
        ctx = lib().cl_solver_context(self._s)
        if not ctx:
            return self.moments(), np.zeros((self.NX, self.NY, self.n))
        m = np.empty((self.NX * self.NY, self.n))
        a = np.empty((self.NX * self.NY, self.n))
        _check(lib().cl_get_state(ctx, _dp(m), _dp(a)), lambda: lib().cl_last_error(ctx))
        return m.reshape(self.NX, self.NY, self.n), a.reshape(self.NX, self.NY, self.n)

    def last_iterations(self):
        ctx = lib().cl_solver_context(self._s)
        it = np.empty(self.NX * self.NY, np.int32)
        _check(lib().cl_get_last_iterations(ctx, _ip(it)), lambda: lib().cl_last_error(ctx))
        return it.reshape(self.NX, self.NY)

    def stats(self):
        ctx = lib().cl_solver_context(self._s)
        s = cl_stats()
        _check(lib().cl_get_stats(ctx, C.byref(s)), lambda: lib().cl_last_error(ctx))
        return {"max_iter": s.max_iter, "iter_mean": s.iter_mean, "num_solves": s.num_solves,
                "hist_reg": list(s.hist_reg), "total_iter": s.total_iter,
                "total_trials": s.total_trials, "fallbacks": s.fallbacks,
                "screened": s.screened, "screen_evals": s.screen_evals,
                "flux_tiles": s.flux_tiles}

    def close(self):
        if self._s:
            lib().cl_solver_destroy(self._s)
            self._s = C.c_void_p()
        self._cctx = None   # after the context is gone: drops a borrowed warm-start network

    def __del__(self):
        if _lib is not None and getattr(self, "_s", None):
            self.close()


# ---------------------------------------------------------------------------
# Partitioned grids: one node per process (GPU) as the reference's MPI build
# runs them (main.cpp:157-193, comm.cpp:31-147, momopt_boundaries.cpp).

NORTH, SOUTH, EAST, WEST = 0, 1, 2, 3
SIDES = (NORTH, SOUTH, EAST, WEST)
OPPOSITE = {NORTH: SOUTH, SOUTH: NORTH, EAST: WEST, WEST: EAST}


def partition(num_cells_x, num_cells_y, nodes_x, nodes_y, num_nodes, node, ax, ay, bx, by):
    """The block of `node` (main.cpp:157-193) as a dict of cl_node's fields."""
    out = cl_node()
    _check(lib().cl_partition(num_cells_x, num_cells_y, nodes_x, nodes_y, num_nodes, node, ax, ay,
                              bx, by, C.byref(out)), lib().cl_global_error)
    return {f: getattr(out, f) for f, _ in cl_node._fields_}


class HaloPlan:
    """comm.cpp:31-147 for one node: peer[side] is the node that side
    exchanges with -- the neighbour in the partition, across the domain edge
    for the periodic initial condition (INIT_COND 2), itself when the
    partition has one node in that direction -- or None at a domain edge.
    The data a node sends towards `side` fills its peer's ghost strip on the
    opposite side."""

    def __init__(self, node, nodes_x, nodes_y, periodic):
        self.node = node
        nx_, ny_ = node // nodes_y, node % nodes_y
        idx = lambda x, y: (y + nodes_y) % nodes_y + nodes_y * ((x + nodes_x) % nodes_x)
        self.peer = {
            NORTH: idx(nx_, ny_ + 1) if (periodic or ny_ < nodes_y - 1) else None,
            SOUTH: idx(nx_, ny_ - 1) if (periodic or ny_ > 0) else None,
            EAST: idx(nx_ + 1, ny_) if (periodic or nx_ < nodes_x - 1) else None,
            WEST: idx(nx_ - 1, ny_) if (periodic or nx_ > 0) else None,
        }


def exchange_local(plans, sends, recvs):
    """All nodes of a partition in one process: recvs[b][opposite side] <-
    sends[a][side] for every side of every node a with peer b (numpy arrays
    or tensors on one device, in launch order)."""
    for a, plan in enumerate(plans):
        for side in SIDES:
            b = plan.peer[side]
            if b is not None:
                recvs[b][OPPOSITE[side]][...] = sends[a][side]


def exchange_distributed(plan, send, recv, group=None):
    """This process's node of a partition with one process per node
    (torch.distributed ranks = nodes; NCCL on GPUs, gloo on CPUs): the
    point-to-point messages of comm.cpp:99-137 in one batch.  Sends go out in
    side order and each receive is posted in the order of the sender's side,
    so backends that match messages by order (NCCL) and by tag agree; a node
    that is its own peer copies locally, as MPI delivers a message to self."""
    import torch.distributed as dist
    ops = []
    for side in SIDES:
        p = plan.peer[side]
        if p is not None and p != plan.node:
            ops.append(dist.P2POp(dist.isend, send[side], p, group, side))
    for side in SIDES:
        p = plan.peer[OPPOSITE[side]]
        if p is not None and p != plan.node:
            ops.append(dist.P2POp(dist.irecv, recv[OPPOSITE[side]], p, group, side))
    for side in SIDES:
        if plan.peer[side] == plan.node:
            recv[OPPOSITE[side]].copy_(send[side])
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()


def deck_value(deck_path, key):
    """A deck entry as the reference's reader sees it (key case-insensitive,
    first whitespace-separated token after it), or None."""
    with open(deck_path) as f:
        for line in f:
            tok = line.split()
            if len(tok) >= 2 and tok[0].upper() == key.upper():
                return tok[1]
    return None


class NodeSolver(Solver):
    """The solver of one node of the deck's NUM_MPI_PARTITIONS_X x _Y
    partition (num_nodes nodes, this one `node`), stepped as the reference's
    MPI build steps it: before each RK stage the halo strips go to the
    neighbour nodes (comm.cpp:31-147), then the stage runs on the device.
    The halo buffers are device tensors; pack, exchange and unpack are
    ordered with the library's stream, so no host synchronisation is needed
    inside a step.  Output files are out_<t>_<node>.{pn,opt}."""

    def __init__(self, deck_path, out_dir=".", node=0, num_nodes=1, device=None):
        import torch
        self._s = C.c_void_p()
        md = C.c_double()
        _check(lib().cl_solver_create_node(deck_path.encode(), out_dir.encode(), node, num_nodes,
                                           C.byref(self._s), C.byref(md)), lib().cl_global_error)
        self._geometry(md.value)
        info = cl_node()
        lib().cl_solver_node(self._s, C.byref(info))
        self.node_info = {f: getattr(info, f) for f, _ in cl_node._fields_}
        periodic = int(deck_value(deck_path, "INIT_COND") or 0) == 2
        self.plan = HaloPlan(node, info.nodes_x, info.nodes_y, periodic)
        counts = (C.c_longlong * 4)()
        _check(lib().cl_solver_halo_counts(self._s, counts), self._err)
        # the linear solver filters the strips an exchange fills like its
        # interior (moment_update.cpp:178-182)
        mask = sum(1 << k for k in SIDES if self.plan.peer[k] is not None)
        lib().cl_solver_set_exchanged_sides(self._s, mask)
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.send = [torch.empty(int(c), dtype=torch.float64, device=self.device) for c in counts]
        self.recv = [torch.empty(int(c), dtype=torch.float64, device=self.device) for c in counts]
        st = C.c_void_p()
        lib().cl_solver_stream(self._s, C.byref(st))
        self.stream = torch.cuda.ExternalStream(st.value, device=self.device)

    def _ptrs(self, bufs, sides):
        return (C.c_void_p * 4)(*[bufs[k].data_ptr() if k in sides else None for k in SIDES])

    def pack(self):
        """getInnerBoundaries for the sides that have a peer."""
        sides = [k for k in SIDES if self.plan.peer[k] is not None]
        if sides:
            _check(lib().cl_solver_halo_pack(self._s, self._ptrs(self.send, sides)), self._err)

    def unpack(self):
        """setOuterBoundaries for the sides that have a peer (the peer of a
        side sends the strip for it)."""
        sides = [k for k in SIDES if self.plan.peer[k] is not None]
        if sides:
            _check(lib().cl_solver_halo_unpack(self._s, self._ptrs(self.recv, sides)), self._err)

    def stage(self, stage, dt):
        _check(lib().cl_solver_stage(self._s, stage, dt), self._err)

    def stage_timed(self, stage, dt):
        """The stage, waited for: (optimisation ms, flux/update ms)."""
        ms = (C.c_float * 2)()
        ctx = lib().cl_solver_context(self._s)
        if ctx:
            _check(lib().cl_stage_timed(ctx, stage, dt, self.dx, self.dy, ms),
                   lambda: lib().cl_last_error(ctx))
            return ms[0], ms[1]
        # the linear moment solver has no optimisation: (0, stage ms)
        pn = lib().cl_solver_pn(self._s)
        _check(lib().cl_pn_stage_timed(pn, stage, dt, self.dx, self.dy, ms),
               lambda: lib().cl_pn_last_error(pn))
        return 0.0, ms[0]

    def exchange(self, group=None):
        """The halo exchange before a stage: pack on the library's stream,
        the point-to-point messages on the current stream, unpack on the
        library's stream, each waiting for the previous one on the device."""
        import torch
        cur = torch.cuda.current_stream(self.device)
        self.pack()
        cur.wait_stream(self.stream)
        exchange_distributed(self.plan, self.send, self.recv, group)
        self.stream.wait_stream(cur)
        self.unpack()

    def sync(self):
        _check(lib().cl_solver_sync(self._s), self._err)

    def update(self, dt, group=None):
        """One RK2 step with the halo exchanged over torch.distributed before
        each stage (momopt_update.cpp:311, :339)."""
        for stage in (1, 2):
            self.exchange(group)
            self.stage(stage, dt)
        self.sync()


def update_nodes_local(nodes, dt):
    """One RK2 step of all nodes of a partition held by this process (one
    GPU), the halo exchanged by device copies: the partitioned run of the
    reference on one device, for tests and for comparing partitions."""
    import torch
    cur = torch.cuda.current_stream()
    plans = [s.plan for s in nodes]
    for stage in (1, 2):
        for s in nodes:
            s.pack()
            cur.wait_stream(s.stream)
        exchange_local(plans, [s.send for s in nodes], [s.recv for s in nodes])
        for s in nodes:
            s.stream.wait_stream(cur)
            s.unpack()
            s.stage(stage, dt)
    for s in nodes:
        s.sync()


def run_deck_distributed(deck_path, out_dir=".", max_steps=-1, group=None):
    """main.cpp:45-251 on one node per torch.distributed rank (the deck's
    NUM_MPI_PARTITIONS_X x _Y must equal the world size): outputs
    out_<t>_<rank>.{pn,opt} at t = 0 and every OUT_DELTA_T up to T_FINAL."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    s = NodeSolver(deck_path, out_dir, node=rank, num_nodes=world)
    if world > 1:
        dist.barrier(group)   # every rank set up before the first halo batch
    t_final = s.t_final
    t, steps = 0.0, 0
    s.output_data(t)
    t_out = min(t + s.out_delta_t, t_final)
    while t_out <= t_final:
        dt = s.max_dt
        while t < t_out:
            t += dt
            if t > t_out:
                dt = t_out - (t - dt)
                t = t_out
            s.update(dt, group)
            steps += 1
            if 0 <= max_steps <= steps:
                s.close()
                return
        s.output_data(t)
        if t_out > t_final - 1e-12 * t_final:
            break
        t_out = min(t_out + s.out_delta_t, t_final)
    s.close()


def solve_batch_noalloc(angular, options, d_u, d_alpha, count, d_iters=None, d_reg=None,
                        d_status=None, stream=None):
    """Batched opt() on device arrays without any device allocation by the
    library (cl_solve_batch_noalloc): for callers whose device memory is owned
    by another allocator.  Arguments are torch tensors or raw addresses."""
    n = angular.n
    # torch tensors are checked here (the kernel would read and write past a
    # short, strided, host or wrongly typed buffer); raw addresses are the
    # caller's responsibility, as in the C ABI
    _check_device_tensor(d_u, "d_u", "float64", count * n, required=True)
    _check_device_tensor(d_alpha, "d_alpha", "float64", count * n, required=True)
    _check_device_tensor(d_iters, "d_iters", "int32", count)
    _check_device_tensor(d_reg, "d_reg", "float64", count)
    _check_device_tensor(d_status, "d_status", "int32", count)
    if stream is not None and hasattr(stream, "cuda_stream"):   # torch.cuda.Stream
        stream = stream.cuda_stream
    ptr = lambda t: None if t is None else (t.data_ptr() if hasattr(t, "data_ptr") else int(t))
    _check(lib().cl_solve_batch_noalloc(C.byref(angular._a), C.byref(options), count, ptr(d_u),
                                        ptr(d_alpha), ptr(d_iters), ptr(d_reg), ptr(d_status),
                                        None if stream is None else int(stream)),
           lib().cl_noalloc_last_error)


def _check_device_tensor(t, name, dtype, elements, required=False):
    """Raises ValueError unless t is None (optional arguments), a raw address,
    or a contiguous CUDA tensor of `dtype` with at least `elements` entries."""
    if t is None:
        if required:
            raise ValueError("%s is required" % name)
        return
    if not hasattr(t, "data_ptr"):
        return
    if str(t.dtype) != "torch." + dtype:
        raise ValueError("%s must be %s, got %s" % (name, dtype, t.dtype))
    if not t.is_cuda:
        raise ValueError("%s must be a CUDA tensor" % name)
    if not t.is_contiguous():
        raise ValueError("%s must be contiguous" % name)
    if t.numel() < elements:
        raise ValueError("%s holds %d elements, %d needed" % (name, t.numel(), elements))


def tc_gemm_bf16(A, B):
    """C = A . B^T (FP32) for BF16 CUDA tensors A [M x K], B [N x K] on the
    tensor-memory GEMM of the network (cl_tc_gemm_bf16)."""
    import torch
    assert A.dtype == torch.bfloat16 and B.dtype == torch.bfloat16 and A.is_cuda and B.is_cuda
    A, B = A.contiguous(), B.contiguous()
    M, K = A.shape
    N = B.shape[0]
    assert B.shape[1] == K
    C_ = torch.empty((M, N), dtype=torch.float32, device=A.device)
    torch.cuda.synchronize()
    _check(lib().cl_tc_gemm_bf16(A.data_ptr(), B.data_ptr(), M, N, K, C_.data_ptr()), lib().cl_global_error)
    return C_


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


class MLP:
    """Learned warm start: n -> width x3 -> n MLP trained and evaluated by the
    library's kernels (cl_mlp_*)."""

    def __init__(self, n, width, moment_type=CL_MN, delta_ppn=1e-10, seed=1):
        self._m = C.c_void_p()
        self.n, self.width = n, width
        self.dims = [n, width, width, width, n]
        _check(lib().cl_mlp_create(n, width, moment_type, delta_ppn, seed, C.byref(self._m)),
               lib().cl_global_error)

    def _err(self):
        return lib().cl_mlp_last_error(self._m)

    def set_output_scaling(self, mean, std):
        mean = np.ascontiguousarray(mean, dtype=np.float32)
        std = np.ascontiguousarray(std, dtype=np.float32)
        _check(lib().cl_mlp_set_output_scaling(self._m, _fp(mean), _fp(std)), self._err)

    def train(self, d_u, d_alpha, count, steps, batch=4096, lr=1e-3, seed=7, record_loss=True):
        ptr = lambda t: t.data_ptr() if hasattr(t, "data_ptr") else int(t)
        losses = np.zeros(max(steps, 1), np.float32)
        _check(lib().cl_mlp_train(self._m, ptr(d_u), ptr(d_alpha), count, steps, batch, lr, seed,
                                  _fp(losses) if record_loss else None), self._err)
        return losses[:steps]

    def predict(self, d_u, d_alpha, count, fallback_kind=1, stream=None):
        ptr = lambda t: None if t is None else (t.data_ptr() if hasattr(t, "data_ptr") else int(t))
        fb = C.c_int(0)
        _check(lib().cl_mlp_predict(self._m, ptr(d_u), ptr(d_alpha), count, fallback_kind,
                                    C.byref(fb), ptr(stream)), self._err)
        return fb.value

    def _bufs(self, withW=True):
        W = [np.zeros((self.dims[l], self.dims[l + 1]), np.float32) for l in range(4)]
        b = [np.zeros(self.dims[l + 1], np.float32) for l in range(4)]
        PW = (C.POINTER(C.c_float) * 4)(*[_fp(w) for w in W])
        Pb = (C.POINTER(C.c_float) * 4)(*[_fp(x) for x in b])
        return W, b, PW, Pb

    def loss_and_grads(self, u, alpha):
        u = np.ascontiguousarray(u, dtype=np.float64)
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        W, b, PW, Pb = self._bufs()
        loss = C.c_float()
        _check(lib().cl_mlp_loss_and_grads(self._m, _dp(u), _dp(alpha), u.shape[0], C.byref(loss),
                                           PW, Pb), self._err)
        return loss.value, W, b

    def get_params(self):
        W, b, PW, Pb = self._bufs()
        _check(lib().cl_mlp_get_params(self._m, PW, Pb), self._err)
        return W, b

    def set_params(self, W, b):
        W = [np.ascontiguousarray(w, dtype=np.float32) for w in W]
        b = [np.ascontiguousarray(x, dtype=np.float32) for x in b]
        PW = (C.POINTER(C.c_float) * 4)(*[_fp(w) for w in W])
        Pb = (C.POINTER(C.c_float) * 4)(*[_fp(x) for x in b])
        _check(lib().cl_mlp_set_params(self._m, PW, Pb), self._err)

    def close(self):
        if self._m:
            lib().cl_mlp_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        if _lib is not None and getattr(self, "_m", None):
            self.close()


def run_deck(deck_path, out_dir=".", max_steps=-1):
    """main.cpp:204-230 on the device; writes out_<t>_0.{pn,opt} to out_dir."""
    _check(lib().cl_run_deck(deck_path.encode(), out_dir.encode(), max_steps),
           lib().cl_global_error)


def sample_moment_vectors(angular, count, seed=12345, s_range=(0.1, 20.0)):
    """Synthetic realizable moment vectors of the batched-optimisation workload.

    alpha_k ~ N(0, s^2) for k >= 1 with s log-uniform in s_range, alpha_0 set
    so that u_0 = 1, and u = <m exp(alpha.m)> evaluated in FP64 on the same
    quadrature (log-sum-exp scaled).  Returns (u, alpha_exact), each [count, n].
    """
    rng = np.random.default_rng(seed)
    n = angular.n
    P = angular.p[:, :n]                     # [nq, n]
    w = angular.w
    s = np.exp(rng.uniform(np.log(s_range[0]), np.log(s_range[1]), size=count))
    alpha = rng.standard_normal((count, n)) * s[:, None]
    alpha[:, 0] = 0.0
    u = np.empty((count, n))
    p0 = P[0, 0]
    for b in range(0, count, 4096):
        a = alpha[b:b + 4096]
        e = a @ P.T                          # [B, nq]
        mx = e.max(axis=1, keepdims=True)
        ex = np.exp(e - mx) * w[None, :]
        mom = ex @ P                         # [B, n] scaled by exp(-mx)
        # u0 = exp(mx + a0 p0) * mom0 = 1  ->  a0 = -(mx + log mom0) / p0
        a0 = -(mx[:, 0] + np.log(mom[:, 0])) / p0
        alpha[b:b + 4096, 0] = a0
        u[b:b + 4096] = mom / mom[:, :1]
    return u, alpha


def isotropic_alpha(n, count, moment_type=CL_MN, delta=1e-10):
    """opt.cpp:27-46 for u = (1, 0, ..., 0)."""
    a = np.zeros((count, n))
    a[:, 0] = (2.0 * np.sqrt(np.pi) * np.log(0.5 / np.sqrt(np.pi)) if moment_type == CL_MN
               else 1.0 - 4.0 * delta * np.pi)
    return a
