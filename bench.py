#!/usr/bin/env python
"""Headline benchmark of the B200 Mn/PPn entropy-closure path.

Metric: Mn cell-solves per second (one cell-solve = one opt() call on one
cell in one RK stage, ghost cells included, 2 (nx+4)(ny+4) per RK2 step, as
MomOptSolver::update does) at gradient tolerance 1e-8, plus RK2 steps/s.

Default workload: the M6 800x800 deck (n = 28 moments, Q = 40 -> 1600
quadrature points, narrow Gaussian pulse sigma = 0.03, floor 1e-8, Gaunt
Hessian as in the reference's example deck), plain Newton, all FP64,
advanced W warm-up RK2 steps from t = 0 and then timed for K steps.  The
state (646,416 cells x 28 moments x {u, alpha}) is 290 MB, larger than L2,
so no explicit L2 flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]
                  [--workload m6_800|pp6_800|m4_lattice_200|m2_50|pn6_800|batch_2e20]

`value` is timed with CUDA events on the library's stream (kernels only,
state resident on the device).  The `e2e` figure steps a state held in
page-locked host memory through the host-state C ABI call (cl_step_host, or
cl_pn_step_host for the linear solver), which copies it up and back every
step with the copies overlapped with the kernels.

--impl reference times the reference algorithm's CPU implementation (the
oracle restatement, OpenMP over all host threads) on the same deck.
Under torchrun (N ranks, one GPU each) grid workloads run partitioned as the
reference's MPI build runs them: the deck's grid is widened N times in x and
split into N x 1 nodes (NUM_MPI_PARTITIONS_X = N), each rank stepping one
node of the workload's size and exchanging its halo with its neighbours over
NCCL before every RK stage (weak scaling).  The timed region is bracketed by
barriers and the max over ranks is reported.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "closures-2d_b200"))

import decks  # noqa: E402

METRIC = "Mn cell-solves/s at ||grad||<=1e-8 and steps/s: NN warm-start vs plain, 1 B200"

WORKLOADS = decks.WORKLOADS


def flops_per_iteration(n, n2, nq, use_gaunt, nnz):
    """Algorithmic FLOPs of one Newton iteration (FMA = 2, exp not counted):
    alpha.m and the Hessian sums over the quadrature, the Gaunt contraction,
    Cholesky and the small dense solves (fobj.cpp:37-129, opt.cpp:209-318)."""
    if use_gaunt:
        per_q = 2 * n + 2 * n2
        return nq * per_q + 2 * nnz + n ** 3 / 3.0 + 6 * n * n
    return nq * (2 * n + n * (n + 1)) + n ** 3 / 3.0 + 6 * n * n


def flops_per_trial(n, nq):
    """One line-search function evaluation (linesearch.cpp:53-82)."""
    return nq * (2 * n + 2)


def flops_per_screen(n, nq):
    """One evaluation of K1's screening pass: alpha.m and the gradient sums
    over the quadrature (no Hessian columns)."""
    return nq * 4 * n


def uniform_tile_fraction(alpha):
    """Fraction of K2+K3's 16x16 tiles whose tile-plus-halo alpha is one
    value, bit for bit (those tiles apply zero flux without the chunk loop);
    alpha [NX][NY][n] with the ghost cells."""
    NX, NY, _ = alpha.shape
    bits = np.ascontiguousarray(alpha).view(np.int64)
    eq = np.all(bits == bits[2, 2], axis=2)
    tx, ty = (NX - 4 + 15) // 16, (NY - 4 + 15) // 16
    hit = 0
    for bx in range(tx):
        for by in range(ty):
            i0, j0 = 2 + 16 * bx, 2 + 16 * by
            if i0 + 18 <= NX and j0 + 18 <= NY and eq[i0 - 2:i0 + 18, j0 - 2:j0 + 18].all():
                hit += 1
    return hit / (tx * ty)


def newton_flops(s0, s1, per_iter, n, nq):
    """Algorithmic FLOPs of K1 between two stats snapshots: full Newton
    iterations, line-search trials, and the screening pass's evaluations (the
    solves it settled count one iteration in total_iter but did not form the
    Hessian)."""
    iters = s1["total_iter"] - s0["total_iter"]
    trials = s1["total_trials"] - s0["total_trials"]
    screened = s1.get("screened", 0) - s0.get("screened", 0)
    evals = s1.get("screen_evals", 0) - s0.get("screen_evals", 0)
    return (iters - screened) * per_iter + trials * flops_per_trial(n, nq) + evals * flops_per_screen(n, nq)


def flops_flux_stage(C, C_int, n, nq):
    """solveFlux per stage: ansatz alpha.m on all cells, stencil + projection
    on interior cells (momopt_update.cpp:96-202)."""
    return C * nq * 2 * n + C_int * nq * (2 * n + 40)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.path = tempfile.mktemp(prefix="clocks_", suffix=".csv")
        self.gpu = gpu_index
        self.proc = None

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                 "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def write_deck(tmpdir, workload, precision="fp64", opt_type=0, nodes=1, contraction="pairs", tune=True):
    """The workload's deck; with nodes > 1 the grid and domain are widened
    nodes times in x and split into nodes x 1 partitions, so every node holds
    the workload's grid."""
    path = os.path.join(tmpdir, "input.deck")
    kw = dict(WORKLOADS[workload])
    kw["opt_type"] = opt_type
    if nodes > 1:
        kw["num_cells_x"] = kw["num_cells_x"] * nodes
        kw["b_x"] = kw.get("a_x", -1.5) + (kw.get("b_x", 1.5) - kw.get("a_x", -1.5)) * nodes
        kw["partitions"] = (nodes, 1)
    kw["extra"] = {}
    if precision == "mixed":
        kw["extra"]["MOMOPT_GPU_PRECISION"] = "mixed"
    if contraction == "single":
        kw["extra"]["MOMOPT_GPU_CONTRACTION"] = "single"
    if not tune:
        kw["extra"]["MOMOPT_GPU_TUNE"] = "0"
    decks.write_deck(path, decks.deck_text(**kw))
    return path


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_oracle_steps(deck, max_steps, budget_s, skip=0):
    """The reference algorithm on the host cores (oracle restatement):
    `skip` untimed RK2 steps of the deck from t = 0, then up to max_steps
    timed ones within about budget_s.  Returns (steps, seconds, solves)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    threads = cpu_threads()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import pyoracle
    pyoracle.build()
    g = pyoracle.GridSolver(deck)
    C = g.NX * g.NY
    if skip > 0:
        g.steps(skip)
    done, t_total = 0, 0.0
    while done < max_steps:
        t0 = time.perf_counter()
        g.steps(1)
        t_total += time.perf_counter() - t0
        done += 1
        if t_total * (done + 1) / done > budget_s:
            break
    g.close()
    return done, t_total, 2 * C * done, threads


def run_oracle_cb_sample(deck, w, opt_type, budget_s):
    """The reference's change-of-basis solve (opt_type 1: optcb, 2: optbfgs)
    on the host cores (oracle
    restatement, OpenMP over the cells): the first stage's cell-solves of the
    deck from t = 0 (every cell from the reference's initial basis), on a
    random sample of cells grown until it takes about budget_s.
    Returns (cells, seconds, threads)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    threads = cpu_threads()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import pyoracle
    pyoracle.build()
    g = pyoracle.GridSolver(deck)
    m, _ = g.state()
    g.close()
    order, Q = w["moment_order"], w["quad_order"]
    moment_type = 0 if w.get("moment_type", "mn") == "mn" else 1
    u_all = m.reshape(-1, m.shape[-1])
    rng = np.random.default_rng(0)
    count = 2 * threads
    while True:
        idx = rng.choice(u_all.shape[0], size=min(count, u_all.shape[0]), replace=False)
        u = u_all[idx].copy()
        P2M, aP = pyoracle.cb_init(u.shape[1], len(idx), moment_type)
        al = np.zeros_like(u)
        t0 = time.perf_counter()
        pyoracle.optcb_batch(order, Q, u, P2M, aP, al, moment_type=moment_type,
                             tol=w["tol"], opt_type=opt_type)
        secs = time.perf_counter() - t0
        if secs >= 0.3 * budget_s or len(idx) == u_all.shape[0]:
            return len(idx), secs, threads
        count = int(count * min(8.0, max(2.0, budget_s / max(secs, 1e-3))))


REF_BIN = os.path.join(REPO, "oracle", "_ref", "closures_ref")


def run_reference_build(w, side, steps, threads, moment=False, skip=0):
    """The reference's own program (oracle/_ref/closures_ref: its main.cpp,
    solvers and OpenMP loops, compiled from its sources) on a centred
    side x side sub-grid of the workload's deck -- the same cell size, time
    step, closure and initial pulse -- timed as the difference of two runs
    that stop at T_FINAL = (skip + 0.5) dt and (skip + steps + 0.5) dt, so
    that start-up, set-up, the `skip` steps before the window and output
    cancel.  Returns (seconds for RK2 steps skip+1 .. skip+steps, cells with
    ghosts)."""
    nx = w["num_cells_x"]
    dx = (w.get("b_x", 1.5) - w.get("a_x", -1.5)) / nx
    cx = 0.5 * (w.get("b_x", 1.5) + w.get("a_x", -1.5))
    cy = 0.5 * (w.get("b_y", 1.5) + w.get("a_y", -1.5))
    half = 0.5 * side * dx
    sub = dict(w, num_cells_x=side, num_cells_y=side, a_x=cx - half, b_x=cx + half, a_y=cy - half,
               b_y=cy + half)
    if moment:
        # moment_init.cpp:69
        dt = sub.get("cfl_factor", 0.9) * 0.5 * dx
    else:
        dt = decks.max_dt(sub)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
    secs = []
    for k in (skip + 0.5, skip + steps + 0.5):
        with tempfile.TemporaryDirectory() as d:
            kw = dict(sub, t_final=k * dt)
            text = decks.moment_deck_text(**kw) if moment else decks.deck_text(**kw)
            decks.write_deck(os.path.join(d, "input.deck"), text)
            t0 = time.perf_counter()
            r = subprocess.run([REF_BIN], cwd=d, env=env, stdout=subprocess.DEVNULL,
                               stderr=subprocess.DEVNULL)
            secs.append(time.perf_counter() - t0)
            if r.returncode != 0:
                raise RuntimeError("reference program exited with %d" % r.returncode)
    return max(secs[1] - secs[0], 1e-9), (side + 4) ** 2


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    w = WORKLOADS[args.workload]
    if os.path.exists(REF_BIN):
        return reference_build_arm(args, world, w)
    with tempfile.TemporaryDirectory() as tmp:
        deck = write_deck(tmp, args.workload)
        # the native arm's headline window: --t-start, then W warm-up steps
        dt = decks.max_dt(w)
        skip = (int(round(args.t_start / dt)) if args.t_start > 0 else 0) + args.warmup
        steps, secs, solves, threads = run_oracle_steps(deck, args.steps, budget_s=100.0, skip=skip)
    value = solves / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-solves/s",
        "n_gpus": world, "steps": steps, "warmup": skip, "ms_per_step": 1e3 * secs / steps,
        "steps_per_s": steps / secs, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": [w["num_cells_x"], w["num_cells_y"]],
                   "moment_order": w["moment_order"], "quad_order": w["quad_order"],
                   "use_gaunt": w["use_gaunt"], "tol": w["tol"], "t_start": skip * dt},
        "cpu_baseline": {"value": value, "unit": "cell-solves/s", "cores": threads,
                         "kind": "port",
                         "sample": "RK2 steps %d..%d of the deck (the native arm's headline window: "
                                   "%d untimed steps from t=0 first), full grid"
                                   % (skip + 1, skip + steps, skip)},
        "e2e": {"value": value, "unit": "cell-solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def reference_build_arm(args, world, w):
    """--impl reference with the compiled reference: its OpenMP program on
    all host threads, on a bounded sample of the workload (a centred
    sub-grid; see run_reference_build)."""
    threads_all = cpu_threads()
    side = REF_SAMPLE_SIDE.get(args.workload, 64)
    steps = 1
    # the native arm's headline window: --t-start, then W warm-up steps
    skip = (int(round(args.t_start / decks.max_dt(w))) if args.t_start > 0 else 0) + args.warmup
    tried = {}
    for th in sorted({1, threads_all}):
        secs_th, C = run_reference_build(w, side, steps, th, skip=skip)
        tried[th] = secs_th
    # the faster of one thread and all threads: the reference's per-cell
    # dynamic schedule can make all threads slower than one
    threads = min(tried, key=tried.get)
    secs = tried[threads]
    value = 2 * C * steps / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-solves/s",
        "n_gpus": world, "steps": steps, "warmup": skip, "ms_per_step": 1e3 * secs / steps,
        "steps_per_s": steps / secs, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": [w["num_cells_x"], w["num_cells_y"]],
                   "moment_order": w["moment_order"], "quad_order": w["quad_order"],
                   "use_gaunt": w["use_gaunt"], "tol": w["tol"], "t_start": skip * decks.max_dt(w),
                   "sample_grid": [side, side]},
        "cpu_baseline": {"value": value, "unit": "cell-solves/s", "cores": threads, "kind": "reference",
                         "sample": "the reference's own program (its sources compiled -O3 -fopenmp "
                                   "-DUSE_OPENMP with a GSL shim and OpenBLAS) on the centred %dx%d "
                                   "sub-grid of the deck (same cell size, time step and pulse), "
                                   "RK2 step %d (the native arm's headline window starts there), %d OpenMP "
                                   "thread(s): the faster of 1 and all %d"
                                   % (side, side, skip + 1, threads, threads_all),
                         "by_threads": {str(k): 2 * C * steps / v for k, v in tried.items()}},
        "e2e": {"value": value, "unit": "cell-solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# The compiled reference spends most of a step in its flux loop, which
# dispatches every cell of every direction separately (schedule(dynamic,1),
# momopt_update.cpp:119-128), so a step of the full 800 x 800 grid takes tens
# of minutes on the host; the bounded sample is a centred sub-grid.
REF_SAMPLE_SIDE = {"m6_800": 96, "pp6_800": 96, "m4_lattice_200": 96, "m2_50": 50}


# DRAM bytes (read + write) per launch of the dominant kernel from one ncu
# capture each: on m6_800 the K1 group of a stage at t = 3 dt, the screening
# pass (662.8 MB, profiles/screen_kernel_m6_800.md; algorithmic state traffic
# 290 MB read, 290 MB written and 145 MB of saved moments) and K1 over the
# cells it left (8.6 MB, profiles/newton_kernel_m6_800.md); a stage-1
# pn_stage launch on pn6_800 (profiles/pn_tile_kernel_pn6_800.md; algorithmic
# 2n doubles + 16 bytes per cell = 297 MB, part of the read served by L2 from
# the stage before).
NCU_TRAFFIC = {("m6_800", "newton"): 671.4e6, ("pn6_800", "pn_stage"): 255.6e6}


def train_grid_mlp(cb, torch, w, n, harvest, args):
    """Learned warm start for a grid workload: (u, alpha*) pairs from the
    warm-up steps' states, each cell re-solved from its stored multipliers so
    the pair is consistent, then an n -> 256^3 -> n MLP trained on them."""
    dev = torch.device("cuda", torch.cuda.current_device())
    ang = cb.Angular(w["moment_order"], w["quad_order"], w["use_gaunt"])
    bctx = cb.Context.for_batches(ang, cb.make_options(tol=w["tol"]))
    us, als = [], []
    t0 = time.perf_counter()
    for m, a in harvest:
        du = torch.from_numpy(m.reshape(-1, n).copy()).to(dev)
        da = torch.from_numpy(a.reshape(-1, n).copy()).to(dev)
        cnt = du.shape[0]
        st = torch.zeros(cnt, dtype=torch.int32, device=dev)
        rg = torch.zeros(cnt, dtype=torch.float64, device=dev)
        bctx.solve_batch_device(du, da, None, rg, st, count=cnt)
        ok = (st == 0) & (rg == 0)
        us.append(du[ok])
        als.append(da[ok])
    bctx.close()
    u = torch.cat(us).contiguous()
    al = torch.cat(als).contiguous()
    sq = np.sqrt(np.pi)
    x = (u / u[:, :1]).cpu().numpy()
    tgt = al.cpu().numpy().copy()
    tgt[:, 0] -= 2.0 * sq * np.log(u[:, 0].cpu().numpy())
    lin = 2.0 * sq * x
    lin[:, 0] = 2.0 * sq * np.log(0.5 / sq)
    resid = tgt - lin
    net = cb.MLP(n, 256, seed=23)
    net.set_output_scaling(resid.mean(axis=0), resid.std(axis=0) + 1e-3)
    losses = net.train(u, al, u.shape[0], steps=args.nn_steps, batch=4096, lr=1e-3)
    torch.cuda.synchronize()
    return {"mlp": net, "pairs": int(u.shape[0]), "train_steps": args.nn_steps,
            "train_s": time.perf_counter() - t0,
            "loss_first": float(losses[:50].mean()), "loss_last": float(losses[-50:].mean())}


def full_run_steps(t_final, dt):
    """Steps of main.cpp:204-230 for one output interval: dt until t reaches
    t_final, the last one shortened.  Returns (steps, dt of the last step)."""
    t, k, last = 0.0, 0, dt
    while t < t_final:
        t += dt
        k += 1
        if t > t_final:
            last = t_final - (t - dt)
            t = t_final
    return k, last


def single_grid_run(args, cb, torch, solver, deck, w, ang, nnz, local):
    """One GPU, one domain: the headline window (W warm-up steps after
    --t-start, then K timed steps), and unless --quick a window of K steps
    near 0.9 t_final and the whole run to t_final (time to solution), all
    on the same simulation."""
    ctx = solver.context()
    stream = ctx.stream()
    dt, dx, dy = solver.max_dt, solver.dx, solver.dy
    C = solver.NX * solver.NY
    C_int = solver.nx * solver.ny
    n = solver.n
    nfull, last_dt = full_run_steps(solver.t_final, dt)
    per_iter = flops_per_iteration(n, ang.n2, ang.nq, w["use_gaunt"], nnz)
    if args.opt_type != 0:
        # the change of basis adds the two triangular solves of
        # H_P = T^-1 H_M T^-T and the basis update T <- T L (n^3 each)
        per_iter += 3.0 * n ** 3
    peak = cb.fp64_peak_tflops()
    interior = np.zeros((solver.NX, solver.NY), bool)
    interior[2:-2, 2:-2] = True

    def advance(k):
        """k captured-graph steps; device ms between events on the library stream."""
        if k <= 0:
            return 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(k):
            ctx.step_async(dt, dx, dy)
        e1.record(stream)
        ctx.sync()
        return e0.elapsed_time(e1)

    def window(k, t_start):
        """k steps kernel by kernel (CUDA events around every kernel)."""
        uniform = uniform_tile_fraction(ctx.get_state()[1])
        s0 = solver.stats()
        km = np.zeros(4)
        for _ in range(k):
            km += np.array(ctx.step_timed(dt, dx, dy))
        s1 = solver.stats()
        it = ctx.last_iterations()
        solves = 2 * C * k
        iters = s1["total_iter"] - s0["total_iter"]
        trials = s1["total_trials"] - s0["total_trials"]
        newton_ms = float(km[0] + km[2])
        flux_ms = float(km[1] + km[3])
        device_ms = float(km.sum())
        f_newton = newton_flops(s0, s1, per_iter, n, ang.nq)
        # the flux work of the tiles that ran it (a tile with one alpha over
        # tile and halo applies zero flux without the kinetic flux loop)
        tiles = ((solver.NX - 4 + 15) // 16) * ((solver.NY - 4 + 15) // 16)
        run_frac = (s1["flux_tiles"] - s0["flux_tiles"]) / float(2 * k * tiles)
        f_flux = 2 * k * flops_flux_stage(C, C_int, n, ang.nq) * run_frac
        return {
            "t_start": t_start, "steps": k,
            "value": solves / (device_ms * 1e-3),
            "value_interior": 2 * C_int * k / (device_ms * 1e-3),
            "ms_per_step": device_ms / k, "steps_per_s": 1e3 * k / device_ms,
            "iter_mean": iters / solves, "trials_per_solve": trials / solves,
            "fallback_restarts": s1["fallbacks"] - s0["fallbacks"],
            "flux_uniform_tiles": uniform,
            "flux_tiles_run": run_frac,
            "screened_per_solve": (s1["screened"] - s0["screened"]) / solves,
            "screen_evals_per_solve": (s1["screen_evals"] - s0["screen_evals"]) / solves,
            "kernel_ms": {"newton": newton_ms, "flux": flux_ms},
            "newton_tflops": f_newton / (newton_ms * 1e-3) / 1e12,
            "flux_tflops": f_flux / (flux_ms * 1e-3) / 1e12,
            "newton_frac": f_newton / (newton_ms * 1e-3) / 1e12 / peak,
            "iter_hist_last_stage": np.bincount(np.minimum(it.ravel(), 20), minlength=21).tolist(),
            "iter_hist_last_stage_interior": np.bincount(np.minimum(it[interior], 20), minlength=21).tolist(),
            "_device_ms": device_ms, "_iters": iters, "_trials": trials,
        }

    step = 0
    full_ms = 0.0
    s_begin = solver.stats()
    n_adv = int(round(args.t_start / dt)) if args.t_start > 0 else 0
    full_ms += advance(n_adv)
    step += n_adv
    full_ms += advance(args.warmup)
    step += args.warmup
    # launch shapes: the autotuner times its candidates on this state
    tuning = {"headline": ctx.tune() if not args.no_tune else ctx.tuning()}
    head_state = ctx.get_state()
    head_iters = ctx.last_iterations()

    sampler = ClockSampler(local)
    torch.cuda.synchronize()
    sampler.start()
    launches0 = cb.launch_count()
    t0 = time.perf_counter()
    head = window(args.steps, step * dt)
    wall = time.perf_counter() - t0
    launches = cb.launch_count() - launches0
    clocks = sampler.stop()
    full_ms += head["_device_ms"]
    step += args.steps

    # the same window again from the same state with every exact shortcut
    # off (K1's exponent-range test, and with it the screening pass and its
    # copies of repeated starts; K2+K3's uniform tiles): the work of the
    # reference's algorithm, and a check that the shortcuts change no result
    end_state, end_iters = ctx.get_state(), ctx.last_iterations()
    ctx.set_state(*head_state)
    ctx.set_last_iterations(head_iters)
    ctx.set_range_test(False)
    ctx.set_uniform_flux_skip(False)
    full_work = window(args.steps, head["t_start"])
    fw_state = ctx.get_state()
    fw_iters = full_work["_iters"]
    fw_trials = full_work["_trials"]
    if args.opt_type == 0:
        full_work["same_state_as_headline"] = bool(np.array_equal(fw_state[0], end_state[0]) and
                                                   np.array_equal(fw_state[1], end_state[1]))
    else:
        # the per-cell bases (P2M, alphaP) of the change of basis are not part
        # of the state that set_state restores, so the second run starts from
        # the bases the first one ended with
        full_work["same_state_as_headline"] = None
    for key in ("_device_ms", "_iters", "_trials"):
        full_work.pop(key)
    ctx.set_range_test(not args.no_shortcuts)
    ctx.set_uniform_flux_skip(not args.no_shortcuts)
    ctx.set_state(*end_state)
    ctx.set_last_iterations(end_iters)

    # end to end through the C ABI with host buffers: every step uploads the
    # state from pinned host memory, runs the RK2 step and reads it back;
    # the device state is put back afterwards so the run continues from the
    # end of the headline window
    e2e_steps = max(1, min(args.steps, 5))
    saved_m, saved_a = ctx.get_state()
    hm = torch.empty((C, n), dtype=torch.float64).pin_memory().numpy()
    ha = torch.empty((C, n), dtype=torch.float64).pin_memory().numpy()
    hm[:] = saved_m.reshape(C, n)
    ha[:] = saved_a.reshape(C, n)
    s_e2e0 = solver.stats()
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.step_host(dt, dx, dy, hm, ha)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t1
    s_e2e1 = solver.stats()
    e2e_iters = s_e2e1["total_iter"] - s_e2e0["total_iter"]
    e2e_trials = s_e2e1["total_trials"] - s_e2e0["total_trials"]
    ctx.set_state(saved_m, saved_a)
    state_bytes = 2 * C * n * 8

    late, full, late_state, nn = None, None, None, None
    if not args.quick:
        n_late = max(step + 2, int(round(args.late_t * nfull)))
        full_ms += advance(n_late - 2 - step)
        # the learned start's training pairs: the two steps before the window
        harvest = []
        for _ in range(2):
            full_ms += advance(1)
            if args.newton_compare:
                dm, da = cb_device_state_clone(ctx, torch, C, n)
                harvest.append((dm, da))
        step = n_late
        if not args.no_tune:
            tuning["late"] = ctx.tune()
        late_state = ctx.get_state()
        late_iters = ctx.last_iterations()
        late = window(args.steps, step * dt)
        full_ms += late["_device_ms"]
        step += args.steps
        if args.newton_compare and args.opt_type == 0 and args.precision == "fp64":
            plain_end = ctx.get_state()
            s_nn0 = solver.stats()
            nn = nn_compare(args, cb, torch, ctx, w, n, harvest, (late_state, late_iters), plain_end, late,
                            window, step * dt - args.steps * dt)
            ctx.set_warm_start(None)
            ctx.set_state(*plain_end)
            s_nn1 = solver.stats()
            # the comparison's windows are not part of the run
            e2e_iters += s_nn1["total_iter"] - s_nn0["total_iter"]
            e2e_trials += s_nn1["total_trials"] - s_nn0["total_trials"]
        del harvest
        full_ms += advance(nfull - 1 - step)
        km_last = ctx.step_timed(last_dt, dx, dy)
        full_ms += float(sum(km_last))
        step = nfull
        s_full1 = solver.stats()
        solves = 2 * C * nfull
        full = {"steps": nfull, "t_final": solver.t_final, "last_dt": last_dt,
                "device_s": full_ms * 1e-3, "steps_per_s": nfull / (full_ms * 1e-3),
                "value": solves / (full_ms * 1e-3), "value_interior": 2 * C_int * nfull / (full_ms * 1e-3),
                "iter_mean": (s_full1["total_iter"] - s_begin["total_iter"] - e2e_iters - fw_iters) / solves,
                "trials_per_solve": (s_full1["total_trials"] - s_begin["total_trials"] - e2e_trials - fw_trials)
                / solves,
                "max_iter": s_full1["max_iter"],
                "timing": "graph steps timed by CUDA events on the library stream, the two windows "
                          "kernel by kernel; the e2e steps after the headline window are not part of "
                          "it (the state is restored after them)"}

    cpu = None
    if not args.no_cpu_baseline and args.opt_type == 0:
        cpu = cpu_window_sample(deck, head_state, "headline window (t = %.5f)" % head["t_start"])
        if late_state is not None and late is not None:
            cpu["late"] = cpu_window_sample(deck, late_state, "late window (t = %.5f)" % late["t_start"])
    elif not args.no_cpu_baseline:
        cells, secs, threads = run_oracle_cb_sample(deck, w, args.opt_type, budget_s=20.0)
        cpu = {"value": cells / secs, "unit": "cell-solves/s", "cores": threads,
               "kind": "port",
               "sample": "%d random cells of the deck's first stage from t=0 (reference initial "
                         "basis), %s on all %d host threads (oracle restatement, -O3 -fopenmp)"
                         % (cells, "optcb" if args.opt_type == 1 else "optbfgs", threads)}

    dominant = "newton" if head["kernel_ms"]["newton"] >= head["kernel_ms"]["flux"] else "flux"
    achieved = head["newton_tflops"] if dominant == "newton" else head["flux_tflops"]
    for win in (head, late):
        if win is not None:
            for key in ("_device_ms", "_iters", "_trials"):
                win.pop(key)
    line = {
        "metric": METRIC, "value": head["value"], "unit": "cell-solves/s", "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"], "steps_per_s": head["steps_per_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f64, Hessian-only tiles split tf32",
        "data": "synthetic",
        "config": {"workload": args.workload, "grid": [w["num_cells_x"], w["num_cells_y"]],
                   "grid_per_gpu": [w["num_cells_x"], w["num_cells_y"]],
                   "moment_order": w["moment_order"], "n": n, "quad_order": w["quad_order"],
                   "nq": ang.nq, "use_gaunt": w["use_gaunt"], "tol": w["tol"],
                   "moment_type": w.get("moment_type", "mn"),
                   "newton": args.newton, "precision": args.precision, "opt_type": args.opt_type,
                   "contraction": args.contraction, "t_start": head["t_start"],
                   "shortcuts": not args.no_shortcuts,
                   "l2": "state 2x%d MB > L2, no flush" % (C * n * 8 // 2 ** 20),
                   "parallelism": "single"},
        "value_interior": head["value_interior"],
        "iter_mean": head["iter_mean"], "trials_per_solve": head["trials_per_solve"],
        "fallback_restarts": head["fallback_restarts"],
        "kernel_ms": head["kernel_ms"],
        "windows": {"headline": head, "headline_full_work": full_work, "late": late},
        "full_run": full,
        "nn": nn,
        "tuning": tuning,
        "roofline": {
            "bound": "fp64", "kernel": dominant, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": NCU_TRAFFIC.get((args.workload, dominant)),
            "peak_source": "FP64 DMMA m16n8k8 throughput measured live (cl_fp64_peak)",
            "other": {"newton_tflops": head["newton_tflops"], "flux_tflops": head["flux_tflops"],
                      # the same window with every exact shortcut off: K1 and
                      # K2+K3 doing the reference algorithm's work on every cell
                      "full_work_newton_frac": full_work["newton_frac"],
                      "full_work_flux_frac": full_work["flux_tflops"] / peak},
        },
        "cpu_baseline": cpu,
        "e2e": {"value": 2 * C * e2e_steps / e2e_s, "unit": "cell-solves/s",
                "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                "steps": e2e_steps, "call": "cl_step_host (page-locked buffers)",
                "ms_per_step": {"total": 1e3 * e2e_s / e2e_steps}},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    solver.close()
    return 0


def cb_device_state_clone(ctx, torch, C, n):
    """Device copies of the context's moments and multipliers (through the
    host; outside any timed region)."""
    dev = torch.device("cuda", torch.cuda.current_device())
    m, a = ctx.get_state()
    return (torch.from_numpy(m.reshape(C, n)).to(dev), torch.from_numpy(a.reshape(C, n)).to(dev))


def nn_compare(args, cb, torch, ctx, w, n, harvest, late_state, plain_end, plain_win, window, t_late):
    """The learned warm start against the plain (previous-stage) start on the
    late window: an n -> W -> W -> W -> n MLP (W = 512 for M6, 256 below)
    trained by the library's own kernels on (u, alpha*) pairs from the two
    steps before the window, each cell re-solved from its stored multipliers
    so that the pair is consistent; then the same K steps from the same state
    with the prediction for every cell and with the prediction only for the
    cells whose previous stage took >= 3 iterations."""
    dev = torch.device("cuda", torch.cuda.current_device())
    ang = cb.Angular(w["moment_order"], w["quad_order"], w["use_gaunt"])
    bctx = cb.Context.for_batches(ang, cb.make_options(tol=w["tol"]))
    t0 = time.perf_counter()
    us, als = [], []
    for du, da in harvest:
        cnt = du.shape[0]
        st = torch.zeros(cnt, dtype=torch.int32, device=dev)
        rg = torch.zeros(cnt, dtype=torch.float64, device=dev)
        bctx.solve_batch_device(du, da, None, rg, st, count=cnt)
        torch.cuda.synchronize()
        ok = (st == 0) & (rg == 0)
        us.append(du[ok])
        als.append(da[ok])
    bctx.close()
    u = torch.cat(us).contiguous()
    al = torch.cat(als).contiguous()
    harvest_s = time.perf_counter() - t0
    sq = np.sqrt(np.pi)
    x = (u / u[:, :1]).cpu().numpy()
    tgt = al.cpu().numpy().copy()
    tgt[:, 0] -= 2.0 * sq * np.log(u[:, 0].cpu().numpy())
    lin = 2.0 * sq * x
    lin[:, 0] = 2.0 * sq * np.log(0.5 / sq)
    resid = tgt - lin
    width = 512 if n >= 28 else 256
    net = cb.MLP(n, width, seed=23)
    net.set_output_scaling(resid.mean(axis=0), resid.std(axis=0) + 1e-3)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    losses = net.train(u, al, u.shape[0], steps=args.nn_steps, batch=4096, lr=1e-3)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t1
    pairs = int(u.shape[0])
    # inference throughput of the network (its forward GEMMs on the tensor
    # memory path): a prediction for every cell of the window's state
    dm = torch.from_numpy(late_state[0][0].reshape(-1, n).copy()).to(dev)
    dpred = torch.empty_like(dm)
    net.predict(dm, dpred, dm.shape[0], fallback_kind=1)
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    reps = 5
    for _ in range(reps):
        net.predict(dm, dpred, dm.shape[0], fallback_kind=1)
    torch.cuda.synchronize()
    pred_ms = 1e3 * (time.perf_counter() - t2) / reps
    flops_cell = 2.0 * (n * width + 2 * width * width + width * n)
    train_flops = 3.0 * flops_cell * 4096 * args.nn_steps
    del u, al, us, als, dm, dpred
    scale = np.abs(plain_end[0][:, :, :1])
    out = {"network": "%d-%d-%d-%d-%d GELU, BF16 weights, FP32 accumulation" % (n, width, width, width, n),
           "pairs": pairs, "pairs_from": "the 2 RK2 steps before the late window, re-solved",
           "train_steps": args.nn_steps, "batch": 4096, "lr": 1e-3, "train_s": train_s, "harvest_s": harvest_s,
           "loss_first": float(losses[:50].mean()), "loss_last": float(losses[-50:].mean()),
           "train_tflops": train_flops / train_s / 1e12,
           "predict_ms_all_cells": pred_ms,
           "predict_tflops": flops_cell * late_state[0][0].reshape(-1, n).shape[0] / (pred_ms * 1e-3) / 1e12,
           "t_start": t_late,
           "plain": {k: plain_win[k] for k in ("value", "iter_mean", "trials_per_solve", "ms_per_step",
                                               "kernel_ms", "iter_hist_last_stage")},
           "modes": {}}
    late_state, late_iters = late_state
    for mode, min_it in (("every_cell", 0), ("cells_prev_iters_ge_3", 3)):
        # the window's starting point, per-cell iteration counts included
        ctx.set_state(*late_state)
        ctx.set_last_iterations(late_iters)
        ctx.set_warm_start(net, min_prev_iters=min_it)
        win = window(args.steps, t_late)
        m_end, _ = ctx.get_state()
        ctx.set_warm_start(None)
        win.pop("_device_ms", None)
        out["modes"][mode] = {
            "value": win["value"], "speedup_vs_plain": win["value"] / plain_win["value"],
            "iter_mean": win["iter_mean"], "trials_per_solve": win["trials_per_solve"],
            "fallback_restarts": win["fallback_restarts"],
            "fallback_rate": win["fallback_restarts"] / (2 * args.steps * m_end.shape[0] * m_end.shape[1]),
            "ms_per_step": win["ms_per_step"], "kernel_ms": win["kernel_ms"],
            "iter_hist_last_stage": win["iter_hist_last_stage"],
            "max_rel_moment_diff_vs_plain": float(np.max(np.abs(m_end - plain_end[0]) / scale)),
        }
    return out


def cpu_window_sample(deck, state, where):
    """One RK2 step of the reference algorithm on the host cores (oracle
    restatement, OpenMP over all threads) from the GPU run's state at the
    start of a window: the CPU baseline on the same cells and time."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    threads = cpu_threads()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import pyoracle
    pyoracle.build()
    g = pyoracle.GridSolver(deck)
    g.set_state(*state)
    C = g.NX * g.NY
    t0 = time.perf_counter()
    g.steps(1)
    secs = time.perf_counter() - t0
    g.close()
    return {"value": 2 * C / secs, "unit": "cell-solves/s", "cores": threads, "kind": "port",
            "sample": "one RK2 step of the same deck from the GPU run's state at the %s, on all %d host "
                      "threads (oracle restatement, -O3 -fopenmp)" % (where, threads)}



def native_arm(args, world, rank, local):
    import torch
    import closures_b200 as cb

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        # a collective of all ranks first: the halo's point-to-point batches
        # then start on an initialised communicator
        dist.barrier()
    w = WORKLOADS[args.workload]
    tmp = tempfile.mkdtemp(prefix="bench_")
    partitioned = world > 1 or args.partitioned
    # one GPU: the bench runs the autotuner itself after the warm-up steps;
    # partitioned nodes tune in their set-up (the deck default)
    deck = write_deck(tmp, args.workload, args.precision, args.opt_type, nodes=world,
                      contraction=args.contraction, tune=partitioned)
    if partitioned:
        solver = cb.NodeSolver(deck, tmp, node=rank, num_nodes=world)
    else:
        solver = cb.Solver(deck, tmp)
    ctx = solver.context()
    if args.no_shortcuts:
        ctx.set_range_test(False)
        ctx.set_uniform_flux_skip(False)
    dt, dx, dy = solver.max_dt, solver.dx, solver.dy
    C = solver.NX * solver.NY
    C_int = solver.nx * solver.ny
    n = solver.n
    ang = cb.Angular(w["moment_order"], w["quad_order"], w["use_gaunt"])
    nnz = 0
    if w["use_gaunt"]:
        off = ang.gaunt_off
        for i in range(n):
            for j in range(i, n):
                nnz += int(off[i * n + j + 1] - off[i * n + j])

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    if not partitioned:
        return single_grid_run(args, cb, torch, solver, deck, w, ang, nnz, local)

    # warm-up (advances the simulation from t = 0)
    nn_info = None
    harvest = []
    for _ in range(args.warmup):
        solver.update(dt)
        if args.newton == "nn":
            harvest.append(ctx.get_state())
    net = None
    if args.newton == "nn":
        nn_info = train_grid_mlp(cb, torch, w, n, harvest, args)
        net = nn_info.pop("mlp")   # held for the whole run: the context borrows its buffers
        ctx.set_warm_start(net)
    peak = cb.fp64_peak_tflops()

    st0 = solver.stats()
    launches0 = cb.launch_count()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    t0 = time.perf_counter()
    kernel_ms = np.zeros(4)
    exchange_ms = 0.0
    for _ in range(args.steps):
        if partitioned:
            for stage in (1, 2):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(solver.stream)
                solver.exchange()
                e1.record(solver.stream)
                k1, fl = solver.stage_timed(stage, dt)
                kernel_ms[2 * (stage - 1)] += k1
                kernel_ms[2 * (stage - 1) + 1] += fl
                exchange_ms += e0.elapsed_time(e1)
        else:
            kernel_ms += np.array(ctx.step_timed(dt, dx, dy))
    barrier()
    wall = time.perf_counter() - t0
    clocks = sampler.stop()
    launches = cb.launch_count() - launches0
    st1 = solver.stats()
    device_ms = float(kernel_ms.sum()) + exchange_ms
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([device_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        device_ms = float(tt.item())

    solves = 2 * C * args.steps
    value = world * solves / (device_ms * 1e-3)
    iters = st1["total_iter"] - st0["total_iter"]
    trials = st1["total_trials"] - st0["total_trials"]
    newton_ms = float(kernel_ms[0] + kernel_ms[2])
    flux_ms = float(kernel_ms[1] + kernel_ms[3])
    per_iter = flops_per_iteration(n, ang.n2, ang.nq, w["use_gaunt"], nnz)
    if args.opt_type != 0:
        # the change of basis adds the two triangular solves of
        # H_P = T^-1 H_M T^-T and the basis update T <- T L (n^3 each)
        per_iter += 3.0 * n ** 3
    f_newton = newton_flops(st0, st1, per_iter, n, ang.nq)
    tiles = ((solver.NX - 4 + 15) // 16) * ((solver.NY - 4 + 15) // 16)
    run_frac = (st1["flux_tiles"] - st0["flux_tiles"]) / float(2 * args.steps * tiles)
    f_flux = 2 * args.steps * flops_flux_stage(C, C_int, n, ang.nq) * run_frac
    ach_newton = f_newton / (newton_ms * 1e-3) / 1e12
    ach_flux = f_flux / (flux_ms * 1e-3) / 1e12
    dominant = "newton" if newton_ms >= flux_ms else "flux"

    # end to end through the C ABI with host buffers: every step uploads the
    # state from pinned host memory, runs the RK2 step and reads it back
    e2e_steps = max(1, min(args.steps, 5))
    hm = torch.empty((C, n), dtype=torch.float64).pin_memory().numpy()
    ha = torch.empty((C, n), dtype=torch.float64).pin_memory().numpy()
    hm2, ha2 = ctx.get_state()
    hm[:] = hm2.reshape(C, n)
    ha[:] = ha2.reshape(C, n)
    lib = cb.lib()
    parts = np.zeros(3)
    barrier()
    t1 = time.perf_counter()
    for _ in range(e2e_steps):
        if partitioned:
            # upload, the exchanged step of this node, read back
            ta = time.perf_counter()
            ctx.set_state(hm, ha)
            tb = time.perf_counter()
            solver.update(dt)
            tc = time.perf_counter()
            rc = lib.cl_get_state(ctx._ctx, cb._dp(hm), cb._dp(ha))
            if rc:
                raise cb.ClosuresError(rc, lib.cl_last_error(ctx._ctx))
            parts += (tb - ta, tc - tb, time.perf_counter() - tc)
        else:
            # the host-state step: copies overlapped with the kernels
            ctx.step_host(dt, dx, dy, hm, ha)
    barrier()
    e2e_s = time.perf_counter() - t1
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e_value = world * 2 * C * e2e_steps / e2e_s
    state_bytes = 2 * C * n * 8

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline and args.opt_type == 0:
        steps, secs, solves_cpu, threads = run_oracle_steps(deck, 1, budget_s=60.0)
        cpu = {"value": solves_cpu / secs, "unit": "cell-solves/s", "cores": threads,
               "kind": "port",
               "sample": "first RK2 step of the same deck from t=0 on all %d host threads "
                         "(oracle restatement, -O3 -fopenmp)" % threads}
    elif world == 1 and rank == 0 and not args.no_cpu_baseline:
        # the oracle's change-of-basis solve transforms the basis rows at
        # every iteration, so a full step takes minutes on the host: a
        # sample of the first stage's cells instead
        cells, secs, threads = run_oracle_cb_sample(deck, w, args.opt_type, budget_s=20.0)
        cpu = {"value": cells / secs, "unit": "cell-solves/s", "cores": threads,
               "kind": "port",
               "sample": "%d random cells of the deck's first stage from t=0 (reference initial "
                         "basis), %s on all %d host threads (oracle restatement, -O3 -fopenmp)"
                         % (cells, "optcb" if args.opt_type == 1 else "optbfgs", threads)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": device_ms / args.steps, "steps_per_s": 1e3 * args.steps / device_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f64, Hessian-only tiles split tf32",
            "data": "synthetic",
            "config": {"workload": args.workload, "grid": [w["num_cells_x"] * world, w["num_cells_y"]],
                       "grid_per_gpu": [w["num_cells_x"], w["num_cells_y"]],
                       "moment_order": w["moment_order"], "n": n, "quad_order": w["quad_order"],
                       "nq": ang.nq, "use_gaunt": w["use_gaunt"], "tol": w["tol"],
                       "moment_type": w["moment_type"] if "moment_type" in w else "mn",
                       "newton": args.newton, "precision": args.precision, "opt_type": args.opt_type,
                       "contraction": args.contraction,
                       "t_start": args.warmup * dt,
                       "l2": "state 2x%d MB > L2, no flush" % (C * n * 8 // 2 ** 20),
                       "parallelism": ("halo %dx1 (NCCL point-to-point before each RK stage)" % world)
                       if partitioned else "single"},
            "iter_mean": iters / solves, "trials_per_solve": trials / solves,
            "fallback_restarts": st1["fallbacks"] - st0["fallbacks"],
            "nn": nn_info,
            "kernel_ms": {"newton": newton_ms, "flux": flux_ms, "halo_exchange": exchange_ms},
            "roofline": {
                "bound": "fp64", "kernel": dominant,
                "achieved": ach_newton if dominant == "newton" else ach_flux,
                "peak": peak, "unit": "TFLOP/s",
                "frac": (ach_newton if dominant == "newton" else ach_flux) / peak,
                "traffic": NCU_TRAFFIC.get((args.workload, dominant)),
                "peak_source": "FP64 DMMA m16n8k8 throughput measured live (cl_fp64_peak)",
                "other": {"newton_tflops": ach_newton, "flux_tflops": ach_flux},
            },
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-solves/s",
                    "h2d_bytes_per_step": state_bytes, "d2h_bytes_per_step": state_bytes,
                    "steps": e2e_steps,
                    "call": "cl_set_state + cl_solver_update + cl_get_state" if partitioned
                    else "cl_step_host (page-locked buffers)",
                    "ms_per_step": dict(zip(("h2d", "step", "d2h"), (1e3 * parts / e2e_steps).tolist()))
                    if partitioned else {"total": 1e3 * e2e_s / e2e_steps}},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "wall_s": wall,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


BATCH_ORDERS = [5, 4, 3, 2, 1]   # most expensive first (longest-processing-time order)


# The linear Pn/FPn solver (SOLVER moment): a P6 Gaussian pulse on 800 x 800
# with the Hauck filter; the quadrature only builds the flux operators.
PN_WORKLOADS = {
    "pn6_800": dict(num_cells_x=800, num_cells_y=800, a_x=-1.5, b_x=1.5, a_y=-1.5, b_y=1.5,
                    gaussian_sigma=0.03, floor=1e-8, sigma=1.0, init_cond="gaussian", moment_order=6,
                    quad_order=40, filter_type="hauck", filter_tune=100, t_final=1.0),
}
PN_METRIC = "linear Pn cell-updates/s (interior cells x RK stages), 1 B200"


def pn_flops_per_update(n):
    """FLOPs of one interior cell in one stage (FMA = 2): four n x n operator
    products, four stencil combinations and the update."""
    return 8 * n * n + 4 * 7 * n + 10 * n


def pn_arm(args, world, rank, local):
    """The linear moment solver: N x 1 partitions of the workload widened N
    times in x under torchrun (as the grid workloads), one node per rank."""
    import torch
    import closures_b200 as cb

    w = dict(PN_WORKLOADS[args.workload])
    tmp = tempfile.mkdtemp(prefix="bench_pn_")
    if world > 1:
        w["num_cells_x"] *= world
        w["b_x"] = w["a_x"] + (w["b_x"] - w["a_x"]) * world
        w["partitions"] = (world, 1)
    deck = os.path.join(tmp, "input.deck")
    decks.write_deck(deck, decks.moment_deck_text(**w))
    if args.impl == "reference":
        if rank != 0:
            return 0
        steps, secs, _, threads = run_oracle_steps(deck, args.steps, budget_s=150.0)
        nx, ny = PN_WORKLOADS[args.workload]["num_cells_x"], PN_WORKLOADS[args.workload]["num_cells_y"]
        value = 2 * nx * ny * steps / secs
        print(json.dumps({
            "impl": "reference", "metric": PN_METRIC, "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": steps, "warmup": 0, "ms_per_step": 1e3 * secs / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": args.workload, "grid": [nx, ny],
                                            "moment_order": w["moment_order"]},
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                             "sample": "first %d RK2 step(s) of the deck from t=0" % steps},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return 0

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        dist.barrier()
    solver = cb.NodeSolver(deck, tmp, node=rank, num_nodes=world)
    dt, n = solver.max_dt, solver.n
    C_int = solver.nx * solver.ny

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        solver.update(dt)
    peak = cb.fp64_peak_tflops()
    launches0 = cb.launch_count()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    stage_ms, exchange_ms = 0.0, 0.0
    exchanging = any(p is not None for p in solver.plan.peer.values())
    for _ in range(args.steps):
        for stage in (1, 2):
            if exchanging:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(solver.stream)
                solver.exchange()
                e1.record(solver.stream)
            stage_ms += solver.stage_timed(stage, dt)[1]
            if exchanging:
                exchange_ms += e0.elapsed_time(e1)
    barrier()
    clocks = sampler.stop()
    launches = cb.launch_count() - launches0
    device_ms = stage_ms + exchange_ms
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([device_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        device_ms = float(tt.item())
    updates = 2 * C_int * args.steps
    value = world * updates / (device_ms * 1e-3)
    achieved = updates * pn_flops_per_update(n) / (stage_ms * 1e-3) / 1e12

    # end to end: the state from pinned host memory, the step, the state back
    C = solver.NX * solver.NY
    hm = torch.empty((C, n), dtype=torch.float64).pin_memory().numpy()
    hm[:] = solver.moments().reshape(C, n)
    e2e_steps = max(1, min(args.steps, 5))
    barrier()
    t1 = time.perf_counter()
    lib = cb.lib()
    for _ in range(e2e_steps):
        if world > 1:
            # upload, the exchanged step of this node, read back
            solver.set_moments(hm)
            solver.update(dt)
            rc = lib.cl_solver_get_state(solver._s, cb._dp(hm))
            if rc:
                raise cb.ClosuresError(rc, lib.cl_solver_last_error(solver._s))
        else:
            # the host-state step: bands of rows overlapped with the stages
            solver.step_host(dt, hm)
    barrier()
    e2e_s = time.perf_counter() - t1
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())

    cpu = None
    if world == 1 and rank == 0 and not args.no_cpu_baseline:
        steps, secs, _, threads = run_oracle_steps(deck, 1, budget_s=60.0)
        cpu = {"value": 2 * C_int * steps / secs, "unit": "cell-updates/s", "cores": threads,
               "kind": "port", "sample": "first RK2 step of the same deck from t=0 on all %d host "
                                         "threads (oracle restatement, -O3 -fopenmp)" % threads}
    if rank == 0:
        print(json.dumps({
            "metric": PN_METRIC, "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": device_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": args.workload, "grid": [w["num_cells_x"], w["num_cells_y"]],
                       "grid_per_gpu": [PN_WORKLOADS[args.workload]["num_cells_x"], w["num_cells_y"]],
                       "moment_order": w["moment_order"], "n": n, "filter": w["filter_type"],
                       "l2": "state 2x%d MB > L2, no flush" % (C * n * 8 // 2 ** 20),
                       "parallelism": ("halo %dx1 (NCCL point-to-point before each RK stage)" % world)
                       if world > 1 else "single"},
            "kernel_ms": {"pn_stage": stage_ms, "halo_exchange": exchange_ms},
            "roofline": {"bound": "fp64", "kernel": "pn_stage", "achieved": achieved, "peak": peak,
                         "unit": "TFLOP/s", "frac": achieved / peak,
                         "traffic": NCU_TRAFFIC.get((args.workload, "pn_stage")),
                         "peak_source": "FP64 DMMA m16n8k8 throughput measured live (cl_fp64_peak)",
                         "flops_per_update": pn_flops_per_update(n),
                         "hbm_gbs_algorithmic": updates * (2.5 * n * 8 + 16) / (stage_ms * 1e-3) / 1e9},
            "cpu_baseline": cpu,
            "e2e": {"value": world * 2 * C_int * e2e_steps / e2e_s, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": C * n * 8, "d2h_bytes_per_step": C * n * 8, "steps": e2e_steps,
                    "call": "cl_solver_set_state + cl_solver_update + cl_solver_get_state" if world > 1
                    else "cl_pn_step_host (page-locked buffer)"},
            "gpu_launches": int(launches), "clocks": clocks}), flush=True)
    solver.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def sample_batch_torch(angular, count, gen, device):
    """Batched-optimisation workload on the device (FP64): alpha_k ~ N(0, s^2),
    s log-uniform in [0.1, 20], alpha_0 such that u_0 = 1, u = <m e^{alpha.m}>."""
    import torch
    n = angular.n
    P = torch.from_numpy(angular.p[:, :n].copy()).to(device)
    w = torch.from_numpy(angular.w.copy()).to(device)
    s = torch.exp(torch.empty(count, dtype=torch.float64, device=device).uniform_(
        np.log(0.1), np.log(20.0), generator=gen))
    alpha = torch.randn((count, n), dtype=torch.float64, device=device, generator=gen) * s[:, None]
    alpha[:, 0] = 0.0
    u = torch.empty((count, n), dtype=torch.float64, device=device)
    p0 = float(angular.p[0, 0])
    for b in range(0, count, 65536):
        a = alpha[b:b + 65536]
        e = a @ P.T
        mx = e.max(dim=1, keepdim=True).values
        ex = torch.exp(e - mx) * w[None, :]
        mom = ex @ P
        alpha[b:b + 65536, 0] = -(mx[:, 0] + torch.log(mom[:, 0])) / p0
        u[b:b + 65536] = mom / mom[:, :1]
    return u, alpha


def batch_arm(args, world, rank, local):
    """Batched opt() bench: 2^20 vectors of orders 1..5 at Q = 40 in one
    persistent launch from the isotropic start, tolerance 1e-8."""
    import torch
    import closures_b200 as cb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    total = 1 << 20
    Q, gaunt = 40, 1
    gen = torch.Generator(device=dev)
    gen.manual_seed(12345 + rank)
    rng = np.random.default_rng(12345 + rank)
    counts = np.bincount(rng.integers(0, len(BATCH_ORDERS), total), minlength=len(BATCH_ORDERS))
    counts = [int(c) for c in counts]
    angs = [cb.Angular(o, Q, gaunt) for o in BATCH_ORDERS]
    inputs = [sample_batch_torch(a, c, gen, dev) for a, c in zip(angs, counts)]
    u0 = [u for u, _ in inputs]
    a_iso = [torch.from_numpy(cb.isotropic_alpha(a.n, c)).to(dev) for a, c in zip(angs, counts)]
    du = [u.clone() for u in u0]
    da = [a.clone() for a in a_iso]
    dit = [torch.zeros(c, dtype=torch.int32, device=dev) for c in counts]
    dreg = [torch.zeros(c, dtype=torch.float64, device=dev) for c in counts]
    dst = [torch.zeros(c, dtype=torch.int32, device=dev) for c in counts]
    opts = cb.make_options(tol=1e-8)
    m = cb.MultiSolver(BATCH_ORDERS, Q, gaunt, opts)
    nets, dstart = None, None
    train_s = 0.0
    if args.newton == "nn":
        # learned warm start: one network per order, trained on (u, alpha*)
        # pairs the plain GPU Newton solver produces for fresh samples
        t0 = time.perf_counter()
        nets, dstart = [], []
        sqpi = np.sqrt(np.pi)
        for k, (a, o) in enumerate(zip(angs, BATCH_ORDERS)):
            nt = 1 << 18
            ut, _ = sample_batch_torch(a, nt, gen, dev)
            at = torch.from_numpy(cb.isotropic_alpha(a.n, nt)).to(dev)
            stt = torch.zeros(nt, dtype=torch.int32, device=dev)
            rgt = torch.zeros(nt, dtype=torch.float64, device=dev)
            ctx = cb.Context.for_batches(a, opts)
            ctx.solve_batch_device(ut, at, None, rgt, stt, count=nt)
            torch.cuda.synchronize()
            ok = (stt == 0) & (rgt == 0)
            ut, at = ut[ok].contiguous(), at[ok].contiguous()
            ctx.close()
            x = ut.cpu().numpy()
            lin = 2.0 * sqpi * x
            lin[:, 0] = 2.0 * sqpi * np.log(0.5 / sqpi)
            resid = at.cpu().numpy() - lin
            net = cb.MLP(a.n, 256, seed=17 + o)
            net.set_output_scaling(resid.mean(axis=0), resid.std(axis=0) + 1e-3)
            net.train(ut, at, ut.shape[0], steps=args.nn_steps, batch=4096, lr=1e-3,
                      record_loss=False)
            nets.append(net)
            dstart.append(torch.empty_like(a_iso[k]))
        train_s = time.perf_counter() - t0

    def one():
        for k in range(len(counts)):
            du[k].copy_(u0[k])
            da[k].copy_(a_iso[k])
        if nets is not None:
            for k in range(len(counts)):
                nets[k].predict(du[k], dstart[k], counts[k], fallback_kind=2)
        m.solve_device(counts, du, da, dit, dreg, dst, d_alpha_start=dstart)

    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    launches0 = cb.launch_count()
    sampler = ClockSampler(local)
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        one()
    e1.record()
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1)
    launches = cb.launch_count() - launches0
    value = total * args.steps / (ms * 1e-3)
    per = {}
    for k, o in enumerate(BATCH_ORDERS):
        it = dit[k].cpu().numpy()
        per[str(o)] = {"count": counts[k], "iter_mean": float(it.mean()),
                       "hist": np.bincount(np.minimum(it, 40), minlength=41).tolist(),
                       "status_nonzero": int((dst[k] != 0).sum().item())}
    # error against the FP64 oracle on a sample per order (CPU, all threads)
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(REPO, "oracle"))
        os.environ["OMP_NUM_THREADS"] = str(cpu_threads())
        import pyoracle
        pyoracle.build()
        t_cpu, n_cpu = 0.0, 0
        for k, o in enumerate(BATCH_ORDERS):
            sl = slice(0, 2000)
            uo = u0[k][sl].cpu().numpy().copy()
            ao = a_iso[k][sl].cpu().numpy().copy()
            t0 = time.perf_counter()
            it_o, _, st_o = pyoracle.opt_batch(o, Q, gaunt, uo, ao, tol=1e-8)
            t_cpu += time.perf_counter() - t0
            n_cpu += uo.shape[0]
            ug = du[k][sl].cpu().numpy()
            err = np.abs(ug - uo) / np.abs(uo[:, :1])
            per[str(o)]["oracle_max_rel_err"] = float(err.max())
            per[str(o)]["oracle_iter_agree"] = float((it_o == dit[k][sl].cpu().numpy()).mean())
        cpu = {"value": n_cpu / t_cpu, "unit": "cell-solves/s", "cores": cpu_threads(), "kind": "port",
               "sample": "first 2000 vectors of each order, opt() from the isotropic start"}
    else:
        cpu = None
    line = {"metric": METRIC, "value": value * world, "unit": "cell-solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": "batch_2e20", "vectors": total,
                                             "orders": BATCH_ORDERS, "quad_order": Q,
                                             "use_gaunt": gaunt, "tol": 1e-8,
                                             "newton": args.newton,
                                             "start": "mlp prediction (isotropic fallback)"
                                             if nets is not None else "isotropic"},
            "nn_train_s": train_s if nets is not None else None,
            "per_order": per, "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clocks}
    if rank == 0:
        print(json.dumps(line), flush=True)
    m.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--workload", default="m6_800",
                    choices=sorted(WORKLOADS) + ["batch_2e20"] + sorted(PN_WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--t-start", type=float, default=0.0,
                    help="grid workloads: advance to this time (untimed graph steps) before the "
                         "warm-up steps and the headline window")
    ap.add_argument("--late-t", type=float, default=0.9,
                    help="single-GPU grid workloads: start of the second K-step window, as a "
                         "fraction of the run's steps")
    ap.add_argument("--quick", action="store_true",
                    help="single-GPU grid workloads: the headline window only (no late window, "
                         "no run to t_final, no learned-start comparison)")
    ap.add_argument("--newton", default="plain", choices=["plain", "nn"],
                    help="batch workload: start from the isotropic multiplier or a learned prediction")
    ap.add_argument("--nn-steps", type=int, default=20000)
    ap.add_argument("--no-nn", dest="newton_compare", action="store_false",
                    help="single-GPU grid workloads: skip the learned-start comparison on the late window")
    ap.add_argument("--no-tune", action="store_true",
                    help="keep the default launch shapes (no autotuner)")
    ap.add_argument("--no-shortcuts", action="store_true",
                    help="grid workloads: every exact shortcut off for the whole run (K1's "
                         "exponent-range test with the screening pass, K2+K3's uniform tiles)")
    ap.add_argument("--opt-type", type=int, default=0, choices=[0, 1, 2],
                    help="grid workloads: MOMOPT_OPTIMIZATION_TYPE (1: change-of-basis Newton, "
                         "2: BFGS sub-iterations in the change of basis)")
    ap.add_argument("--contraction", default="pairs", choices=["pairs", "single"],
                    help="grid workloads: the quadrature directions phi, phi + pi contracted together "
                         "through the basis parity (default) or one at a time (MOMOPT_GPU_CONTRACTION)")
    ap.add_argument("--partitioned", action="store_true",
                    help="grid workloads: step through the partitioned (halo-exchange) path even "
                         "on one GPU, as a 1 x 1 partition")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                    help="grid workloads: Hessian-only tiles in split TF32 (MOMOPT_GPU_PRECISION mixed)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.workload == "batch_2e20":
        return batch_arm(args, world, rank, local)
    if args.workload in PN_WORKLOADS:
        return pn_arm(args, world, rank, local)
    if args.impl == "reference":
        return reference_arm(args, world, rank)
    return native_arm(args, world, rank, local)


if __name__ == "__main__":
    sys.exit(main())
