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

WORKLOADS = {
    # the M6 / PP6 800x800 pulse (configs of the headline)
    "m6_800": dict(num_cells_x=800, num_cells_y=800, a_x=-1.5, b_x=1.5, a_y=-1.5, b_y=1.5,
                   gaussian_sigma=0.03, floor=1e-8, sigma=1.0, init_cond="gaussian",
                   moment_order=6, quad_order=40, tol=1e-8, use_gaunt=1, t_final=1.0,
                   moment_type="mn"),
    "pp6_800": dict(num_cells_x=800, num_cells_y=800, a_x=-1.5, b_x=1.5, a_y=-1.5, b_y=1.5,
                    gaussian_sigma=0.03, floor=1e-8, sigma=1.0, init_cond="gaussian",
                    moment_order=6, quad_order=40, tol=1e-8, use_gaunt=1, t_final=1.0,
                    moment_type="ppn"),
    # M4 lattice, 200x200 on [-3.5,3.5]^2, Q=30
    "m4_lattice_200": dict(num_cells_x=200, num_cells_y=200, a_x=-3.5, b_x=3.5, a_y=-3.5,
                           b_y=3.5, init_cond="lattice", floor=1e-10, moment_order=4,
                           quad_order=30, tol=1e-8, use_gaunt=1, t_final=3.2),
    # M2 50x50 Gaussian, Q=20 (the reference's CPU-runnable case)
    "m2_50": dict(num_cells_x=50, num_cells_y=50, gaussian_sigma=0.4, floor=1e-4,
                  moment_order=2, quad_order=20, tol=1e-8, use_gaunt=0, t_final=0.5),
}


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
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
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


def write_deck(tmpdir, workload, precision="fp64", opt_type=0, nodes=1, contraction="pairs"):
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
    decks.write_deck(path, decks.deck_text(**kw))
    return path


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_oracle_steps(deck, max_steps, budget_s):
    """The reference algorithm on the host cores (oracle restatement):
    full RK2 steps of the deck from t = 0.  Returns (steps, seconds, solves)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    threads = cpu_threads()
    os.environ["OMP_NUM_THREADS"] = str(threads)
    import pyoracle
    pyoracle.build()
    g = pyoracle.GridSolver(deck)
    C = g.NX * g.NY
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


def reference_arm(args, world, rank):
    if rank != 0:
        return 0
    with tempfile.TemporaryDirectory() as tmp:
        deck = write_deck(tmp, args.workload)
        steps, secs, solves, threads = run_oracle_steps(deck, args.steps, budget_s=150.0)
    value = solves / secs
    w = WORKLOADS[args.workload]
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-solves/s",
        "n_gpus": world, "steps": steps, "warmup": 0, "ms_per_step": 1e3 * secs / steps,
        "steps_per_s": steps / secs, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "grid": [w["num_cells_x"], w["num_cells_y"]],
                   "moment_order": w["moment_order"], "quad_order": w["quad_order"],
                   "use_gaunt": w["use_gaunt"], "tol": w["tol"]},
        "cpu_baseline": {"value": value, "unit": "cell-solves/s", "cores": threads,
                         "kind": "port",
                         "sample": "first %d RK2 step(s) of the deck from t=0, full grid" % steps},
        "e2e": {"value": value, "unit": "cell-solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# DRAM bytes (read + write) per launch of the dominant kernel from one ncu
# capture of the workload: newton on m6_800 (profiles/newton_kernel_m6_800.md;
# algorithmic state traffic of that launch 290 MB read + 433 MB written) and
# a stage-1 pn_stage launch on pn6_800 (profiles/pn_tile_kernel_pn6_800.md;
# algorithmic 2n doubles + 16 bytes per cell = 297 MB, part of the read
# served by L2 from the stage before).
NCU_TRAFFIC = {("m6_800", "newton"): 670.6e6, ("pn6_800", "pn_stage"): 255.6e6}


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
    deck = write_deck(tmp, args.workload, args.precision, args.opt_type, nodes=world,
                      contraction=args.contraction)
    partitioned = world > 1 or args.partitioned
    if partitioned:
        solver = cb.NodeSolver(deck, tmp, node=rank, num_nodes=world)
    else:
        solver = cb.Solver(deck, tmp)
    ctx = solver.context()
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
    f_newton = iters * per_iter + \
        trials * flops_per_trial(n, ang.nq)
    f_flux = 2 * args.steps * flops_flux_stage(C, C_int, n, ang.nq)
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
    ap.add_argument("--newton", default="plain", choices=["plain", "nn"],
                    help="batch workload: start from the isotropic multiplier or a learned prediction")
    ap.add_argument("--nn-steps", type=int, default=4000)
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
