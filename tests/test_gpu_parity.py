"""GPU parity: the CUDA path through the C ABI against the oracle and the
reference's goldens.

Tolerances of the all-FP64 path:
  * where the reference algorithm is well conditioned (the reference goldens,
    moment vectors away from the realizability boundary) results agree with
    the oracle to 1e-10 relative (moment k scaled by |u_0|) and iteration
    counts and regularisation decisions agree exactly;
  * near the realizability boundary the reference's own decisions (Armijo
    test, condition estimate, stopping test) are decided by FP64 rounding:
    the oracle built with and without FMA contraction already disagrees
    there.  The GPU must stay inside that reproducibility envelope: no more
    disagreeing vectors than oracle-vs-oracle(FMA) (plus slack), and on the
    vectors where all three agree, moment differences within 1e-10 or the
    envelope's own spread, whichever is larger.
"""
import os

import numpy as np
import pytest

import closures_b200 as cb
import decks
import helpers
import pyoracle as oracle_lib

pytestmark = pytest.mark.gpu

TOL = 1e-10


def test_dmma_layout_selftest():
    cb.selftest()


def _start(a, count, moment_type, u, alpha_exact, warm, seed):
    if moment_type == cb.CL_PPN:
        return cb.isotropic_alpha(a.n, count, cb.CL_PPN, 1e-10)
    if warm:
        return alpha_exact + 1e-3 * np.random.default_rng(seed).standard_normal(alpha_exact.shape)
    return cb.isotropic_alpha(a.n, count)


def _batch_case(order, Q, gaunt, count, moment_type=cb.CL_MN, tol=1e-8, seed=7, s_range=(0.1, 20.0),
                warm=False, envelope=False, contraction=cb.CL_CONTRACT_PAIRS):
    a = cb.Angular(order, Q, gaunt)
    u, alpha_exact = cb.sample_moment_vectors(a, count, seed=seed, s_range=s_range)
    alpha0 = _start(a, count, moment_type, u, alpha_exact, warm, seed)
    opts = cb.make_options(moment_type=moment_type, tol=tol, contraction=contraction)
    ctx = cb.Context.for_batches(a, opts)
    res = {}
    u_g, a_g = u.copy(), alpha0.copy()
    res["gpu"] = (u_g, a_g) + tuple(ctx.solve_batch(u_g, a_g, check=False))
    variants = [("oracle", False)] + ([("fma", True)] if envelope else [])
    for name, fma in variants:
        u_o, a_o = u.copy(), alpha0.copy()
        res[name] = (u_o, a_o) + tuple(oracle_lib.opt_batch(order, Q, gaunt, u_o, a_o,
                                                            moment_type=moment_type, tol=tol,
                                                            fma=fma))
    return a, res, alpha_exact


def _agree(x, y):
    return (x[2] == y[2]) & (x[3] == y[3]) & (x[4] == y[4])


def _du(x, y, mask):
    if not mask.any():
        return 0.0
    return float(np.max(np.abs(x[0] - y[0])[mask] / np.abs(y[0][mask, :1])))


BATCH_CASES = [(1, 20, 0), (2, 20, 0), (2, 20, 1), (3, 30, 1), (4, 30, 0), (4, 40, 1), (5, 40, 1), (5, 30, 0),
               (6, 40, 1), (6, 40, 0)]


@pytest.mark.parametrize("s_max", [2.0, 20.0])
@pytest.mark.parametrize("order,Q,gaunt", BATCH_CASES)
def test_batch_matches_oracle(order, Q, gaunt, s_max):
    """Default contraction: Mn orders whose fused instance takes the
    direction-pair layout run it."""
    _check_batch(*_batch_case(order, Q, gaunt, 700, s_range=(0.1, s_max), envelope=True)[:2])


@pytest.mark.parametrize("order,Q,gaunt", [(2, 20, 1), (3, 30, 0), (4, 30, 0), (6, 40, 1)])
def test_batch_single_contraction_matches_oracle(order, Q, gaunt):
    """One direction at a time (CL_CONTRACT_SINGLE), the layout the
    direction pairs replace by default."""
    _check_batch(*_batch_case(order, Q, gaunt, 700, s_range=(0.1, 20.0), envelope=True,
                              contraction=cb.CL_CONTRACT_SINGLE)[:2])


def _check_batch(a, r):
    g, o, f = r["gpu"], r["oracle"], r["fma"]
    n_go = int((~_agree(g, o)).sum())
    n_fo = int((~_agree(f, o)).sum())
    if n_fo == 0:
        # rounding does not move the reference algorithm on this sample:
        # identical decisions and 1e-10 agreement are required
        assert n_go == 0, "gpu/oracle decisions differ on %d vectors" % n_go
        assert (o[4] == 0).all()
        assert _du(g, o, np.ones(len(o[2]), bool)) < TOL
        np.testing.assert_allclose(g[1], o[1], rtol=0, atol=1e-8 * (1 + np.abs(o[1]).max()))
        return
    assert n_go <= 3 * n_fo + 0.01 * len(o[2]) + 2, "gpu/oracle disagree on %d, fma/oracle on %d" % (
        n_go, n_fo)
    all3 = _agree(g, o) & _agree(f, o) & (o[4] == 0)
    # Rounding moves the reference here.  Two solutions that both meet the
    # stopping test ||g|| <= tol ||u/u0|| differ by at most twice that in the
    # returned moments (u + g); near-singular Hessians (cond ~ 1e9 at s = 20)
    # make the final gradient rounding-dominated at that level, and the
    # quadrature sums run in another order on the device than in either
    # oracle build.
    unorm = float(np.max(np.linalg.norm(o[0][all3] / o[0][all3, :1], axis=1))) if all3.any() else 0.0
    assert _du(g, o, all3) <= max(TOL, 5.0 * _du(f, o, all3), 2.0 * 1e-8 * unorm)


def test_batch_recovers_exact_multipliers():
    a, r, alpha_exact = _batch_case(3, 30, 1, 300, s_range=(0.1, 2.0))
    u_g, a_g, it_g, reg_g, st_g = r["gpu"]
    assert (reg_g == 0).all()
    np.testing.assert_allclose(a_g, alpha_exact, rtol=0, atol=1e-6)


@pytest.mark.parametrize("order,Q,gaunt", [(2, 20, 0), (3, 30, 1), (5, 40, 1)])
def test_batch_matches_oracle_ppn(order, Q, gaunt):
    a, r, _ = _batch_case(order, Q, gaunt, 400, moment_type=cb.CL_PPN, s_range=(0.1, 3.0),
                          envelope=True)
    g, o, f = r["gpu"], r["oracle"], r["fma"]
    assert (g[4] == 0).all() and (o[4] == 0).all()
    n_go = int((~_agree(g, o)).sum())
    n_fo = int((~_agree(f, o)).sum())
    assert n_go <= 3 * n_fo + 0.01 * len(o[2]) + 2
    m = _agree(g, o) & _agree(f, o)
    assert _du(g, o, m) <= max(TOL, 5.0 * _du(f, o, m))


def test_isotropic_known_answer():
    # u = (u0, 0, ...) -> alpha = isotropic alpha scaled, in one iteration
    a = cb.Angular(3, 30, 1)
    u = np.zeros((5, a.n))
    u[:, 0] = [0.5, 1.0, 2.0, 1e-4, 7.0]
    # opt() takes the unscaled multiplier: isotropic alpha for u0 shifted by 2 sqrt(pi) ln u0
    alpha = cb.isotropic_alpha(a.n, 5)
    alpha[:, 0] += 2 * np.sqrt(np.pi) * np.log(u[:, 0])
    ctx = cb.Context.for_batches(a, cb.make_options())
    it, reg, st = ctx.solve_batch(u, alpha)
    assert (st == 0).all() and (it == 1).all() and (reg == 0).all()
    expect = 2 * np.sqrt(np.pi) * np.log(u[:, 0] / (2 * np.sqrt(np.pi)))
    np.testing.assert_allclose(alpha[:, 0], expect, rtol=0, atol=1e-13)
    assert np.abs(alpha[:, 1:]).max() < 1e-13


def test_negative_u0_reports_error():
    a = cb.Angular(2, 20, 0)
    u, _ = cb.sample_moment_vectors(a, 8, seed=3)
    u[5, 0] = -1.0
    alpha = cb.isotropic_alpha(a.n, 8)
    ctx = cb.Context.for_batches(a, cb.make_options())
    it, reg, st = ctx.solve_batch(u, alpha, check=False)
    assert st[5] == cb.CL_ERR_U0
    assert (np.delete(st, 5) == 0).all()
    with pytest.raises(cb.ClosuresError) as e:
        ctx.solve_batch(u.copy(), cb.isotropic_alpha(a.n, 8))
    assert e.value.code == cb.CL_ERR_U0


def test_regularization_ladder_within_envelope():
    # vectors pushed outside the realizable set exercise the whole ladder
    a = cb.Angular(2, 20, 0)
    u, _ = cb.sample_moment_vectors(a, 256, seed=11, s_range=(20.0, 60.0))
    u[:, 1:] *= 1.02
    a0 = cb.isotropic_alpha(a.n, 256)
    ctx = cb.Context.for_batches(a, cb.make_options(tol=1e-8))
    out = {}
    u_g, a_g = u.copy(), a0.copy()
    out["gpu"] = (u_g, a_g) + tuple(ctx.solve_batch(u_g, a_g, check=False))
    for name, fma in (("oracle", False), ("fma", True)):
        u_o, a_o = u.copy(), a0.copy()
        out[name] = (u_o, a_o) + tuple(oracle_lib.opt_batch(2, 20, 0, u_o, a_o, tol=1e-8, fma=fma))
    g, o, f = out["gpu"], out["oracle"], out["fma"]
    assert (o[3] > 0).any(), "case did not reach the ladder"
    reg_go = (g[3] != o[3]).sum()
    reg_fo = (f[3] != o[3]).sum()
    assert reg_go <= 3 * reg_fo + 5
    m = _agree(g, o) & _agree(f, o) & (o[4] == 0)
    # Regularised solves are ill conditioned: both results still satisfy the
    # stopping test ||g|| <= tol ||u|| on the same regularised target, so they
    # can differ by up to 2 tol relative whatever the rounding.
    assert _du(g, o, m) <= max(2 * 1e-8, 5.0 * _du(f, o, m))


GOLDEN = [(ic, t) for ic in ["delta", "gaussian", "lattice", "smooth"] for t in ["mn", "ppn"]]


@pytest.mark.parametrize("ic,t", GOLDEN)
def test_driver_reproduces_reference_golden(tmp_path, ic, t):
    deck = tmp_path / "input.deck"
    decks.write_deck(str(deck), decks.regression_deck(ic, t, extra={"MOMOPT_TOL_GAMMA": "1.1"}))
    cb.run_deck(str(deck), str(tmp_path))
    hdr, cur = helpers.read_pn(str(tmp_path / "out_1.030_0.pn"))
    ghdr, ref = helpers.read_golden(ic, t)
    assert hdr == ghdr
    assert helpers.density_rel_l2(cur, ref) < TOL
    assert helpers.moment_rel_inf(cur, ref) < 1e-9
    opt = open(str(tmp_path / "out_1.030_0.opt")).read().splitlines()
    assert opt[0].startswith("Max number of iterations:")
    assert opt[2] == "Number of optimizations: 524160"


@pytest.mark.parametrize("ic,t", [("gaussian", "mn"), ("smooth", "ppn")])
def test_driver_reproduces_golden_current_algorithm(tmp_path, ic, t):
    deck = tmp_path / "input.deck"
    decks.write_deck(str(deck), decks.regression_deck(ic, t))
    cb.run_deck(str(deck), str(tmp_path))
    _, cur = helpers.read_pn(str(tmp_path / "out_1.030_0.pn"))
    _, ref = helpers.read_golden(ic, t)
    assert helpers.density_rel_l2(cur, ref) < TOL


GRID_CASES = [
    # (name, deck kwargs, steps)
    ("m2_gaussian_q20_nogaunt", dict(num_cells_x=50, num_cells_y=50, gaussian_sigma=0.4,
                                     moment_order=2, quad_order=20, tol=1e-8, use_gaunt=0), 6),
    ("m4_lattice_q30", dict(num_cells_x=40, num_cells_y=40, a_x=-3.5, b_x=3.5, a_y=-3.5, b_y=3.5,
                            init_cond="lattice", floor=1e-10, moment_order=4, quad_order=30,
                            tol=1e-8, use_gaunt=1), 4),
    ("pp3_periodic", dict(num_cells_x=24, num_cells_y=20, init_cond="smooth", moment_order=3,
                          quad_order=20, tol=1e-8, moment_type="ppn", use_gaunt=0), 4),
    ("m6_pulse_q40", dict(num_cells_x=24, num_cells_y=24, gaussian_sigma=0.1, floor=1e-8,
                          moment_order=6, quad_order=40, tol=1e-8, use_gaunt=1), 2),
    # one direction at a time in the flux and the Newton evaluation
    ("m4_lattice_q30_single", dict(num_cells_x=40, num_cells_y=40, a_x=-3.5, b_x=3.5, a_y=-3.5,
                                   b_y=3.5, init_cond="lattice", floor=1e-10, moment_order=4,
                                   quad_order=30, tol=1e-8, use_gaunt=1,
                                   extra={"MOMOPT_GPU_CONTRACTION": "single"}), 4),
    ("pp3_periodic_single", dict(num_cells_x=24, num_cells_y=20, init_cond="smooth", moment_order=3,
                                 quad_order=20, tol=1e-8, moment_type="ppn", use_gaunt=0,
                                 extra={"MOMOPT_GPU_CONTRACTION": "single"}), 4),
]


def _dilate(mask, r):
    """Cells within Chebyshev distance r of a marked cell."""
    out = mask.copy()
    for di in range(-r, r + 1):
        for dj in range(-r, r + 1):
            sh = np.zeros_like(mask)
            src = mask[max(0, -di):mask.shape[0] - max(0, di), max(0, -dj):mask.shape[1] - max(0, dj)]
            sh[max(0, di):max(0, di) + src.shape[0], max(0, dj):max(0, dj) + src.shape[1]] = src
            out |= sh
    return out


@pytest.mark.parametrize("name,kw,steps", GRID_CASES, ids=[c[0] for c in GRID_CASES])
def test_grid_steps_match_oracle(tmp_path, name, kw, steps):
    """Grid steps in lockstep, stage by stage.  Every step starts the GPU and
    both oracle builds from the oracle's state; after each stage the per-cell
    iteration counts show where a decision (Armijo, condition, stopping test,
    ladder) differed between any two of them.  The flux spreads such a cell's
    difference two cells per stage, so every cell farther than that from a
    differing decision must agree with the oracle to 1e-10 relative, except
    cells where a line search took another step length with the same count of
    iterations (a decision the counts do not show): at most 1 % of the cells,
    within the stopping test's resolution 2 tol ||u/u0|| (opt.cpp:286-293).
    The cells within reach are held to the grid bound of a flipped ladder rung
    (r = 1e-3 relative, twice) or three times the oracle builds' own spread."""
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(**kw))
    tol = kw["tol"]
    g = cb.NodeSolver(deck, str(tmp_path), node=0, num_nodes=1)
    ctx = g.context()
    orcs = [oracle_lib.GridSolver(deck, node=0, num_nodes=1), oracle_lib.GridSolver(deck, fma=True, node=0,
                                                                                     num_nodes=1)]
    periodic = int(cb.deck_value(deck, "INIT_COND")) == 2
    plan = cb.HaloPlan(0, 1, 1, periodic)
    recv = [np.zeros(c) for c in orcs[0].halo_counts()]
    dt = g.max_dt
    assert dt == orcs[0].max_dt
    C, n = g.NX * g.NY, g.n
    decided = 0
    for _ in range(steps):
        m0, a0 = orcs[0].state()
        ctx.set_state(m0.reshape(C, n), a0.reshape(C, n))
        orcs[1].set_state(m0, a0)
        for o in orcs:
            o.save_old()
        reach = np.zeros((g.NX, g.NY), bool)
        for stage in (1, 2):
            g.exchange()
            g.stage(stage, dt)
            g.sync()
            for o in orcs:
                if periodic:
                    sends = [o.halo_pack(k) for k in cb.SIDES]
                    cb.exchange_local([plan], [sends], [recv])
                    for k in cb.SIDES:
                        o.halo_unpack(k, recv[k])
                o.stage_exchanged(dt)
                if stage == 2:
                    o.average()
            it_g, it_o, it_f = g.last_iterations(), orcs[0].last_iterations(), orcs[1].last_iterations()
            differ = (it_g != it_o) | (it_f != it_o)
            assert (it_g != it_o).mean() <= 0.01
            decided += int(differ.sum())
            # a stage-1 decision reaches two cells in each of the two fluxes
            reach |= _dilate(differ, 4 if stage == 1 else 2)
        m_g, _ = g.context_state()
        m_o, _ = orcs[0].state()
        m_f, _ = orcs[1].state()
        scale = np.abs(m_o[:, :, :1])
        err = np.max(np.abs(m_g - m_o) / scale, axis=2)
        env = np.max(np.abs(m_f - m_o) / scale, axis=2)
        far = ~reach
        unorm = np.linalg.norm(m_o / m_o[:, :, :1], axis=2)
        step_len = far & (err > TOL)
        assert (err[step_len] <= 2.0 * tol * unorm[step_len]).all(), \
            "%.3e outside the reach of any differing decision" % err[far].max()
        assert step_len.sum() <= max(5, 0.01 * far.sum())
        if reach.any():
            assert err[reach].max() <= max(2e-3, 3.0 * env[reach].max())
    g.close()
    for o in orcs:
        o.close()


def test_multi_order_launch_matches_oracle():
    """Vectors of five moment orders share one persistent launch (cl_multi_*)."""
    import torch

    orders, Q, gaunt = [5, 4, 3, 2, 1], 20, 1
    counts = [120, 200, 150, 300, 64]
    opts = cb.make_options(tol=1e-8)
    m = cb.MultiSolver(orders, Q, gaunt, opts)
    dev = torch.device("cuda", 0)
    host, dev_u, dev_a, dev_it, dev_reg, dev_st = [], [], [], [], [], []
    for order, count in zip(orders, counts):
        a = cb.Angular(order, Q, gaunt)
        u, _ = cb.sample_moment_vectors(a, count, seed=100 + order, s_range=(0.1, 2.0))
        a0 = cb.isotropic_alpha(a.n, count)
        host.append((u, a0))
        dev_u.append(torch.from_numpy(u.copy()).to(dev))
        dev_a.append(torch.from_numpy(a0.copy()).to(dev))
        dev_it.append(torch.zeros(count, dtype=torch.int32, device=dev))
        dev_reg.append(torch.zeros(count, dtype=torch.float64, device=dev))
        dev_st.append(torch.full((count,), 9, dtype=torch.int32, device=dev))
    m.solve_device(counts, dev_u, dev_a, dev_it, dev_reg, dev_st)
    torch.cuda.synchronize()
    for k, (order, count) in enumerate(zip(orders, counts)):
        u, a0 = host[k]
        uo, ao = u.copy(), a0.copy()
        it_o, reg_o, st_o = oracle_lib.opt_batch(order, Q, gaunt, uo, ao, tol=1e-8)
        ug = dev_u[k].cpu().numpy()
        it_g = dev_it[k].cpu().numpy()
        st_g = dev_st[k].cpu().numpy()
        assert (st_g == 0).all() and (st_o == 0).all()
        agree = it_g == it_o
        assert agree.mean() >= 0.98
        assert np.max(np.abs(ug - uo)[agree] / np.abs(uo[agree, :1])) < TOL
    m.close()


def test_driver_binary_reproduces_golden(tmp_path):
    """The drop-in executable bin/closures_gpu (the reference's main.cpp loop
    over the C ABI) run as the reference is run: input.deck in the working
    directory, out_<t>_0.{pn,opt} written beside it."""
    import subprocess
    binary = os.path.join(helpers.PKG_DIR, "bin", "closures_gpu")
    decks.write_deck(str(tmp_path / "input.deck"), decks.regression_deck("gaussian", "mn"))
    r = subprocess.run([binary], cwd=str(tmp_path), capture_output=True, text=True)
    assert r.returncode == 0, r.stdout[-2000:]
    hdr, cur = helpers.read_pn(str(tmp_path / "out_1.030_0.pn"))
    ghdr, ref = helpers.read_golden("gaussian", "mn")
    assert hdr == ghdr
    assert helpers.density_rel_l2(cur, ref) < TOL
    assert (tmp_path / "out_1.030_0.opt").exists()
