"""Pins the oracle's restatement of the linear Pn/FPn solver (SOLVER moment,
src/moment/*.cpp) against the reference's sixteen regression goldens
(tests/regression/moment/<ic>/<filter>.pn, site_scons/testing.py:252-276):
relative L2 error of the density below the harness's 1e-10
(site_scons/testing.py:9, 168) and every moment within 1e-10 of u0, for one
node and for the 2 x 2 partition the harness also runs (testing.py:269-276,
the MPI build against the same goldens)."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

import closures_b200 as cb
import decks
import helpers
import pyoracle as oracle_lib

ICS = ["delta", "gaussian", "lattice", "smooth"]
FILTERS = ["none", "hauck", "sspline", "lanczos"]
CASES = [(ic, f) for ic in ICS for f in FILTERS]


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    helpers.build_oracle()
    root = tmp_path_factory.mktemp("oracle_moment")
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        jobs = {(ic, f): ex.submit(helpers.run_oracle, decks.regression_moment_deck(ic, f),
                                   str(root / ("%s_%s" % (ic, f))), -1, 2)
                for ic, f in CASES}
        return {k: v.result() for k, v in jobs.items()}


@pytest.mark.parametrize("ic,filt", CASES)
def test_oracle_reproduces_moment_golden(runs, ic, filt):
    h, m = helpers.read_pn(os.path.join(runs[(ic, filt)], "out_1.030_0.pn"))
    hr, mr = helpers.read_moment_golden(ic, filt)
    assert h == hr
    assert helpers.density_rel_l2(m, mr) < 1e-10
    assert helpers.moment_rel_inf(m, mr) < 1e-10
    assert not os.path.exists(os.path.join(runs[(ic, filt)], "out_1.030_0.opt"))


def run_partitioned(deck, nodes_x, nodes_y):
    """main.cpp's time loop to T_FINAL on every node of the partition in one
    process, the halo exchanged between the nodes before each stage after
    the stage's filter (moment_update.cpp:178-182)."""
    nodes = nodes_x * nodes_y
    solvers = [oracle_lib.GridSolver(deck, node=k, num_nodes=nodes) for k in range(nodes)]
    periodic = int(cb.deck_value(deck, "INIT_COND")) == 2
    plans = [cb.HaloPlan(k, nodes_x, nodes_y, periodic) for k in range(nodes)]
    recvs = [[np.zeros(c) for c in s.halo_counts()] for s in solvers]
    t_final = float(cb.deck_value(deck, "T_FINAL"))
    t, dt = 0.0, solvers[0].max_dt
    t_out = min(t + float(cb.deck_value(deck, "OUT_DELTA_T")), t_final)
    while t < t_out:
        t += dt
        if t > t_out:
            dt = t_out - (t - dt)
            t = t_out
        for s in solvers:
            s.save_old()
        for _stage in (1, 2):
            for s in solvers:
                s.pre_exchange()
            sends = [[s.halo_pack(k) for k in cb.SIDES] for s in solvers]
            cb.exchange_local(plans, sends, recvs)
            for s, plan, r in zip(solvers, plans, recvs):
                for k in cb.SIDES:
                    if plan.peer[k] is not None:
                        s.halo_unpack(k, r[k])
                s.stage_exchanged(dt)
        for s in solvers:
            s.average()
    out = [(s.node_info(), s.state()[0]) for s in solvers]
    for s in solvers:
        s.close()
    return out


def assemble(parts, nodes_x, nodes_y):
    """util/formats.py:95-128 (Composite): node blocks into one interior."""
    sx = [parts[x * nodes_y][0]["size_x"] for x in range(nodes_x)]
    sy = [parts[y][0]["size_y"] for y in range(nodes_y)]
    n = parts[0][1].shape[2]
    out = np.zeros((sum(sx), sum(sy), n))
    for info, m in parts:
        x0 = sum(sx[: info["node_x"]])
        y0 = sum(sy[: info["node_y"]])
        out[x0: x0 + info["size_x"], y0: y0 + info["size_y"]] = m[2:-2, 2:-2]
    return out


@pytest.mark.parametrize("ic,filt", [("delta", "none"), ("lattice", "hauck"), ("smooth", "sspline"),
                                     ("gaussian", "lanczos")])
def test_oracle_partitioned_reproduces_moment_golden(tmp_path, ic, filt):
    helpers.build_oracle()
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.regression_moment_deck(ic, filt, partitions=(2, 2)))
    m = assemble(run_partitioned(deck, 2, 2), 2, 2)
    _, mr = helpers.read_moment_golden(ic, filt)
    assert helpers.density_rel_l2(m, mr) < 1e-10
    assert helpers.moment_rel_inf(m, mr) < 1e-10
