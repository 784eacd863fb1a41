"""The linear Pn/FPn solver (SOLVER moment) on the GPU: the reference's
sixteen moment goldens through the drop-in driver, the 2 x 2 partitioned
run the reference's harness also checks against them (testing.py:269-276),
and larger, higher-order grids against the oracle."""
import os

import numpy as np
import pytest

import closures_b200 as cb
import decks
import helpers
import pyoracle as oracle_lib

pytestmark = pytest.mark.gpu

ICS = ["delta", "gaussian", "lattice", "smooth"]
FILTERS = ["none", "hauck", "sspline", "lanczos"]


@pytest.mark.parametrize("ic", ICS)
@pytest.mark.parametrize("filt", FILTERS)
def test_moment_golden(tmp_path, ic, filt):
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.regression_moment_deck(ic, filt))
    cb.run_deck(deck, str(tmp_path))
    h, m = helpers.read_pn(str(tmp_path / "out_1.030_0.pn"))
    hr, mr = helpers.read_moment_golden(ic, filt)
    err_l2 = helpers.density_rel_l2(m, mr)
    err_k = helpers.moment_rel_inf(m, mr)
    print("moment %s/%s: density rel L2 %.3e, moments %.3e" % (ic, filt, err_l2, err_k))
    assert h == hr
    assert err_l2 < 1e-10 and err_k < 1e-10
    assert not os.path.exists(str(tmp_path / "out_1.030_0.opt"))


def _run_nodes_to_final(nodes, t_final, out_delta_t):
    """main.cpp:204-230 on all nodes of a partition (one device)."""
    t, dt = 0.0, nodes[0].max_dt
    t_out = min(t + out_delta_t, t_final)
    while t < t_out:
        t += dt
        if t > t_out:
            dt = t_out - (t - dt)
            t = t_out
        cb.update_nodes_local(nodes, dt)


@pytest.mark.parametrize("ic,filt", [("delta", "none"), ("lattice", "hauck"), ("smooth", "sspline"),
                                     ("gaussian", "lanczos"), ("smooth", "none")])
def test_moment_partitioned_golden(tmp_path, ic, filt):
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.regression_moment_deck(ic, filt, partitions=(2, 2)))
    nodes = [cb.NodeSolver(deck, str(tmp_path), node=k, num_nodes=4) for k in range(4)]
    _run_nodes_to_final(nodes, nodes[0].t_final, nodes[0].out_delta_t)
    sx = [nodes[x * 2].node_info["size_x"] for x in range(2)]
    sy = [nodes[y].node_info["size_y"] for y in range(2)]
    m = np.zeros((sum(sx), sum(sy), nodes[0].n))
    for s in nodes:
        info = s.node_info
        x0, y0 = sum(sx[: info["node_x"]]), sum(sy[: info["node_y"]])
        m[x0: x0 + info["size_x"], y0: y0 + info["size_y"]] = s.moments()[2:-2, 2:-2]
        s.close()
    _, mr = helpers.read_moment_golden(ic, filt)
    err_l2 = helpers.density_rel_l2(m, mr)
    err_k = helpers.moment_rel_inf(m, mr)
    print("moment 2x2 %s/%s: density rel L2 %.3e, moments %.3e" % (ic, filt, err_l2, err_k))
    assert err_l2 < 1e-10 and err_k < 1e-10


@pytest.mark.parametrize("order,filt,ic", [(6, "hauck", "lattice"), (9, "lanczos", "smooth"),
                                           (1, "none", "gaussian")])
def test_moment_steps_match_oracle(tmp_path, order, filt, ic):
    helpers.build_oracle()
    kw = dict(num_cells_x=96, num_cells_y=80, init_cond=ic, moment_order=order,
              quad_order=2 * order + 10, filter_type=filt)
    if ic == "lattice":
        kw.update(a_x=-3.5, b_x=3.5, a_y=-3.5, b_y=3.5, floor=1e-10)
    elif ic == "smooth":
        kw.update(a_x=0.0, b_x=1.0, a_y=0.0, b_y=1.0)
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.moment_deck_text(**kw))
    o = oracle_lib.GridSolver(deck)
    g = cb.Solver(deck, str(tmp_path))
    assert g.kind == cb.CL_SOLVER_MOMENT and g.max_dt == o.max_dt
    for _ in range(10):
        o.steps(1)
        g.update(g.max_dt)
    # interior cells: the ghost strips of a periodic deck are refilled before
    # every stage, and the device state returned between steps keeps the copy
    # taken before the first stage where the reference's holds the second's
    mo = o.state()[0][2:-2, 2:-2]
    mg = g.moments()[2:-2, 2:-2]
    err = float(np.max(np.abs(mg - mo)) / np.max(np.abs(mo[:, :, 0])))
    print("moment order %d %s %s: max |gpu - oracle| / max u0 = %.3e" % (order, filt, ic, err))
    assert err < 1e-12
    o.close()
    g.close()


@pytest.mark.parametrize("order,filt,ic,nx", [(6, "hauck", "gaussian", 200), (3, "none", "lattice", 203),
                                             (9, "lanczos", "gaussian", 70), (2, "sspline", "smooth", 48)])
def test_step_host_equals_device_step(tmp_path, order, filt, ic, nx):
    """cl_pn_step_host (bands of rows uploaded, stepped and read back while
    later bands are still going up; the periodic deck takes the plain calls)
    equals set_state + step + get_state bit for bit."""
    import torch
    kw = dict(num_cells_x=nx, num_cells_y=nx - 6, init_cond=ic, moment_order=order,
              quad_order=2 * order + 10, filter_type=filt)
    if ic == "lattice":
        kw.update(a_x=-3.5, b_x=3.5, a_y=-3.5, b_y=3.5, floor=1e-10)
    elif ic == "smooth":
        kw.update(a_x=0.0, b_x=1.0, a_y=0.0, b_y=1.0)
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.moment_deck_text(**kw))
    a = cb.Solver(deck, str(tmp_path))
    b = cb.Solver(deck, str(tmp_path))
    shape = (a.NX * a.NY, a.n)
    hm = torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    hm[:] = a.moments().reshape(shape)
    for step in range(3):
        b.set_moments(hm)
        b.update(a.max_dt)
        ref = b.moments().reshape(shape)
        a.step_host(a.max_dt, hm)
        np.testing.assert_array_equal(hm, ref, err_msg="step %d" % step)
    a.close()
    b.close()
