"""Partitioned grids on the CPU: the block partition of main.cpp:157-193,
the halo peers of comm.cpp:31-147, the strips of momopt_boundaries.cpp, and
the exchange protocol of closures_b200.exchange_distributed over gloo
(world sizes 2 and 4, one process per node) against the same partitioned run
exchanged in one process."""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import closures_b200 as cb
import decks
import helpers
import pyoracle as oracle_lib


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _partition_formula(cells_x, cells_y, nx_, ny_, node, ax, ay, bx, by):
    """main.cpp:170-191 written out for the check."""
    dx, dy = (bx - ax) / cells_x, (by - ay) / cells_y
    node_x, node_y = node // ny_, node % ny_
    sx = cells_x // nx_
    if node_x < cells_x % nx_:
        sx += 1
        ix = ax + dx * sx * node_x
    else:
        ix = bx - dx * sx * (nx_ - node_x)
    sy = cells_y // ny_
    if node_y < cells_y % ny_:
        sy += 1
        iy = ay + dy * sy * node_y
    else:
        iy = by - dy * sy * (ny_ - node_y)
    return node_x, node_y, sx, sy, ix, iy


@pytest.mark.parametrize("cells,parts", [((10, 7), (1, 1)), ((10, 7), (3, 1)), ((10, 7), (2, 3)),
                                         ((5, 9), (4, 2)), ((64, 64), (2, 2))])
def test_partition_matches_main_cpp(tmp_path, cells, parts):
    ax, ay, bx, by = -1.5, -0.75, 1.25, 2.0
    nodes = parts[0] * parts[1]
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(num_cells_x=cells[0], num_cells_y=cells[1], a_x=ax, b_x=bx,
                                           a_y=ay, b_y=by, partitions=parts, moment_order=1,
                                           quad_order=4))
    total_x = 0
    for node in range(nodes):
        p = cb.partition(cells[0], cells[1], parts[0], parts[1], nodes, node, ax, ay, bx, by)
        nx_, ny_, sx, sy, ix, iy = _partition_formula(cells[0], cells[1], parts[0], parts[1], node,
                                                      ax, ay, bx, by)
        assert (p["node_x"], p["node_y"], p["size_x"], p["size_y"]) == (nx_, ny_, sx, sy)
        assert p["init_x"] == ix and p["init_y"] == iy
        o = oracle_lib.GridSolver(deck, node=node, num_nodes=nodes).node_info()
        assert (o["size_x"], o["size_y"], o["node_x"], o["node_y"]) == (sx, sy, nx_, ny_)
        assert o["init_x"] == ix and o["init_y"] == iy
        if p["node_y"] == 0:
            total_x += p["size_x"]
    assert total_x == cells[0]


def test_partition_errors():
    with pytest.raises(cb.ClosuresError) as e:
        cb.partition(3, 8, 4, 1, 4, 0, 0, 0, 1, 1)
    assert "larger than number of cells" in str(e.value)
    with pytest.raises(cb.ClosuresError) as e:
        cb.partition(8, 8, 2, 2, 3, 0, 0, 0, 1, 1)
    assert "numPartitionsX * numPartitionsY" in str(e.value)


def test_halo_plan_peers():
    # comm.cpp:14-29 (mpiIndex) and the send conditions of :61-137
    p = cb.HaloPlan(0, 1, 1, periodic=False)
    assert all(p.peer[k] is None for k in cb.SIDES)
    p = cb.HaloPlan(0, 1, 1, periodic=True)
    assert all(p.peer[k] == 0 for k in cb.SIDES)
    # 3 x 2 nodes, node = node_x * 2 + node_y
    p = cb.HaloPlan(2, 3, 2, periodic=False)      # node_x 1, node_y 0
    assert (p.peer[cb.NORTH], p.peer[cb.SOUTH], p.peer[cb.EAST], p.peer[cb.WEST]) == (3, None, 4, 0)
    p = cb.HaloPlan(2, 3, 2, periodic=True)
    assert (p.peer[cb.NORTH], p.peer[cb.SOUTH], p.peer[cb.EAST], p.peer[cb.WEST]) == (3, 3, 4, 0)
    p = cb.HaloPlan(5, 3, 2, periodic=True)       # node_x 2, node_y 1
    assert (p.peer[cb.NORTH], p.peer[cb.SOUTH], p.peer[cb.EAST], p.peer[cb.WEST]) == (4, 4, 1, 3)
    # the neighbour relation is symmetric across opposite sides
    for periodic in (False, True):
        plans = [cb.HaloPlan(k, 3, 2, periodic) for k in range(6)]
        for a, pa in enumerate(plans):
            for side in cb.SIDES:
                b = pa.peer[side]
                if b is not None:
                    assert plans[b].peer[cb.OPPOSITE[side]] == a


def test_halo_strips_match_boundaries_cpp(tmp_path):
    """Pack/unpack of the oracle node against the index formulas of
    momopt_boundaries.cpp:30-188 on a state of distinct values."""
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(num_cells_x=7, num_cells_y=5, partitions=(2, 1),
                                           moment_order=1, quad_order=4))
    g = oracle_lib.GridSolver(deck, node=1, num_nodes=2)
    m, a = g.state()
    NX, NY, n = m.shape
    m = np.arange(m.size, dtype=np.float64).reshape(m.shape)
    g.set_state(m, a)
    sx, sy = NX - 4, NY - 4
    north = g.halo_pack(cb.NORTH).reshape(2, sx, n)
    east = g.halo_pack(cb.EAST).reshape(2, sy, n)
    for j in range(2):
        np.testing.assert_array_equal(north[j], m[2:NX - 2, NY - 4 + j])
        np.testing.assert_array_equal(east[j], m[NX - 4 + j, 2:NY - 2])
    np.testing.assert_array_equal(g.halo_pack(cb.SOUTH).reshape(2, sx, n)[1], m[2:NX - 2, 3])
    np.testing.assert_array_equal(g.halo_pack(cb.WEST).reshape(2, sy, n)[0], m[2, 2:NY - 2])
    g.halo_unpack(cb.WEST, -np.ones(2 * sy * n))
    g.halo_unpack(cb.NORTH, -2 * np.ones(2 * sx * n))
    m2, _ = g.state()
    assert (m2[0:2, 2:NY - 2] == -1).all() and (m2[2:NX - 2, NY - 2:] == -2).all()
    # corners untouched
    assert (m2[0:2, 0:2] == m[0:2, 0:2]).all() and (m2[0:2, NY - 2:] == m[0:2, NY - 2:]).all()


def _run_local(deck, nodes, steps):
    """The partitioned oracle run with every node in this process."""
    solvers = [oracle_lib.GridSolver(deck, node=k, num_nodes=nodes) for k in range(nodes)]
    periodic = int(cb.deck_value(deck, "INIT_COND")) == 2
    info = solvers[0].node_info()
    plans = [cb.HaloPlan(k, info["nodes_x"], info["nodes_y"], periodic) for k in range(nodes)]
    recvs = [[np.zeros(c) for c in s.halo_counts()] for s in solvers]
    for _ in range(steps):
        for s in solvers:
            s.save_old()
        for _stage in (1, 2):
            sends = [[s.halo_pack(k) for k in cb.SIDES] for s in solvers]
            cb.exchange_local(plans, sends, recvs)
            for s, plan, r in zip(solvers, plans, recvs):
                for k in cb.SIDES:
                    if plan.peer[k] is not None:
                        s.halo_unpack(k, r[k])
                s.stage_exchanged(s.max_dt)
        for s in solvers:
            s.average()
    return [s.state() for s in solvers]


CASES = [
    ("gaussian_2x1", dict(num_cells_x=14, num_cells_y=10, gaussian_sigma=0.4, partitions=(2, 1))),
    ("periodic_2x2", dict(num_cells_x=12, num_cells_y=10, init_cond="smooth", partitions=(2, 2),
                          a_x=0.0, b_x=1.0, a_y=0.0, b_y=1.0)),
    ("lattice_1x2", dict(num_cells_x=28, num_cells_y=30, init_cond="lattice", partitions=(1, 2),
                         a_x=-3.5, b_x=3.5, a_y=-3.5, b_y=3.5, floor=1e-10)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_exchange_over_gloo_matches_in_process_run(tmp_path, name, kw):
    helpers.build_oracle()
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(moment_order=2, quad_order=12, tol=1e-8, **kw))
    nodes = kw["partitions"][0] * kw["partitions"][1]
    steps = 2
    local = _run_local(deck, nodes, steps)
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(_free_port()),
               WORLD_SIZE=str(nodes), OMP_NUM_THREADS="1")
    worker = os.path.join(os.path.dirname(os.path.abspath(__file__)), "node_worker.py")
    procs = []
    for rank in range(nodes):
        out = str(tmp_path / ("node%d.npz" % rank))
        procs.append((subprocess.Popen([sys.executable, worker, deck, str(steps), out],
                                       env=dict(env, RANK=str(rank)), stdout=subprocess.PIPE,
                                       stderr=subprocess.STDOUT), out))
    for p, _ in procs:
        try:
            log = p.communicate(timeout=240)[0].decode(errors="replace")
        except subprocess.TimeoutExpired:
            for q, _ in procs:
                q.kill()
            raise
        assert p.returncode == 0, log[-3000:]
    for rank, (_, out) in enumerate(procs):
        r = np.load(out)
        m_loc, a_loc = local[rank]
        np.testing.assert_array_equal(r["moments"], m_loc)
        np.testing.assert_array_equal(r["alpha"], a_loc)


def test_partitioned_run_close_to_single_node(tmp_path):
    """A partitioned run differs from the single-node run only through the
    ghost cells' first solves (their multipliers start from the floor value,
    as in the reference's MPI build): agreement to the Newton tolerance."""
    helpers.build_oracle()
    kw = dict(num_cells_x=14, num_cells_y=10, gaussian_sigma=0.4, moment_order=2, quad_order=12,
              tol=1e-10)
    deck1 = str(tmp_path / "one.deck")
    decks.write_deck(deck1, decks.deck_text(**kw))
    deck2 = str(tmp_path / "two.deck")
    decks.write_deck(deck2, decks.deck_text(partitions=(2, 2), **kw))
    one = oracle_lib.GridSolver(deck1)
    one.steps(2)
    m1, _ = one.state()
    parts = _run_local(deck2, 4, 2)
    # reassemble the interior as util/formats.py Composite does
    sx = [parts[k * 2][0].shape[0] - 4 for k in range(2)]
    sy = [parts[k][0].shape[1] - 4 for k in range(2)]
    for k, (m, _) in enumerate(parts):
        x0 = sum(sx[: k // 2])
        y0 = sum(sy[: k % 2])
        ref = m1[2 + x0: 2 + x0 + sx[k // 2], 2 + y0: 2 + y0 + sy[k % 2]]
        got = m[2:-2, 2:-2]
        assert np.max(np.abs(got - ref) / np.abs(ref[:, :, :1])) < 1e-7
