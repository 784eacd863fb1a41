"""K1's exponent-range convergence test (cl_set_range_test) and the
screening pass that uses it.

At a Mn evaluation whose gradient meets the tolerance, the reference
(opt.cpp:244-306) factors H, estimates its condition number and converges
when the estimate is at most MOMOPT_COND_H_MAX.  K1 decides that outcome
without forming H when the range of alpha . p over the quadrature (bounded
from the multipliers) bounds cond(H) below MOMOPT_COND_H_MAX / 4.  With the
direction-pair layout, a screening pass evaluates every cell first with the
gradient columns only and settles the cells that converge there; K1 solves
the rest from their starts.  Both only skip work, so every result must be
bit-identical with the test off, where each evaluation goes through K1's
Hessian, its factorisation and the condition bounds.  K2+K3's uniform-tile
shortcut likewise: the same states with every tile running the flux loop.
"""
import numpy as np
import pytest

import closures_b200 as cb
import decks

pytestmark = pytest.mark.gpu

M6 = dict(num_cells_x=60, num_cells_y=60, gaussian_sigma=0.08, floor=1e-8, moment_order=6, quad_order=40,
          tol=1e-8, use_gaunt=1)
M2_PRODUCTS = dict(num_cells_x=40, num_cells_y=40, gaussian_sigma=0.1, floor=1e-6, moment_order=2,
                   quad_order=20, tol=1e-8, use_gaunt=0)
M4_LATTICE = dict(num_cells_x=40, num_cells_y=40, a_x=-3.5, b_x=3.5, a_y=-3.5, b_y=3.5, init_cond="lattice",
                  floor=1e-10, moment_order=4, quad_order=30, tol=1e-8, use_gaunt=1)

CASES = {
    "m6_gaunt_pairs": (M6, None),
    "m6_gaunt_single": (M6, (8, cb.CL_CONTRACT_SINGLE, cb.CL_CONTRACT_PAIRS)),
    "m6_gaunt_4warp": (M6, (4, cb.CL_CONTRACT_PAIRS, cb.CL_CONTRACT_PAIRS)),
    "m2_products": (M2_PRODUCTS, None),
    "m4_lattice": (M4_LATTICE, None),
}


def _grid_run(tmp_path, kw, shape, on, steps):
    deck = str(tmp_path / ("input_%d.deck" % on))
    decks.write_deck(deck, decks.deck_text(**kw, extra={"MOMOPT_GPU_TUNE": "0"}))
    s = cb.Solver(deck, str(tmp_path))
    ctx = s.context()
    if shape is not None:
        ctx.set_launch_shape(*shape)
    ctx.set_range_test(on)
    for _ in range(steps):
        s.update(s.max_dt)
    m, a = ctx.get_state()
    it = s.last_iterations()
    st = s.stats()
    s.close()
    return m, a, it, st


@pytest.mark.parametrize("case", sorted(CASES))
def test_grid_bit_identical_with_and_without(tmp_path, case):
    kw, shape = CASES[case]
    on = _grid_run(tmp_path, kw, shape, 1, 4)
    off = _grid_run(tmp_path, kw, shape, 0, 4)
    assert np.array_equal(on[0], off[0]) and np.array_equal(on[1], off[1])
    assert np.array_equal(on[2], off[2])
    for key in ("total_iter", "total_trials", "hist_reg"):
        assert on[3][key] == off[3][key], key


def _batch(ctx, u, alpha):
    uu, aa = u.copy(), alpha.copy()
    it, reg, st = ctx.solve_batch(uu, aa, check=False)
    return uu, aa, it, reg, st


@pytest.mark.parametrize("order,Q,gaunt", [(6, 40, 1), (3, 30, 0), (4, 30, 1)])
def test_batch_bit_identical_with_and_without(order, Q, gaunt):
    """Cold starts (isotropic), the converged multipliers as starts (every
    vector converges at its first evaluation) and perturbed starts."""
    a = cb.Angular(order, Q, gaunt)
    u, alpha_exact = cb.sample_moment_vectors(a, 4096, seed=31, s_range=(0.1, 20.0))
    ctxs = {}
    for on in (1, 0):
        ctxs[on] = cb.Context.for_batches(a, cb.make_options(tol=1e-8))
        ctxs[on].set_range_test(on)
    cold = {on: _batch(ctxs[on], u, cb.isotropic_alpha(a.n, u.shape[0])) for on in (1, 0)}
    for x, y in zip(cold[1], cold[0]):
        assert np.array_equal(x, y)
    assert np.all(cold[1][4] == 0)
    conv = cold[1][1]
    again = {on: _batch(ctxs[on], u, conv) for on in (1, 0)}
    for x, y in zip(again[1], again[0]):
        assert np.array_equal(x, y)
    warm = conv + 1e-4 * np.random.default_rng(5).standard_normal(conv.shape)
    pert = {on: _batch(ctxs[on], u, warm) for on in (1, 0)}
    for x, y in zip(pert[1], pert[0]):
        assert np.array_equal(x, y)
    for c in ctxs.values():
        c.close()


def test_host_step_bit_identical_with_and_without(tmp_path):
    """The banded host-state step (screening per band, each band with its
    own list of cells left for K1) against the device step with the test
    off."""
    import torch
    kw = dict(num_cells_x=320, num_cells_y=330, gaussian_sigma=0.2, floor=1e-6, moment_order=4,
              quad_order=30, tol=1e-8, use_gaunt=1)
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(**kw, extra={"MOMOPT_GPU_TUNE": "0"}))
    a = cb.Solver(deck, str(tmp_path))
    b = cb.Solver(deck, str(tmp_path))
    ca, cbx = a.context(), b.context()
    cbx.set_range_test(False)
    shape = (ca.NX * ca.NY, ca.n)
    hm = torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    ha = torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    m0, a0 = ca.get_state()
    hm[:] = m0.reshape(shape)
    ha[:] = a0.reshape(shape)
    for _ in range(3):
        ca.step_host(a.max_dt, a.dx, a.dy, hm, ha)
        cbx.step(a.max_dt, a.dx, a.dy)
    mr, ar = cbx.get_state()
    np.testing.assert_array_equal(hm, mr.reshape(shape))
    np.testing.assert_array_equal(ha, ar.reshape(shape))
    sa, sb = ca.stats(), cbx.stats()
    assert sa["num_solves"] == sb["num_solves"] and sa["total_iter"] == sb["total_iter"]
    assert sa["hist_reg"] == sb["hist_reg"]
    a.close()
    b.close()


@pytest.mark.parametrize("case", ["m6_gaunt_pairs", "m4_lattice"])
def test_uniform_flux_tiles_same_result(tmp_path, case):
    """K2+K3 with the uniform-tile shortcut (a tile whose alpha, halo
    included, is one value applies zero flux) against every tile running
    the flux loop: the same states (np.array_equal: up to the sign of zero),
    and the shortcut did skip tiles."""
    kw, _ = CASES[case]
    runs = {}
    for on in (1, 0):
        deck = str(tmp_path / ("flux_%d.deck" % on))
        decks.write_deck(deck, decks.deck_text(**kw, extra={"MOMOPT_GPU_TUNE": "0"}))
        s = cb.Solver(deck, str(tmp_path))
        ctx = s.context()
        ctx.set_uniform_flux_skip(bool(on))
        for _ in range(4):
            s.update(s.max_dt)
        m, a = ctx.get_state()
        runs[on] = (m, a, s.stats()["flux_tiles"])
        tiles = ((kw["num_cells_x"] + 15) // 16) * ((kw["num_cells_y"] + 15) // 16)
        s.close()
    assert np.array_equal(runs[1][0], runs[0][0]) and np.array_equal(runs[1][1], runs[0][1])
    assert runs[0][2] == 8 * tiles            # 4 steps, 2 stages, every tile
    assert runs[1][2] <= runs[0][2]
    if case == "m6_gaunt_pairs":
        assert runs[1][2] < runs[0][2]        # the pulse has not reached the corners
