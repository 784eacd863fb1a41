"""The launch-shape autotuner (cl_tune) and the shapes it chooses between.

K1's two launch shapes (32 cells and 8 warps per CTA, or 16 cells and 4 warps
with two CTAs per SM) evaluate every cell with the same tensor-core MMAs in
the same order, so a grid run is bit-identical in either.  The two tile
layouts (direction pairs or one direction at a time) form the same sums in
another order; each is held to the oracle by the grid criteria.  The tuner
must time every candidate, pick the fastest, apply it, and serve the choice
from its cache to a second context of the same configuration.
"""
import os

import numpy as np
import pytest

import closures_b200 as cb
import decks
import pyoracle as oracle_lib

pytestmark = pytest.mark.gpu

# M6, Q = 40, Gaunt: a 124 x 124 pulse (128^2 cells with ghosts, above the
# tuner's 16384-cell threshold)
DECK = dict(num_cells_x=124, num_cells_y=124, gaussian_sigma=0.05, floor=1e-8, moment_order=6,
            quad_order=40, tol=1e-8, use_gaunt=1)


def _solver(tmp_path, tune):
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(**DECK, extra={"MOMOPT_GPU_TUNE": str(tune)}))
    return deck, cb.Solver(deck, str(tmp_path))


def _run(s, shape, steps=2):
    ctx = s.context()
    ctx.set_launch_shape(*shape)
    for _ in range(steps):
        s.update(s.max_dt)
    return ctx.get_state()


def test_launch_shapes_bit_identical(tmp_path):
    """16 cells / 4 warps per CTA against 32 cells / 8 warps: same bits."""
    _, s8 = _solver(tmp_path, 0)
    m8, a8 = _run(s8, (8, cb.CL_CONTRACT_PAIRS, cb.CL_CONTRACT_PAIRS))
    it8 = s8.last_iterations()
    s8.close()
    _, s4 = _solver(tmp_path, 0)
    m4, a4 = _run(s4, (4, cb.CL_CONTRACT_PAIRS, cb.CL_CONTRACT_PAIRS))
    assert s4.context().tuning()["newton_cells_per_cta"] == 16
    assert np.array_equal(m4, m8) and np.array_equal(a4, a8)
    assert np.array_equal(s4.last_iterations(), it8)
    s4.close()


@pytest.mark.parametrize("shape", [(8, 1, 1), (4, 0, 1), (8, 1, 0)])
def test_tile_layouts_match_oracle(tmp_path, shape):
    """Every tile layout the tuner may pick against the oracle (per cell:
    1e-10 where the two oracle builds agree, the envelope elsewhere)."""
    deck, s = _solver(tmp_path, 0)
    m_g, _ = _run(s, shape)
    s.close()
    orc = oracle_lib.GridSolver(deck)
    fma = oracle_lib.GridSolver(deck, fma=True)
    orc.steps(2)
    fma.steps(2)
    m_o, _ = orc.state()
    m_f, _ = fma.state()
    orc.close()
    fma.close()
    import helpers
    ok, rep = helpers.per_cell_parity(m_g, m_o, m_f)
    assert ok, rep


def test_tuner_picks_fastest_and_caches(tmp_path, monkeypatch):
    cache = tmp_path / "tune_cache.txt"
    monkeypatch.setenv("CL_TUNE_CACHE", str(cache))
    deck, s = _solver(tmp_path, 0)
    ctx = s.context()
    t = ctx.tune()
    k1 = [c for c in t["candidates"] if c["kernel"] == "newton"]
    fl = [c for c in t["candidates"] if c["kernel"] == "flux"]
    # M6 / Gaunt / Mn / FP64: both launch shapes of the pair layout and the
    # single-direction layout for K1, both layouts for the flux
    assert len(k1) == 3 and len(fl) == 2
    assert all(c["ms"] > 0 for c in t["candidates"])
    best = min(k1, key=lambda c: c["ms"])
    assert (t["newton_warps"], t["newton_contraction"]) == (best["warps"], best["contraction"])
    assert t["flux_contraction"] == min(fl, key=lambda c: c["ms"])["contraction"]
    assert ctx.tuning()["newton_warps"] == t["newton_warps"]
    # the tuned shape steps the grid
    s.update(s.max_dt)
    s.close()
    # a second context of the same configuration (tuned in its set-up, the
    # deck's default) takes the choice from the cache
    deck2 = str(tmp_path / "input2.deck")
    decks.write_deck(deck2, decks.deck_text(**DECK))
    s2 = cb.Solver(deck2, str(tmp_path))
    t2 = s2.context().tuning()
    s2.close()
    assert t2["from_cache"]
    assert (t2["newton_warps"], t2["newton_contraction"], t2["flux_contraction"]) == \
        (t["newton_warps"], t["newton_contraction"], t["flux_contraction"])
    assert cache.exists() and "n28_n291_nq1600_gaunt1" in cache.read_text()
