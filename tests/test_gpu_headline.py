"""Parity on the headline deck: M6 (n = 28) on 800 x 800 cells, Q = 40
(1600 directions), Gaunt Hessian, narrow pulse sigma = 0.03 with floor 1e-8,
tolerance 1e-8 -- the deck the bench times (decks.WORKLOADS["m6_800"]).

Two RK2 steps on the GPU through the drop-in solver and in the oracle built
with and without FMA contraction, compared cell by cell (helpers.
per_cell_parity: 1e-10 relative wherever the two oracle builds agree, their
spread elsewhere, a bounded number of stopping-test flips), plus identical
optimisation statistics.  The oracle takes about a minute on the host.
"""
import numpy as np
import pytest

import closures_b200 as cb
import decks
import helpers
import pyoracle

pytestmark = pytest.mark.gpu


def test_headline_deck_two_steps(tmp_path):
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(**decks.WORKLOADS["m6_800"]))
    s = cb.Solver(deck, str(tmp_path))
    for _ in range(2):
        s.update(s.max_dt)
    m_g, _ = s.context_state()
    st_g, it_g = s.stats(), s.last_iterations()
    s.close()
    orc = pyoracle.GridSolver(deck)
    orc.steps(2)
    m_o, _ = orc.state()
    st_o, it_o = orc.stats(), orc.last_iterations()
    orc.close()
    fma = pyoracle.GridSolver(deck, fma=True)
    fma.steps(2)
    m_f, _ = fma.state()
    fma.close()
    ok, rep = helpers.per_cell_parity(m_g, m_o, m_f)
    assert ok, rep
    assert st_g["num_solves"] == st_o["num_solves"] == 4 * 804 * 804
    assert st_g["hist_reg"] == st_o["hist_reg"]
    assert (it_g != it_o).mean() <= 1e-3
    assert abs(st_g["iter_mean"] - st_o["iter_mean"]) <= 1e-3 * st_o["iter_mean"]
