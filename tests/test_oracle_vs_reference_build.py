"""The oracle against the reference itself.

oracle/_ref/closures_ref is the reference's own program compiled from its
sources (oracle/Makefile `ref`: its main.cpp, solvers and opt/ routines, a
GSL shim and the OpenBLAS LAPACK).  Where it was built, every deck here runs
through both to the same end time and the .pn outputs are compared cell by
cell: to 1e-10 relative where the oracle built with and without FMA
contraction agrees (rounding decides nothing there), and within the
oracle builds' own spread elsewhere (the reference's LAPACK is another
rounding again).  The checks skip where the reference could not be built.
"""
import os
import subprocess

import numpy as np
import pytest

import decks
import helpers
import pyoracle

REF_BIN = os.path.join(helpers.REPO, "oracle", "_ref", "closures_ref")

pytestmark = pytest.mark.skipif(not os.path.exists(REF_BIN), reason="reference build (oracle/_ref) absent")

CASES = [
    ("m2_gaussian_nogaunt", dict(num_cells_x=30, num_cells_y=26, gaussian_sigma=0.4, floor=1e-4,
                                 moment_order=2, quad_order=20, tol=1e-8, use_gaunt=0)),
    ("m6_pulse_gaunt", dict(num_cells_x=20, num_cells_y=20, gaussian_sigma=0.1, floor=1e-8,
                            moment_order=6, quad_order=40, tol=1e-8, use_gaunt=1)),
    ("m4_lattice", dict(num_cells_x=28, num_cells_y=28, a_x=-3.5, b_x=3.5, a_y=-3.5, b_y=3.5,
                        init_cond="lattice", floor=1e-10, moment_order=4, quad_order=30, tol=1e-8,
                        use_gaunt=1)),
    ("pp3_periodic", dict(num_cells_x=20, num_cells_y=18, init_cond="smooth", moment_order=3,
                          quad_order=20, tol=1e-8, moment_type="ppn", use_gaunt=0)),
]


def _final_pn(d):
    pns = sorted(f for f in os.listdir(d) if f.endswith(".pn") and not f.startswith("out_0.000"))
    return helpers.read_pn(os.path.join(d, pns[-1]))


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_oracle_matches_reference_program(tmp_path, name, kw):
    kw = dict(kw)
    kw["t_final"] = 2.5 * decks.max_dt(kw)    # two full RK2 steps and a shortened one
    outs = {}
    for who in ("reference", "oracle", "fma"):
        d = tmp_path / who
        d.mkdir()
        deck = str(d / "input.deck")
        decks.write_deck(deck, decks.deck_text(**kw))
        if who == "reference":
            env = dict(os.environ, OMP_NUM_THREADS="1", OPENBLAS_NUM_THREADS="1")
            r = subprocess.run([REF_BIN], cwd=str(d), env=env, capture_output=True, text=True)
            assert r.returncode == 0, r.stdout[-500:]
        else:
            g = pyoracle.GridSolver(deck, fma=(who == "fma"))
            g.run(str(d))
            g.close()
        outs[who] = _final_pn(str(d))
    (h_r, m_r), (h_o, m_o), (_, m_f) = outs["reference"], outs["oracle"], outs["fma"]
    assert h_r == h_o
    ok, rep = helpers.per_cell_parity(m_r, m_o, m_f)
    assert ok, rep
