"""Pins the oracle against the reference's own regression goldens.

The reference's harness runs each momopt golden deck and requires a relative
L2 error of the density below 1e-10 (site_scons/testing.py:9, 127-131, 168).
Findings encoded here:
  * gaussian and smooth goldens are reproduced by the current reference
    algorithm (no supplementary gamma test);
  * delta and lattice goldens are reproduced only with the supplementary
    stopping test gamma = modcfl(d) <= 1.1 active -- the test that is
    commented out in the current reference (opt.cpp:99-126, :339, :343;
    momopt_update.cpp:226).  Those two goldens were written by that revision.
"""
import concurrent.futures as cf
import os

import pytest

import decks
import helpers

CASES = [(ic, t) for ic in ["delta", "gaussian", "lattice", "smooth"] for t in ["mn", "ppn"]]
HEAD_CASES = [(ic, t) for (ic, t) in CASES if ic in ("gaussian", "smooth")]


@pytest.fixture(scope="module")
def golden_runs(tmp_path_factory):
    helpers.build_oracle()
    root = tmp_path_factory.mktemp("oracle_golden")
    jobs = {}
    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        for ic, t in CASES:
            d = str(root / ("%s_%s_gamma" % (ic, t)))
            text = decks.regression_deck(ic, t, extra={"MOMOPT_TOL_GAMMA": "1.1"})
            jobs[(ic, t, "gamma")] = ex.submit(helpers.run_oracle, text, d, -1, 2)
        for ic, t in HEAD_CASES:
            d = str(root / ("%s_%s_head" % (ic, t)))
            jobs[(ic, t, "head")] = ex.submit(helpers.run_oracle, decks.regression_deck(ic, t),
                                              d, -1, 2)
        return {k: v.result() for k, v in jobs.items()}


@pytest.mark.parametrize("ic,t", CASES)
def test_oracle_reproduces_golden_with_gamma(golden_runs, ic, t):
    hdr, cur = helpers.read_pn(os.path.join(golden_runs[(ic, t, "gamma")], "out_1.030_0.pn"))
    ghdr, ref = helpers.read_golden(ic, t)
    assert hdr == ghdr
    assert helpers.density_rel_l2(cur, ref) < 1e-10
    assert helpers.moment_rel_inf(cur, ref) < 1e-9


@pytest.mark.parametrize("ic,t", HEAD_CASES)
def test_oracle_reproduces_golden_head(golden_runs, ic, t):
    hdr, cur = helpers.read_pn(os.path.join(golden_runs[(ic, t, "head")], "out_1.030_0.pn"))
    _, ref = helpers.read_golden(ic, t)
    assert helpers.density_rel_l2(cur, ref) < 1e-10
    assert helpers.moment_rel_inf(cur, ref) < 1e-12


def test_initial_output_header(golden_runs):
    hdr, m0 = helpers.read_pn(os.path.join(golden_runs[("gaussian", "mn", "gamma")],
                                           "out_0.000_0.pn"))
    assert (hdr["nx"], hdr["ny"], hdr["n"]) == (36, 74, 10)
    assert (hdr["ax"], hdr["ay"], hdr["bx"], hdr["by"]) == (-1.55, -1.62, 1.45, 1.38)
    assert (m0[:, :, 1:] == 0).all()
