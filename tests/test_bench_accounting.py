"""The bench's accounting of the exact shortcuts (host side, no device).

The roofline credits K1 only with the work it did: full Newton iterations,
line-search trials and the screening pass's evaluations, never the
iterations of solves the screening pass settled (a copied start did no work
at all).  K2+K3 is credited only for the tiles that ran the flux loop.  The
fraction of uniform tiles reported beside it is computed from the state on
the host, with the kernel's rule: one alpha, bit for bit, over the tile and
its 2-cell halo.
"""
import os
import sys

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402


def _stats(total_iter, trials, screened, evals):
    return {"total_iter": total_iter, "total_trials": trials, "screened": screened, "screen_evals": evals}


def test_newton_flops_credits_work_done():
    n, nq, per_iter = 28, 1600, 4.0e5
    s0 = _stats(0, 0, 0, 0)
    # 1000 solves: 900 settled by screening (100 of them evaluated, 800
    # copies), 100 solved by K1 in 300 iterations with 50 trials
    s1 = _stats(900 + 300, 50, 900, 100 + 100)
    f = bench.newton_flops(s0, s1, per_iter, n, nq)
    expect = 300 * per_iter + 50 * bench.flops_per_trial(n, nq) + 200 * bench.flops_per_screen(n, nq)
    assert f == expect
    # without screening the count is the plain one
    s2 = _stats(1200, 50, 0, 0)
    assert bench.newton_flops(s0, s2, per_iter, n, nq) == 1200 * per_iter + 50 * bench.flops_per_trial(n, nq)


def test_uniform_tile_fraction_rule():
    NX = NY = 4 + 64    # 4 x 4 tiles of 16 x 16 interior cells
    alpha = np.zeros((NX, NY, 6))
    alpha[..., 0] = -3.0
    assert bench.uniform_tile_fraction(alpha) == 1.0
    # the centre of tile (1, 1): that tile only
    alpha[2 + 16 + 8, 2 + 16 + 8, 3] = 1e-300
    assert bench.uniform_tile_fraction(alpha) == 15 / 16
    # the last column of tile (1, 1): also in the halo of tile (1, 2)
    alpha[2 + 16 + 8, 2 + 16 + 15, 3] = 1e-300
    assert bench.uniform_tile_fraction(alpha) == 14 / 16
    # a corner of tile (1, 1): in the halo squares of (0, 0), (0, 1), (1, 0)
    alpha[2 + 16, 2 + 16, 3] = 1e-300
    assert bench.uniform_tile_fraction(alpha) == 11 / 16
    # the sign of zero counts as a different value, as in the kernel's
    # bitwise comparison
    alpha2 = np.zeros((NX, NY, 6))
    alpha2[2 + 40, 2 + 40, 5] = -0.0
    assert bench.uniform_tile_fraction(alpha2) == 15 / 16
