"""Mixed-precision Hessian (CL_MIXED): the Hessian-only column tiles are
accumulated from split-TF32 products, f, the gradient, the stopping test and
the line search stay FP64.  Solutions therefore still meet the FP64 stopping
test; they are compared with the FP64 path on the same inputs."""
import numpy as np
import pytest

import closures_b200 as cb
import decks

pytestmark = pytest.mark.gpu

CASES = [(2, 20, 0, cb.CL_MN), (3, 30, 1, cb.CL_MN), (4, 30, 0, cb.CL_MN), (6, 40, 1, cb.CL_MN),
         (3, 20, 1, cb.CL_PPN), (5, 40, 1, cb.CL_PPN)]


def _solve(a, u, al, moment_type, precision):
    ctx = cb.Context.for_batches(a, cb.make_options(moment_type=moment_type, tol=1e-8,
                                                    precision=precision))
    uu, aa = u.copy(), al.copy()
    it, reg, st = ctx.solve_batch(uu, aa, check=False)
    ctx.close()
    return uu, aa, it, reg, st


@pytest.mark.parametrize("order,Q,gaunt,mt", CASES)
def test_mixed_matches_fp64(order, Q, gaunt, mt):
    a = cb.Angular(order, Q, gaunt)
    u, _ = cb.sample_moment_vectors(a, 600, seed=21, s_range=(0.1, 3.0))
    al = cb.isotropic_alpha(a.n, u.shape[0], mt, 1e-10)
    u64, a64, it64, reg64, st64 = _solve(a, u, al, mt, cb.CL_FP64)
    u32, a32, it32, reg32, st32 = _solve(a, u, al, mt, cb.CL_MIXED)
    assert (st64 == 0).all() and (st32 == 0).all()
    ok = (reg64 == 0) & (reg32 == 0)
    assert ok.mean() > 0.98
    # both meet ||g|| <= 1e-8 ||u/u0||: the returned moments agree to about that
    unorm = np.linalg.norm(u64[ok] / u64[ok, :1], axis=1)
    err = np.max(np.abs(u32[ok] - u64[ok]) / np.abs(u64[ok, :1]) / unorm[:, None])
    assert err <= 3e-8, err
    # an FP32-accurate Hessian costs at most a few extra Newton iterations
    print("mean iterations fp64 %.3f mixed %.3f" % (it64[ok].mean(), it32[ok].mean()))
    assert it32[ok].mean() <= it64[ok].mean() + 1.0


def test_mixed_grid_steps_match_fp64(tmp_path):
    kw = dict(num_cells_x=24, num_cells_y=24, gaussian_sigma=0.1, floor=1e-8, moment_order=6,
              quad_order=40, tol=1e-8, use_gaunt=1)
    out = {}
    for prec in ("fp64", "mixed"):
        d = tmp_path / prec
        d.mkdir()
        extra = {"MOMOPT_GPU_PRECISION": "mixed"} if prec == "mixed" else None
        deck = str(d / "input.deck")
        decks.write_deck(deck, decks.deck_text(extra=extra, **kw))
        s = cb.Solver(deck, str(d))
        for _ in range(3):
            s.update(s.max_dt)
        out[prec] = (s.context_state()[0], s.stats())
        s.close()
    m64, st64 = out["fp64"]
    m32, st32 = out["mixed"]
    assert st64["hist_reg"] == st32["hist_reg"]
    err = float(np.max(np.abs(m32 - m64) / np.abs(m64[:, :, :1])))
    print("grid mixed vs fp64: %.3e, iterations %.3f vs %.3f" % (err, st32["iter_mean"], st64["iter_mean"]))
    assert err < 1e-6


def test_mixed_rejected_where_not_provided():
    # a launch of several orders runs the runtime-count kernel: FP64 only
    with pytest.raises(cb.ClosuresError):
        cb.MultiSolver([3, 2], 20, 1, cb.make_options(precision=cb.CL_MIXED))
    # order 6 without the Gaunt table has 51 column tiles: general contractions only
    a = cb.Angular(6, 40, 0)
    with pytest.raises(cb.ClosuresError):
        cb.Context.for_batches(a, cb.make_options(precision=cb.CL_MIXED))


def test_mixed_cfg2_lattice_against_fp64_and_oracle(tmp_path):
    """The M4 lattice at 200 x 200, Q = 30 (the deck mixed precision is meant
    for) for three RK2 steps, cell by cell: mixed against the FP64 GPU path and
    against the FP64 oracle, to 1e-6 relative (the accuracy asked of the mixed
    path).  The comparison with the oracle is made on
    the cells whose result rounding does not decide (the two oracle builds and
    the FP64 GPU path agree to 1e-10), which must be nearly all of them."""
    import pyoracle
    kw = dict(decks.WORKLOADS["m4_lattice_200"])
    steps = 3
    out = {}
    for prec in ("fp64", "mixed"):
        d = tmp_path / prec
        d.mkdir()
        extra = {"MOMOPT_GPU_PRECISION": "mixed"} if prec == "mixed" else None
        deck = str(d / "input.deck")
        decks.write_deck(deck, decks.deck_text(extra=extra, **kw))
        s = cb.Solver(deck, str(d))
        for _ in range(steps):
            s.update(s.max_dt)
        out[prec] = s.context_state()[0]
        s.close()
    ref = {}
    for name, fma in (("oracle", False), ("fma", True)):
        g = pyoracle.GridSolver(str(tmp_path / "fp64" / "input.deck"), fma=fma)
        g.steps(steps)
        ref[name] = g.state()[0]
        g.close()
    m64, m32, m_o, m_f = out["fp64"], out["mixed"], ref["oracle"], ref["fma"]
    scale = np.abs(m_o[:, :, :1])
    cell = lambda a, b: np.max(np.abs(a - b) / scale, axis=2)
    e64, e32, env, e3264 = cell(m64, m_o), cell(m32, m_o), cell(m_f, m_o), cell(m32, m64)
    stable = (env <= 1e-10) & (e64 <= 1e-10)
    print("cells %d, decision-stable %d; mixed vs oracle there %.3e, mixed vs fp64 (all) %.3e"
          % (stable.size, stable.sum(), e32[stable].max(), e3264.max()))
    assert stable.mean() >= 0.95
    assert e32[stable].max() <= 1e-6
    assert (e3264 <= 1e-6).mean() >= 0.99
