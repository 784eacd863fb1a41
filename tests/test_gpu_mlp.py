"""The learned warm start: the MLP kernels' loss and gradients against an FP64
numpy restatement of the same network (weights and activations rounded to
BF16 where the kernels round them), training, and Newton from the predicted
start converging to the same moments with fewer iterations."""
import numpy as np
import pytest

import closures_b200 as cb
import pyoracle as oracle_lib

pytestmark = pytest.mark.gpu

SQRT_PI = np.sqrt(np.pi)


def bf16(x):
    """Round-to-nearest-even to bfloat16, returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    from scipy.special import erf
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    from scipy.special import erf
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def reference_loss_grads(W, b, u, alpha, mean, std):
    """FP64 forward/backward of the MSE on standardised targets, with BF16
    rounding of weights, inputs, activations and the backpropagated errors
    at the places the kernels round them (GEMM operands)."""
    xr = u / u[:, :1]
    x = bf16(xr)
    a0 = alpha.copy()
    a0[:, 0] -= np.log(u[:, 0]) * 2.0 * SQRT_PI
    lin = 2.0 * SQRT_PI * xr
    lin[:, 0] = 2.0 * SQRT_PI * np.log(0.5 / SQRT_PI)
    T = (a0 - lin - mean) / std
    Wb = [bf16(w) for w in W]
    acts, zs = [x], []
    h = x
    for l in range(4):
        z = h @ Wb[l] + b[l]
        zs.append(z)
        if l < 3:
            h = bf16(gelu(z))
            acts.append(h)
    Y = zs[-1]
    total = Y.size
    loss = np.mean((Y - T) ** 2)
    dZ = 2.0 * (Y - T) / total
    gW, gb = [None] * 4, [None] * 4
    for l in range(3, -1, -1):
        gW[l] = acts[l].T @ bf16(dZ)
        gb[l] = dZ.sum(axis=0)
        if l > 0:
            dA = bf16(dZ) @ Wb[l].T
            dZ = dA * gelu_grad(zs[l - 1])
    return loss, gW, gb


def test_gradients_match_fp64_reference():
    a = cb.Angular(2, 20, 0)
    u, alpha = cb.sample_moment_vectors(a, 256, seed=4, s_range=(0.1, 3.0))
    m = cb.MLP(a.n, 64, seed=11)
    mean = np.array([-4.5] + [0.0] * (a.n - 1), np.float32)
    std = np.array([1.5] + [2.0] * (a.n - 1), np.float32)
    m.set_output_scaling(mean, std)
    loss, gW, gb = m.loss_and_grads(u, alpha)
    W, b = m.get_params()
    rloss, rW, rb = reference_loss_grads([w.astype(np.float64) for w in W],
                                         [x.astype(np.float64) for x in b], u, alpha,
                                         mean.astype(np.float64), std.astype(np.float64))
    assert abs(loss - rloss) <= 1e-3 * rloss
    for l in range(4):
        assert np.linalg.norm(gW[l] - rW[l]) <= 2e-2 * np.linalg.norm(rW[l]), l
        assert np.linalg.norm(gb[l] - rb[l]) <= 2e-2 * np.linalg.norm(rb[l]), l
    m.close()


def _solve_pairs(order, Q, gaunt, count, seed):
    """(u, alpha*) from the GPU Newton solve of sampled vectors."""
    a = cb.Angular(order, Q, gaunt)
    u, _ = cb.sample_moment_vectors(a, count, seed=seed, s_range=(0.1, 20.0))
    al = cb.isotropic_alpha(a.n, count)
    ctx = cb.Context.for_batches(a, cb.make_options(tol=1e-8))
    it, reg, st = ctx.solve_batch(u, al, check=False)
    ok = (st == 0) & (reg == 0)
    ctx.close()
    return a, u[ok], al[ok], it[ok]


def test_warm_start_reduces_iterations_same_answer():
    import torch

    order, Q, gaunt = 4, 30, 1
    a, u, alpha, it = _solve_pairs(order, Q, gaunt, 200000, seed=31)
    dev = torch.device("cuda", 0)
    du = torch.from_numpy(u).to(dev)
    da = torch.from_numpy(alpha).to(dev)
    lin = 2.0 * SQRT_PI * u
    lin[:, 0] = 2.0 * SQRT_PI * np.log(0.5 / SQRT_PI)
    resid = alpha - lin
    mean = resid.mean(axis=0).astype(np.float32)
    std = (resid.std(axis=0) + 1e-3).astype(np.float32)
    m = cb.MLP(a.n, 256, seed=5)
    m.set_output_scaling(mean, std)
    losses = m.train(du, da, u.shape[0], steps=10000, batch=4096, lr=1e-3)
    print("loss first/last", losses[:50].mean(), losses[-50:].mean())
    assert losses[-50:].mean() < 0.7 * losses[:50].mean()
    # fresh vectors: Newton from isotropic vs from the prediction (isotropic fallback)
    ut, _ = cb.sample_moment_vectors(a, 8000, seed=77, s_range=(0.1, 20.0))
    cnt = ut.shape[0]
    iso = cb.isotropic_alpha(a.n, cnt)
    ctx = cb.Context.for_batches(a, cb.make_options(tol=1e-8))

    def run(start):
        du_ = torch.from_numpy(ut.copy()).to(dev)
        da_ = torch.from_numpy(iso.copy()).to(dev)
        it_ = torch.zeros(cnt, dtype=torch.int32, device=dev)
        rg_ = torch.zeros(cnt, dtype=torch.float64, device=dev)
        st_ = torch.zeros(cnt, dtype=torch.int32, device=dev)
        ctx.solve_batch_device(du_, da_, it_, rg_, st_, count=cnt, d_alpha_start=start)
        torch.cuda.synchronize()
        return (du_.cpu().numpy(), it_.cpu().numpy(), rg_.cpu().numpy(), st_.cpu().numpy())

    u1, it1, reg1, st1 = run(None)
    dstart = torch.empty((cnt, a.n), dtype=torch.float64, device=dev)
    fb = m.predict(torch.from_numpy(ut.copy()).to(dev), dstart, cnt, fallback_kind=2)
    s0 = ctx.stats()["fallbacks"]
    u2, it2, reg2, st2 = run(dstart)
    restarts = ctx.stats()["fallbacks"] - s0
    ok = (st1 == 0) & (st2 == 0)
    print("iterations isotropic start %.3f, predicted start %.3f, non-finite predictions %d, "
          "restarts from the fallback %d" % (it1[ok].mean(), it2[ok].mean(), fb, restarts))
    # the predicted start never adds a regularisation step or an error; where
    # the plain path regularises because a line search or condition test
    # failed on its way, a better start can converge without one
    assert (st1 == st2).all() and (reg2 <= reg1).all()
    print("vectors regularised from the plain start but not from the prediction: %d"
          % int((reg2 < reg1).sum()))
    ok &= reg1 == reg2
    assert it2[ok].mean() < 0.9 * it1[ok].mean(), (it1[ok].mean(), it2[ok].mean())
    # both are solutions to tolerance 1e-8: moments agree well inside 1e-6
    err = np.abs(u2 - u1)[ok] / np.abs(u1[ok, :1])
    assert err.max() < 1e-6
    m.close()
    ctx.close()


def test_grid_warm_start_matches_plain(tmp_path):
    """cl_set_warm_start on a grid: a network trained on the run's own
    (u, alpha*) pairs gives the predicted starts (fallback: the previous
    stage's alpha); the steps reach the same moments as plain steps."""
    import torch
    import decks

    # a deck whose decisions rounding does not move (the grid parity test
    # holds it to 1e-10 against the oracle): both runs must then agree to
    # the solver tolerance, with the same regularisation steps
    kw = dict(num_cells_x=24, num_cells_y=24, gaussian_sigma=0.1, floor=1e-8, moment_order=6,
              quad_order=40, tol=1e-8, use_gaunt=1)
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(**kw))
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    s1 = cb.Solver(deck, str(tmp_path / "a"))
    s2 = cb.Solver(deck, str(tmp_path / "b"))
    for _ in range(3):
        s1.update(s1.max_dt)
        s2.update(s2.max_dt)
    n = s2.n
    dev = torch.device("cuda", 0)
    m, al = s2.context_state()
    du = torch.from_numpy(m.reshape(-1, n).copy()).to(dev)
    da = torch.from_numpy(al.reshape(-1, n).copy()).to(dev)
    cnt = du.shape[0]
    ang = cb.Angular(6, 40, 1)
    bctx = cb.Context.for_batches(ang, cb.make_options(tol=1e-8))
    st = torch.zeros(cnt, dtype=torch.int32, device=dev)
    bctx.solve_batch_device(du, da, None, None, st, count=cnt)
    torch.cuda.synchronize()
    bctx.close()
    assert (st == 0).all()
    u, a = du.cpu().numpy(), da.cpu().numpy()
    tgt = a.copy()
    tgt[:, 0] -= 2.0 * SQRT_PI * np.log(u[:, 0])
    lin = 2.0 * SQRT_PI * u / u[:, :1]
    lin[:, 0] = 2.0 * SQRT_PI * np.log(0.5 / SQRT_PI)
    resid = tgt - lin
    net = cb.MLP(n, 128, seed=3)
    net.set_output_scaling(resid.mean(axis=0).astype(np.float32),
                           (resid.std(axis=0) + 1e-3).astype(np.float32))
    net.train(du, da, cnt, steps=400, batch=512, lr=1e-3, record_loss=False)
    s2.context().set_warm_start(net)
    del net   # the context keeps the network alive
    f0 = s2.stats()["fallbacks"]
    for _ in range(3):
        s1.update(s1.max_dt)
        s2.update(s2.max_dt)
    m1, _ = s1.context_state()
    m2, _ = s2.context_state()
    st1, st2 = s1.stats(), s2.stats()
    print("iterations plain %.3f, learned start %.3f, fallback restarts %d"
          % (st1["iter_mean"], st2["iter_mean"], st2["fallbacks"] - f0))
    assert st1["hist_reg"] == st2["hist_reg"]
    err = float(np.max(np.abs(m2 - m1) / np.abs(m1[:, :, :1])))
    assert err < 1e-6, err
    s2.context().set_warm_start(None)
    s1.close()
    s2.close()
