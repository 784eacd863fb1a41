"""CPU checks of the C ABI library: it loads, exports every declared entry
point, its host-side angular set-up matches the oracle's, and the compute
entry points refuse to run without a GPU (no CPU fallback)."""
import os
import re

import numpy as np
import pytest
import torch

import closures_b200 as cb
import decks
import helpers
import pyoracle as oracle_lib

HEADER = os.path.join(helpers.REPO, "include", "closures_gpu.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = cb.lib()
    names = declared_symbols()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


@pytest.mark.parametrize("order,Q,gaunt", [(1, 8, 0), (2, 20, 0), (2, 20, 1), (3, 30, 1),
                                           (4, 30, 1), (5, 40, 0), (6, 40, 1)])
def test_angular_setup_matches_oracle(order, Q, gaunt):
    a = cb.Angular(order, Q, gaunt)
    o = oracle_lib.setup(order, Q, gaunt)
    assert (a.n, a.n2, a.nq) == (o["n"], o["n2"], o["nq"])
    np.testing.assert_allclose(a.w, o["w"], rtol=1e-13, atol=0)
    assert abs(a.w.sum() - 4 * np.pi) < 1e-12
    np.testing.assert_allclose(a.xi, o["xi"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(a.eta, o["eta"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(a.p, o["p"], rtol=0, atol=1e-13)
    if gaunt:
        assert (a.gaunt_off == o["off"]).all()
        assert (a.gaunt_idx == o["idx"]).all()
        np.testing.assert_allclose(a.gaunt_val, o["val"], rtol=1e-11, atol=1e-13)


def test_basis_orthonormal_and_condon_shortley():
    a = cb.Angular(3, 30, 0)
    G = (a.p * a.w[:, None]).T @ a.p
    # the z-even harmonics are orthonormal over the sphere (hemisphere x2)
    np.testing.assert_allclose(G, np.eye(a.n), atol=1e-13)
    # Y_{1,1} ~ -sqrt(3/4pi) sin(theta) cos(phi) with the Condon-Shortley phase
    q = 0
    mu = np.sqrt(1 - a.xi[q] ** 2 - a.eta[q] ** 2)
    assert a.p[q, 2] * a.xi[q] < 0


def test_sampler_realizable_and_normalised():
    a = cb.Angular(3, 20, 0)
    u, alpha = cb.sample_moment_vectors(a, 64, seed=1)
    assert np.allclose(u[:, 0], 1.0)
    m = np.exp(alpha @ a.p[:, :a.n].T) @ (a.p[:, :a.n] * a.w[:, None])
    np.testing.assert_allclose(m, u, rtol=1e-10, atol=1e-12)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    a = cb.Angular(2, 8, 0)
    with pytest.raises(cb.ClosuresError) as e:
        cb.Context.for_batches(a, cb.make_options())
    assert e.value.code == cb.CL_ERR_CUDA


def test_optimization_types_are_validated(tmp_path):
    """MOMOPT_OPTIMIZATION_TYPE 0-2 pass validation and, without a GPU, stop
    at the device; type 3 and BFGS without sub-iterations
    (MOMOPT_MAX_BFGS_ITER 0, where optbfgs.cpp never steps) are input errors."""
    def solver_error(name, **kw):
        d = tmp_path / name
        decks.write_deck(str(d), decks.deck_text(num_cells_x=4, num_cells_y=4, moment_order=1,
                                                  quad_order=4, **kw))
        with pytest.raises(cb.ClosuresError) as e:
            cb.Solver(str(d), str(tmp_path))
        return e.value
    for t in (1, 2):
        assert solver_error("deck%d" % t, opt_type=t).code == cb.CL_ERR_CUDA
    e = solver_error("deck3", opt_type=3)
    assert e.code == cb.CL_ERR_ARG and "OPTIMIZATION_TYPE" in str(e)
    e = solver_error("deck_bfgs0", opt_type=2, max_bfgs_iter=0)
    assert e.code == cb.CL_ERR_ARG and "MAX_BFGS_ITER" in str(e)


def test_moment_solver_deck_is_validated(tmp_path):
    """SOLVER moment (the linear Pn/FPn solver) passes the deck checks and,
    without a GPU, stops at the device; a missing MOMENT_* key is an input
    error as moment_init.cpp:57-61 makes it."""
    d = tmp_path / "moment.deck"
    decks.write_deck(str(d), decks.moment_deck_text(num_cells_x=4, num_cells_y=4, moment_order=2,
                                                    quad_order=8))
    with pytest.raises(cb.ClosuresError) as e:
        cb.Solver(str(d), str(tmp_path))
    assert e.value.code == cb.CL_ERR_CUDA
    text = "\n".join(l for l in open(d).read().splitlines() if not l.startswith("MOMENT_FILTER_TUNE"))
    decks.write_deck(str(d), text + "\n")
    with pytest.raises(cb.ClosuresError) as e:
        cb.Solver(str(d), str(tmp_path))
    assert e.value.code == cb.CL_ERR_ARG and "MOMENT_" in str(e.value)


def test_missing_deck_key_is_an_input_error(tmp_path):
    text = decks.deck_text(num_cells_x=4, num_cells_y=4, moment_order=1, quad_order=4)
    text = "\n".join(l for l in text.splitlines() if not l.startswith("MOMOPT_MAX_BFGS_ITER"))
    d = tmp_path / "deck"
    decks.write_deck(str(d), text + "\n")
    with pytest.raises(cb.ClosuresError) as e:
        cb.Solver(str(d), str(tmp_path))
    assert e.value.code == cb.CL_ERR_ARG
    assert "MOMOPT_MAX_BFGS_ITER" in str(e.value)


def test_wrong_solver_type(tmp_path):
    d = tmp_path / "deck"
    decks.write_deck(str(d), decks.deck_text(solver="kinetic", num_cells_x=4, num_cells_y=4))
    with pytest.raises(cb.ClosuresError) as e:
        cb.Solver(str(d), str(tmp_path))
    assert "Solver type does not exist" in str(e.value)


def test_error_text_by_code():
    """Each return code has its own message: a timed-out device wait is not
    reported as an exhausted regularisation ladder (both the context and the
    allocation-free entry point take their messages from cl_error_text)."""
    assert cb.error_text(cb.CL_ERR_U0) == "u[0] < 0"
    assert cb.error_text(cb.CL_ERR_MAXREG) == "Max regularization achieved."
    assert cb.error_text(cb.CL_ERR_TIMEOUT) == "device wait timed out"
    assert cb.error_text(-99) == "device error"
    texts = {cb.error_text(c) for c in (cb.CL_OK, cb.CL_ERR_ARG, cb.CL_ERR_CUDA, cb.CL_ERR_U0,
                                        cb.CL_ERR_MAXREG, cb.CL_ERR_TIMEOUT, cb.CL_ERR_STATE)}
    assert len(texts) == 7


def test_noalloc_wrapper_checks_tensors():
    """solve_batch_noalloc refuses tensors the kernel would overrun or
    misread, before anything reaches the library."""
    a = cb.Angular(2, 8, 0)
    o = cb.make_options()
    u64 = torch.zeros((4, a.n), dtype=torch.float64)
    with pytest.raises(ValueError, match="float64"):
        cb.solve_batch_noalloc(a, o, u64.float(), u64, 4)
    with pytest.raises(ValueError, match="CUDA"):
        cb.solve_batch_noalloc(a, o, u64, u64, 4)
    with pytest.raises(ValueError, match="required"):
        cb.solve_batch_noalloc(a, o, None, u64, 4)


BIN = os.path.join(helpers.PKG_DIR, "bin", "closures_gpu")


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_driver_binary_fails_cleanly_without_device(tmp_path):
    """The drop-in executable (host/main.cpp, the reference's main.cpp loop)
    stops with the library's message and abort(), as utils_abort() does, when
    there is no device -- no CPU fallback."""
    import subprocess
    deck = tmp_path / "input.deck"
    decks.write_deck(str(deck), decks.deck_text(num_cells_x=8, num_cells_y=8, moment_order=2, quad_order=8))
    r = subprocess.run([BIN, str(deck), str(tmp_path)], capture_output=True, text=True, cwd=str(tmp_path))
    assert r.returncode != 0
    assert "device" in (r.stdout + r.stderr).lower()
    assert not any(f.endswith(".pn") for f in os.listdir(str(tmp_path)))
