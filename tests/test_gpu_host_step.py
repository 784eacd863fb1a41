"""The host-state step (cl_step_host): one RK2 step on host arrays with the
copies overlapped with the kernels must equal, bit for bit, the state
uploaded with cl_set_state, stepped with cl_step and read back with
cl_get_state -- for banded uploads and a split second-stage flux (grids of
at least two waves of flux tiles), for a grid too small to split, and for
the periodic deck whose ghost copy needs the whole grid up first."""
import numpy as np
import pytest
import torch

import closures_b200 as cb
import decks

pytestmark = pytest.mark.gpu

CASES = [
    ("m2_gaussian_320", dict(num_cells_x=320, num_cells_y=330, gaussian_sigma=0.2, floor=1e-4,
                             moment_order=2, quad_order=12, tol=1e-8, use_gaunt=0)),
    ("m3_gaussian_40", dict(num_cells_x=40, num_cells_y=36, gaussian_sigma=0.4, moment_order=3,
                            quad_order=30, tol=1e-8, use_gaunt=1)),
    ("m2_periodic_48", dict(num_cells_x=48, num_cells_y=40, init_cond="smooth", moment_order=2,
                            quad_order=12, a_x=0.0, b_x=1.0, a_y=0.0, b_y=1.0, tol=1e-8)),
    ("pp2_gaussian_320_cb", dict(num_cells_x=320, num_cells_y=320, gaussian_sigma=0.3, floor=1e-4,
                                 moment_order=2, quad_order=12, tol=1e-8, use_gaunt=0, moment_type="ppn",
                                 opt_type=1)),
]


@pytest.mark.parametrize("name,kw", CASES, ids=[c[0] for c in CASES])
def test_step_host_equals_device_step(tmp_path, name, kw):
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(**kw))
    a = cb.Solver(deck, str(tmp_path))
    b = cb.Solver(deck, str(tmp_path))
    ca, cbx = a.context(), b.context()
    shape = (ca.NX * ca.NY, ca.n)
    hm = torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    ha = torch.empty(shape, dtype=torch.float64).pin_memory().numpy()
    m0, a0 = ca.get_state()
    hm[:] = m0.reshape(shape)
    ha[:] = a0.reshape(shape)
    for step in range(3):
        cbx.set_state(hm, ha)
        cbx.step(a.max_dt, a.dx, a.dy)
        mr, ar = cbx.get_state()
        ca.step_host(a.max_dt, a.dx, a.dy, hm, ha)
        np.testing.assert_array_equal(hm, mr.reshape(shape), err_msg="moments, step %d" % step)
        np.testing.assert_array_equal(ha, ar.reshape(shape), err_msg="alpha, step %d" % step)
    sa, sb = ca.stats(), cbx.stats()
    assert sa["num_solves"] == sb["num_solves"] and sa["total_iter"] == sb["total_iter"]
    a.close()
    b.close()


def test_step_host_pageable_buffers(tmp_path):
    """Ordinary (pageable) numpy arrays: copies without overlap, same result."""
    deck = str(tmp_path / "input.deck")
    decks.write_deck(deck, decks.deck_text(num_cells_x=30, num_cells_y=28, gaussian_sigma=0.4,
                                           moment_order=2, quad_order=12, tol=1e-8))
    a = cb.Solver(deck, str(tmp_path))
    b = cb.Solver(deck, str(tmp_path))
    ca, cbx = a.context(), b.context()
    m, al = ca.get_state()
    hm = np.ascontiguousarray(m.reshape(-1, ca.n))
    ha = np.ascontiguousarray(al.reshape(-1, ca.n))
    ca.step_host(a.max_dt, a.dx, a.dy, hm, ha)
    cbx.step(a.max_dt, a.dx, a.dy)
    mr, ar = cbx.get_state()
    np.testing.assert_array_equal(hm, mr.reshape(hm.shape))
    np.testing.assert_array_equal(ha, ar.reshape(ha.shape))
    with pytest.raises(ValueError):
        ca.step_host(a.max_dt, a.dx, a.dy, hm[:-1], ha)
    a.close()
    b.close()
