"""input.deck writers for the tests and the bench.

The deck format is the reference's flat key/value file
(input_deck_reader.cpp:17-78).  The regression deck reproduces the values the
reference's harness writes for its momopt goldens (site_scons/testing.py:143-146
and util/decks.py:26-56, 58-104): 36x74 cells on [-1.55,1.45]x[-1.62,1.38],
t_final 1.03, sigma 1.111, Gaussian sigma 1.7 (0 for "delta"), floor 1e-4,
order 3, Q 30, tol 1e-4, cond 1e10, max_iter 100, Gaunt 1, theta 2.
"""

INIT_CONDS = {"delta": 0, "gaussian": 0, "lattice": 1, "smooth": 2}
MOMENT_TYPES = {"mn": 0, "ppn": 1}


def deck_text(solver="momopt", num_cells_x=50, num_cells_y=50, a_x=-1.5, b_x=1.5,
              a_y=-1.5, b_y=1.5, t_final=1.0, out_delta_t=1000.1, gaussian_sigma=0.4,
              floor=1e-4, init_cond="gaussian", sigma=1.0, moment_order=3, quad_order=30,
              cfl_factor=0.9, tol=1e-4, cond_h_max=1e10, cond_h_max_bfgs=20, max_iter=100,
              max_bfgs_iter=5, use_gaunt=1, theta=2.0, delta_ppn=1e-10, moment_type="mn",
              opt_type=0, partitions=(1, 1), extra=None):
    ic = INIT_CONDS[init_cond] if isinstance(init_cond, str) else int(init_cond)
    mt = MOMENT_TYPES[moment_type] if isinstance(moment_type, str) else int(moment_type)
    lines = [
        "SOLVER %s" % solver,
        "NUM_CELLS_X %d" % num_cells_x,
        "NUM_CELLS_Y %d" % num_cells_y,
        "NUM_MPI_PARTITIONS_X %d" % partitions[0],
        "NUM_MPI_PARTITIONS_Y %d" % partitions[1],
        "A_X %.17f" % a_x,
        "B_X %.17f" % b_x,
        "A_Y %.17f" % a_y,
        "B_Y %.17f" % b_y,
        "T_FINAL %.17f" % t_final,
        "OUT_DELTA_T %.17f" % out_delta_t,
        "GAUSSIAN_SIGMA %.17f" % gaussian_sigma,
        "FLOOR %.17f" % floor,
        "INIT_COND %d" % ic,
        "SIGMA %.17f" % sigma,
        "MOMOPT_MOMENT_ORDER %d" % moment_order,
        "MOMOPT_QUAD_ORDER %d" % quad_order,
        "MOMOPT_CFL_FACTOR %.17f" % cfl_factor,
        "MOMOPT_TOL %.17f" % tol,
        "MOMOPT_COND_H_MAX %.17f" % cond_h_max,
        "MOMOPT_COND_H_MAX_BFGS %d" % cond_h_max_bfgs,
        "MOMOPT_MAX_ITER %d" % max_iter,
        "MOMOPT_MAX_BFGS_ITER %d" % max_bfgs_iter,
        "MOMOPT_USE_GAUNT %d" % use_gaunt,
        "MOMOPT_THETA %.17f" % theta,
        "MOMOPT_DELTA_PPN %.17f" % delta_ppn,
        "MOMOPT_MOMENT_TYPE %d" % mt,
        "MOMOPT_OPTIMIZATION_TYPE %d" % opt_type,
    ]
    for k, v in (extra or {}).items():
        lines.append("%s %s" % (k, v))
    return "\n".join(lines) + "\n"


FILTER_TYPES = {"none": 0, "hauck": 1, "sspline": 2, "lanczos": 3}


def moment_deck_text(moment_order=3, quad_order=30, filter_type="none", filter_tune=100,
                     cfl_factor=0.9, **grid):
    """A deck for SOLVER moment (the linear Pn/FPn solver): the grid keys of
    deck_text and the MOMENT_* keys of moment_init.cpp:57-61 (util/decks.py
    writes the same five)."""
    ft = FILTER_TYPES[filter_type] if isinstance(filter_type, str) else int(filter_type)
    base = deck_text(solver="moment", **grid)
    lines = [l for l in base.splitlines() if not l.startswith("MOMOPT_")]
    lines += [
        "MOMENT_MOMENT_ORDER %d" % moment_order,
        "MOMENT_QUAD_ORDER %d" % quad_order,
        "MOMENT_FILTER_TYPE %d" % ft,
        "MOMENT_FILTER_TUNE %d" % filter_tune,
        "MOMENT_CFL_FACTOR %.17f" % cfl_factor,
    ]
    return "\n".join(lines) + "\n"


def regression_moment_deck(init_cond, filter_type, **kw):
    """The deck the reference's regression harness runs for one moment-solver
    golden (site_scons/testing.py:109-160, 252-276)."""
    args = dict(num_cells_x=36, num_cells_y=74, a_x=-1.55, b_x=1.45, a_y=-1.62, b_y=1.38,
                t_final=1.03, sigma=1.111, init_cond=init_cond,
                gaussian_sigma=0.0 if init_cond == "delta" else 1.7, filter_type=filter_type)
    args.update(kw)
    return moment_deck_text(**args)


def regression_deck(init_cond, moment_type, **kw):
    """The deck the reference's regression harness runs for one momopt golden."""
    args = dict(num_cells_x=36, num_cells_y=74, a_x=-1.55, b_x=1.45, a_y=-1.62, b_y=1.38,
                t_final=1.03, sigma=1.111, init_cond=init_cond,
                gaussian_sigma=0.0 if init_cond == "delta" else 1.7,
                moment_type=moment_type)
    args.update(kw)
    return deck_text(**args)


def write_deck(path, text):
    with open(path, "w") as f:
        f.write(text)


def max_dt(kw):
    """The time step a deck written by deck_text(**kw) runs at:
    CFL * (2 / (2 + theta)) * dx dy / (dx + dy) (momopt_init.cpp:72)."""
    nx, ny = kw.get("num_cells_x", 50), kw.get("num_cells_y", 50)
    dx = (kw.get("b_x", 1.5) - kw.get("a_x", -1.5)) / nx
    dy = (kw.get("b_y", 1.5) - kw.get("a_y", -1.5)) / ny
    cfl, theta = kw.get("cfl_factor", 0.9), kw.get("theta", 2.0)
    return cfl * (2.0 / (2.0 + theta)) * dx * dy / (dx + dy)


# The benchmark workloads (deck_text keyword sets).
WORKLOADS = {
    # the M6 / PP6 800x800 pulse (configs of the headline)
    "m6_800": dict(num_cells_x=800, num_cells_y=800, a_x=-1.5, b_x=1.5, a_y=-1.5, b_y=1.5,
                   gaussian_sigma=0.03, floor=1e-8, sigma=1.0, init_cond="gaussian",
                   moment_order=6, quad_order=40, tol=1e-8, use_gaunt=1, t_final=1.0,
                   moment_type="mn"),
    "pp6_800": dict(num_cells_x=800, num_cells_y=800, a_x=-1.5, b_x=1.5, a_y=-1.5, b_y=1.5,
                    gaussian_sigma=0.03, floor=1e-8, sigma=1.0, init_cond="gaussian",
                    moment_order=6, quad_order=40, tol=1e-8, use_gaunt=1, t_final=1.0,
                    moment_type="ppn"),
    # M4 lattice, 200x200 on [-3.5,3.5]^2, Q=30
    "m4_lattice_200": dict(num_cells_x=200, num_cells_y=200, a_x=-3.5, b_x=3.5, a_y=-3.5,
                           b_y=3.5, init_cond="lattice", floor=1e-10, moment_order=4,
                           quad_order=30, tol=1e-8, use_gaunt=1, t_final=3.2),
    # M2 50x50 Gaussian, Q=20 (the reference's CPU-runnable case)
    "m2_50": dict(num_cells_x=50, num_cells_y=50, gaussian_sigma=0.4, floor=1e-4,
                  moment_order=2, quad_order=20, tol=1e-8, use_gaunt=0, t_final=0.5),
}
