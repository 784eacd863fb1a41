"""Shared helpers for the tests: paths, .pn files, oracle build and runs."""
import lzma
import math
import os
import struct
import subprocess
import threading

import numpy as np

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(REPO, "oracle")
GOLDEN_DIR = os.path.join(REPO, "tests", "golden")
PKG_DIR = os.path.join(REPO, "closures-2d_b200")

# util/formats.py:168-191 -- "=2q4dq" header then [nx][ny][n] doubles
PN_HEADER = struct.Struct("=2q4dq")



def build_oracle():
    """Builds the oracle (test infrastructure) once per session."""
    import pyoracle
    return pyoracle.build()


def parse_pn(data):
    nx, ny, ax, ay, bx, by, n = PN_HEADER.unpack(data[:PN_HEADER.size])
    m = np.frombuffer(data[PN_HEADER.size:], dtype="<f8").reshape(nx, ny, n)
    return {"nx": nx, "ny": ny, "ax": ax, "ay": ay, "bx": bx, "by": by, "n": n}, m


def read_pn(path):
    with open(path, "rb") as f:
        return parse_pn(f.read())


def read_golden(ic, mtype):
    with lzma.open(os.path.join(GOLDEN_DIR, "momopt", "%s_%s.pn.xz" % (ic, mtype)), "rb") as f:
        return parse_pn(f.read())


def read_moment_golden(ic, filt):
    with lzma.open(os.path.join(GOLDEN_DIR, "moment", "%s_%s.pn.xz" % (ic, filt)), "rb") as f:
        return parse_pn(f.read())


def density(m):
    """util/formats.py:185-189: density grid u0 / (2 sqrt(pi))."""
    return m[:, :, 0] / (2.0 * math.sqrt(math.pi))


def density_rel_l2(cur, ref):
    """The reference harness metric |cur - ref| / |ref| on the density grid
    (site_scons/testing.py:127-131, util/formats.py:36-71 at equal sizes)."""
    a, b = density(cur), density(ref)
    return float(np.sqrt(np.sum((a - b) ** 2)) / np.sqrt(np.sum(b ** 2)))


def moment_rel_inf(cur, ref):
    """max |cur_k - ref_k| / |ref_0| over cells and moments."""
    return float(np.max(np.abs(cur - ref) / np.abs(ref[:, :, :1])))


def run_oracle(deck_text, workdir, max_steps=-1, threads=None):
    exe = build_oracle()
    os.makedirs(workdir, exist_ok=True)
    deck = os.path.join(workdir, "input.deck")
    with open(deck, "w") as f:
        f.write(deck_text)
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    subprocess.run([exe, deck, workdir, str(max_steps)], check=True, env=env,
                   stdout=subprocess.DEVNULL)
    return workdir


def per_cell_parity(m_g, m_o, m_f, tol=1e-10, factor=3.0, newton_tol=1e-8, max_flip_frac=0.01):
    """Grid parity cell by cell, of m_g against the oracle m_o and the oracle
    built with FMA contraction m_f ([NX][NY][n] each; moments scaled by the
    oracle's |u_0| of the cell).  Each cell falls in one class:
      exact     the two oracle builds agree to tol (rounding decides nothing
                in the cell's history) and m_g agrees to tol;
      envelope  the oracle builds differ (an Armijo, condition or stopping
                decision taken on values equal to the last ulp, and the cells
                its flux reached) and m_g is within factor x that spread + tol;
      flip      neither, but within the stopping test's own resolution
                2 newton_tol ||u/u0|| (opt.cpp:286-293): a third rounding
                (another summation order, another LAPACK) ends one more or
                one fewer Newton iteration where the oracle builds agree;
      bad       anything else.
    Passes when no cell is bad and at most max_flip_frac of the cells (and
    at least 5 allowed) are flips.  Returns (passed, report)."""
    scale = np.abs(m_o[:, :, :1])
    err = np.max(np.abs(m_g - m_o) / scale, axis=2)
    env = np.max(np.abs(m_f - m_o) / scale, axis=2)
    unorm = np.linalg.norm(m_o / m_o[:, :, :1], axis=2)
    stable = env <= tol
    exact = stable & (err <= tol)
    envelope = ~stable & (err <= factor * env + tol)
    flip = ~exact & ~envelope & (err <= 2.0 * newton_tol * unorm)
    bad = ~exact & ~envelope & ~flip
    allowed = max(5, int(max_flip_frac * err.size))
    report = {"cells": int(err.size), "exact": int(exact.sum()), "envelope": int(envelope.sum()),
              "flip": int(flip.sum()), "bad": int(bad.sum()), "flip_allowed": allowed,
              "max_err": float(err.max()), "max_env": float(env.max()),
              "max_err_where_stable": float(err[stable].max()) if stable.any() else 0.0,
              "bad_cells": np.argwhere(bad)[:10].tolist()}
    return (not bad.any()) and int(flip.sum()) <= allowed, report


REF_OPT = os.path.join(REPO, "oracle", "_ref", "ref_opt")


def ref_opt_batch(order, Q, use_gaunt, u, alpha, moment_type=0, tol=1e-8, max_iter=100, cond_h_max=1e10,
                  delta_ppn=1e-10, threads=1):
    """The reference's own opt() (oracle/_ref/ref_opt: opt.cpp, fobj.cpp,
    linesearch.cpp and its set-up, compiled from the reference's sources) on
    each row of u/alpha, in place.  Returns iters, regs, status (0, or -2 where
    the regularisation ladder ran out).  Needs the reference build."""
    import tempfile
    import decks
    n = u.shape[1]
    with tempfile.TemporaryDirectory() as d:
        decks.write_deck(os.path.join(d, "input.deck"),
                         decks.deck_text(num_cells_x=2, num_cells_y=2, moment_order=order, quad_order=Q,
                                         use_gaunt=use_gaunt, moment_type=moment_type, tol=tol,
                                         max_iter=max_iter, cond_h_max=cond_h_max, delta_ppn=delta_ppn))
        with open(os.path.join(d, "in.bin"), "wb") as f:
            f.write(np.array([u.shape[0], n], np.int32).tobytes())
            f.write(np.ascontiguousarray(u, np.float64).tobytes())
            f.write(np.ascontiguousarray(alpha, np.float64).tobytes())
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OPENBLAS_NUM_THREADS="1")
        subprocess.run([REF_OPT, "in.bin", "out.bin"], cwd=d, env=env, check=True, stdout=subprocess.DEVNULL)
        raw = open(os.path.join(d, "out.bin"), "rb").read()
    count = u.shape[0]
    off = 0
    u[:] = np.frombuffer(raw, np.float64, count * n, off).reshape(count, n)
    off += 8 * count * n
    alpha[:] = np.frombuffer(raw, np.float64, count * n, off).reshape(count, n)
    off += 8 * count * n
    iters = np.frombuffer(raw, np.int32, count, off).copy()
    off += 4 * count
    regs = np.frombuffer(raw, np.float64, count, off).copy()
    off += 8 * count
    status = np.frombuffer(raw, np.int32, count, off).copy()
    return iters, regs, status
