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
