"""Copies the reference's regression goldens into tests/golden/: the eight
momopt files and the sixteen of the linear moment solver.

The reference's regression harness (site_scons/testing.py:109-303) compares
out_1.030_0.pn against tests/regression/momopt/<ic>/<type>.pn.  Those files
are data (36x74x10 doubles after a 56-byte "=2q4dq" header,
util/formats.py:168-191); they are stored here xz-compressed so the tests run
where the reference tree is absent.  Run once, in a tree that has the reference:

    python tests/golden/make_golden.py /path/to/closures-2d
"""
import lzma
import os
import sys

ICS = ["delta", "gaussian", "lattice", "smooth"]
TYPES = ["mn", "ppn"]
FILTERS = ["none", "hauck", "sspline", "lanczos"]   # site_scons/testing.py:19


def main(ref_root):
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "momopt")
    os.makedirs(here, exist_ok=True)
    for ic in ICS:
        for t in TYPES:
            src = os.path.join(ref_root, "tests", "regression", "momopt", ic, t + ".pn")
            with open(src, "rb") as f:
                data = f.read()
            dst = os.path.join(here, "%s_%s.pn.xz" % (ic, t))
            with lzma.open(dst, "wb", preset=9 | lzma.PRESET_EXTREME) as f:
                f.write(data)
            print(dst, len(data))
    # the moment solver's goldens: tests/regression/moment/<ic>/<filter>.pn
    # (site_scons/testing.py:252-276, same grid and time as momopt)
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "moment")
    os.makedirs(here, exist_ok=True)
    for ic in ICS:
        for f in FILTERS:
            src = os.path.join(ref_root, "tests", "regression", "moment", ic, f + ".pn")
            with open(src, "rb") as fh:
                data = fh.read()
            dst = os.path.join(here, "%s_%s.pn.xz" % (ic, f))
            with lzma.open(dst, "wb", preset=9 | lzma.PRESET_EXTREME) as fh:
                fh.write(data)
            print(dst, len(data))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the closures-2d checkout>")
    main(sys.argv[1])
