"""Fixtures at the benchmark workloads' own sizes, from the reference solver.

* ``config1_full.npz``: the 2D mode-II workload at full size -- two blocks of
  401 x 201 nodes (h = 0.1 km), slip weakening, RK3 at CFL 0.3, 1000 steps --
  written by ``fdfault_b200.problems.mode2_rupture`` and run by the unmodified
  reference binary (oracle/_ref/fdfault_ref).  Stored: on-fault slip, slip
  rate and shear stress every 5 steps, and vx / vy at steps 500 and 1000 on
  every second node in x and y.
* ``test2d.npz``: the reference's own example input problems/test2d.in
  (801 x 802 nodes, RK4, slip weakening with barrier boxcars), with its step
  count cut to TEST2D_STEPS and its output list replaced by a smaller one of
  the same kind (fault slip rate and shear stress every step, vx on every
  fourth node at the last step).  The edited input text is stored in the
  fixture, so the tests need no reference checkout.

Needs the reference sources (``oracle.reference_dir()``) to build the binary:

    python tests/golden/make_fullsize.py [config1] [test2d]
"""

import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
from fdfault_b200 import problems as P  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
TEST2D_STEPS = 100


def config1_problem(datadir):
    nx, ny, nt = 401, 201, 1000
    outs = [P.Output("f_" + f, f, 0, nt, 5, (0, ny, 0), (nx - 1, ny, 0), (1, 1, 1)) for f in ("U", "V", "S")]
    outs += [P.Output("vol_" + f, f, nt // 2, nt, nt // 2, (0, 0, 0), (nx - 1, 2 * ny - 1, 0), (2, 2, 1))
             for f in ("vx", "vy")]
    return P.mode2_rupture(nx=nx, ny=ny, h=0.1, nt=nt, name="config1", datadir=datadir, outputs=outs)


def test2d_text(datadir):
    """problems/test2d.in with nt = TEST2D_STEPS, the given data directory and
    a reduced output list."""
    src = open(os.path.join(oracle.reference_dir(), "problems", "test2d.in")).read().split("\n")
    i = src.index("[fdfault.problem]")
    src[i + 2] = datadir
    src[i + 3] = str(TEST2D_STEPS)
    o = src.index("[fdfault.outputlist]")
    e = src.index("[fdfault.frontlist]")
    nt = TEST2D_STEPS
    units = ["V", "V", "0 %d 1" % nt, "0 800 1", "401 401 1", "0 0 1",
             "S", "S", "0 %d 1" % nt, "0 800 1", "401 401 1", "0 0 1",
             "vx", "vx", "%d %d 1" % (nt, nt), "0 800 4", "0 801 4", "0 0 1",
             "", ""]
    return "\n".join(src[:o + 1] + units + src[e:])


def read_units(datadir, name, units):
    out = {}
    for unit, field in units:
        u = oracle.read_unit(datadir, name, unit, field)
        out["unit/" + unit] = u["data"]
        if "t" in u:
            out["t/" + unit] = u["t"]
    return out


def make_config1():
    tmp = tempfile.mkdtemp(prefix="golden_c1_")
    prob = config1_problem(tmp + "/")
    infile = prob.write(os.path.join(tmp, "config1.in"))
    t0 = time.time()
    r = oracle.run_reference(infile, tmp, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    arrays = read_units(tmp, "config1", [(o.name, o.field) for o in prob.outputs])
    np.savez_compressed(os.path.join(HERE, "config1_full.npz"), **arrays)
    print("config1", time.time() - t0, "s", sum(a.size for a in arrays.values()), "values")


def make_test2d():
    tmp = tempfile.mkdtemp(prefix="golden_t2d_")
    text = test2d_text(tmp + "/")
    infile = os.path.join(tmp, "test2d.in")
    with open(infile, "w") as fh:
        fh.write(text)
    t0 = time.time()
    r = oracle.run_reference(infile, tmp, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError(r.stderr)
    arrays = read_units(tmp, "test2d", [("V", "V"), ("S", "S"), ("vx", "vx")])
    arrays["input"] = np.array(test2d_text("@DATADIR@"))
    np.savez_compressed(os.path.join(HERE, "test2d.npz"), **arrays)
    print("test2d", time.time() - t0, "s", sum(a.size for a in arrays.values()), "values")


if __name__ == "__main__":
    if not os.path.exists(oracle.REF_BIN):
        oracle.build()
    todo = sys.argv[1:] or ["config1", "test2d"]
    if "config1" in todo:
        make_config1()
    if "test2d" in todo:
        make_test2d()
