"""The output path writes the same files as the reference, byte for byte: the
data, time, coordinate (_x/_y/_z) and .m/.py metadata files of every output
unit and of the rupture fronts, for a 2D rupture, a 3D rupture with strided
volume snapshots and a curved 2D fault (fixture: tests/golden/output_files.npz,
the reference binary's files for the same inputs).  The unit windows are
gathered on the device and copied asynchronously while the steps go on."""

import os

import numpy as np
import pytest

import helpers
from cases import build_case
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu

FILE_CASES = ["m2_sw", "p3_sw", "m2_curve"]


@pytest.mark.parametrize("name", FILE_CASES)
def test_output_files_identical_to_reference(tmp_path, name):
    gold = {k.split("/", 1)[1]: v for k, v in helpers.load_golden("output_files").items()
            if k.startswith(name + "/")}
    assert gold
    tmp = str(tmp_path)
    prob = build_case(name, tmp)
    infile = prob.write(os.path.join(tmp, prob.name + ".in"))
    with fs.Problem(infile, precision=fs.FP64) as p:
        p.solve()
    written = {fn for fn in os.listdir(tmp) if fn.startswith(prob.name + "_")}
    assert written == set(gold), sorted(written ^ set(gold))
    for fn, ref in gold.items():
        with open(os.path.join(tmp, fn), "rb") as fh:
            got = fh.read()
        assert got == ref.tobytes(), fn
