"""The CPU oracle (C restatement) reproduces the reference solver bit for bit.

The golden fixtures were written by the unmodified reference solver
(tests/golden/make_golden.py); here the oracle runs the same problems and
every output unit value and rupture time must be identical."""

import os

import numpy as np
import pytest

import cases
import helpers
import oracle

FMAP = {"v": oracle.V, "u": oracle.U, "s": oracle.SS, "sn": oracle.SN, "state": oracle.STATE,
        "vx": oracle.VX, "ux": oracle.UX, "sx": oracle.SX}


def run_oracle_outputs(prob, infile):
    o = oracle.Oracle(infile)
    out = {}
    fault_units = [u for u in prob.outputs if not u.name.startswith("vol_")]
    vol_units = [u for u in prob.outputs if u.name.startswith("vol_")]
    series = {u.name: [] for u in fault_units}
    for step in range(o.nt + 1):
        if step:
            o.step()
        for u in fault_units:
            series[u.name].append(helpers.fault_sel(prob, u, u.field, lambda n, k: o.fault(n, FMAP[k]).copy()))
        for u in vol_units:
            if step == o.nt:
                c = helpers.vol_comp(prob, u.field)
                a = o.abs_field(c) if c < o.nfields else o.field(oracle.F)[c].copy()
                out["unit/" + u.name] = a.reshape(prob.nx)[helpers.unit_slice(prob, u)]
    for k, v in series.items():
        out["unit/" + k] = np.array(v)
    for n, itf in enumerate(prob.interfaces):
        if itf.kind != "locked" and prob.front is not None:
            out["front/%d" % n] = o.fault(n, oracle.TFRONT).copy()
    o.close()
    return out


@pytest.mark.parametrize("name", sorted(cases.CASES))
def test_oracle_matches_reference(name, tmp_path):
    prob = cases.build_case(name, str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    got = run_oracle_outputs(prob, infile)
    gold = helpers.load_golden(name)
    for key, ref in gold.items():
        if key.startswith("t/"):
            continue
        a = got[key].reshape(-1)
        b = ref.reshape(-1)
        assert a.shape == b.shape, key
        assert np.array_equal(a, b), "%s: max diff %g" % (key, np.max(np.abs(a - b)))


@pytest.mark.skipif(not os.path.exists(oracle.REF_BIN), reason="reference binary not built")
def test_reference_binary_reproduces_golden(tmp_path):
    """The fixtures are current: the live reference binary still writes them."""
    name = "m2_sw"
    prob = cases.build_case(name, str(tmp_path))
    infile = prob.write(os.path.join(str(tmp_path), prob.name + ".in"))
    oracle.run_reference(infile, str(tmp_path))
    gold = helpers.load_golden(name)
    for o in prob.outputs:
        u = oracle.read_unit(str(tmp_path), prob.name, o.name, o.field)
        assert np.array_equal(u["data"], gold["unit/" + o.name])
