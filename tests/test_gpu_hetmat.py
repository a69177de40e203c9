"""Heterogeneous material and the plastic return-map rule on the GPU.

* A material file (fields.cpp:582-711) is honoured by every part of the
  stage: bit-identity with the reference for the hetmat cases is in
  test_gpu_parity.py; here, a file holding the blocks' own uniform values
  reproduces the homogeneous run (to rounding: the reference forms the
  per-direction coefficients directly from the node's values instead of by
  the homogeneous path's chained rescaling).
* The FP32 marching kernels hold one material per block, so a heterogeneous
  problem runs the reference-order kernel whatever kind is asked for.
* The reference's return map (block.cpp:442-589) takes its bulk modulus
  truncated to an integer and, in 3D, only the nodes its z loop reaches; rule 1
  applies it at every node with the exact modulus.  Where the reference's loop
  would not terminate, stepping under rule 0 fails and rule 1 runs.
"""

import os

import numpy as np
import pytest

import cases
from fdfault_b200 import problems as P
from fdfault_b200 import solver as fs

pytestmark = pytest.mark.gpu


def write(prob, tmp):
    prob.datadir = tmp.rstrip("/") + "/"
    return prob.write(os.path.join(tmp, prob.name + ".in"))


def fields(p):
    return np.array([p.field(c) for c in range(p.nfields + p.nfieldsp)])


# (not mode II plastic: with a material file the reference's sigma_zz rate
# takes its second modulus from the next x row's density, block.cpp:1289-1291)
@pytest.mark.parametrize("name", ["m2_sw", "p3_sw", "p3_plastic_yield"])
def test_uniform_material_file_matches_homogeneous(tmp_path, name):
    tmp = str(tmp_path)
    prob = cases.build_case(name, tmp, outputs=False)
    home = write(prob, tmp)
    nx, ny, nz = prob.nx
    b = next(iter(prob.blocks.values()))
    prob.name = name + "_matfile"
    P.write_material(os.path.join(tmp, "uniform.mat"), *[np.full((nx, ny, nz), v) for v in (b.rho, b.lam, b.g)])
    prob.matfile = os.path.join(tmp, "uniform.mat")
    het = write(prob, tmp)
    out = []
    for f in (home, het):
        with fs.Problem(f, precision=fs.FP64) as p:
            p.step(10)
            out.append((fields(p), p.fault(0, fs.V).copy(), p.dt))
    assert out[0][2] == out[1][2]   # same time step from the per-node wave speeds
    scale = np.abs(out[0][0]).max()
    err = np.abs(out[0][0] - out[1][0]).max() / scale
    print(name, "uniform material file vs homogeneous: max relative difference %.3g" % err)
    assert err <= 1e-11
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-11 * np.abs(out[0][1]).max()


@pytest.mark.parametrize("name,kind", [("p3_hetmat", 3), ("p3_hetmat", 1), ("m2_hetmat", 1)])
def test_hetmat_runs_reference_order_kernel(tmp_path, name, kind):
    prob = cases.build_case(name, str(tmp_path), outputs=False)
    with fs.Problem(write(prob, str(tmp_path)), precision=fs.FP32) as p:
        assert p.set_volume_kernel(kind) == 0
        p.step(4)
        p.synchronize()
        assert np.all(np.isfinite(fields(p)))


def _deep_plastic(tmp, nz):
    return cases._yielding(cases._p3("p3_deep_%d" % nz, tmp, nt=10, nz=nz), 0.5, True)


def test_plastic_rule_where_reference_loop_does_not_end(tmp_path):
    """nz = 61 > trunc(lambda + 2/3 G) + 1 = 54: the reference's z loop would
    revisit node 54 for ever.  Rule 0 refuses to step; rule 1 steps."""
    prob = _deep_plastic(str(tmp_path), 61)
    with fs.Problem(write(prob, str(tmp_path)), precision=fs.FP64) as p:
        with pytest.raises(fs.FdfaultError, match="does not terminate"):
            p.step(1)
        p.set_plastic_rule(fs.Problem.PLASTIC_EVERY_NODE)
        p.step(3)
        p.synchronize()
        gp = p.field(p.nfields + 1).reshape(prob.nx)
    assert np.all(np.isfinite(gp))
    # yielding below the first z plane: only the every-node rule reaches it
    assert np.abs(gp[:, :, 1:]).max() > 0.


def test_plastic_rules_differ_as_described(tmp_path):
    """Rule 0 yields only on each block's first z plane (trunc(K) + 1 = 54 is
    past nz = 15); rule 1 everywhere the stress exceeds the limit."""
    prob = cases.build_case("p3_plastic_yield", str(tmp_path), outputs=False)
    infile = write(prob, str(tmp_path))
    gp = {}
    for rule in (0, 1):
        with fs.Problem(infile, precision=fs.FP64) as p:
            p.set_plastic_rule(rule)
            p.step(6)
            gp[rule] = p.field(p.nfields + 1).reshape(prob.nx)
    assert np.abs(gp[0][:, :, 1:]).max() == 0.
    assert np.abs(gp[0][:, :, 0]).max() > 0.
    assert np.abs(gp[1][:, :, 1:]).max() > 0.


def test_plastic_rule_change_drops_captured_graphs(tmp_path):
    """Graph replay after a rule change follows the new rule (the captured
    launches carry the block table by value)."""
    prob = cases.build_case("m2_plastic_yield", str(tmp_path), outputs=False)
    infile = write(prob, str(tmp_path))
    res = {}
    for graphs in (False, True):
        with fs.Problem(infile, precision=fs.FP64) as p:
            p.use_graphs(graphs)
            p.step(4)
            p.set_plastic_rule(fs.Problem.PLASTIC_EVERY_NODE)
            p.step(4)
            res[graphs] = fields(p)
    assert np.array_equal(res[False], res[True])
