"""The reference's return-map loop and heterogeneous material files, on the CPU.

block::calc_plastic (src/block.cpp:442-589) declares `double k` and then an
`int k` z-loop index; the bulk modulus it assigns lands in the loop index.
The oracle follows that control flow (pinned by the yielding golden cases,
which the reference solver wrote); these tests check its consequences
directly: in 3D only each block column's first z node yields when
trunc(K) + 1 is past the block, and the loop never ends when it is not.
"""

import os

import numpy as np
import pytest

import cases
import oracle
from fdfault_b200 import problems as P


def _write(prob, tmp):
    prob.datadir = tmp.rstrip("/") + "/"
    return prob.write(os.path.join(tmp, prob.name + ".in"))


def test_reference_loop_yields_only_first_z_plane(tmp_path):
    prob = cases.build_case("p3_plastic_yield", str(tmp_path), outputs=False)
    o = oracle.Oracle(_write(prob, str(tmp_path)))
    o.run(6)
    gp = o.field(oracle.F)[o.nfields + 1].reshape(prob.nx).copy()
    o.close()
    assert np.abs(gp[:, :, 0]).max() > 0.
    assert np.abs(gp[:, :, 1:]).max() == 0.


def test_reference_loop_does_not_terminate_on_deep_blocks(tmp_path):
    # trunc(lambda + 2/3 G) + 1 = 54 < nz = 61: the loop revisits z node 54
    prob = cases._yielding(cases._p3("p3_deep", str(tmp_path), nt=4, nz=61), 0.5, True)
    o = oracle.Oracle(_write(prob, str(tmp_path)))
    with pytest.raises(RuntimeError, match="does not terminate"):
        o.step()
    o.close()


def test_oracle_rejects_mode3_material_file(tmp_path):
    prob = cases.build_case("m3", str(tmp_path), outputs=False)
    prob.matfile = os.path.join(str(tmp_path), "m3.mat")
    P.layered_material(prob, prob.matfile, seed=1)
    with pytest.raises(RuntimeError, match="mode III"):
        oracle.Oracle(_write(prob, str(tmp_path)))


def test_material_writer(tmp_path):
    prob = cases.build_case("p3_sw", str(tmp_path), outputs=False)
    path = P.layered_material(prob, os.path.join(str(tmp_path), "m.mat"), seed=3)
    m = np.fromfile(path, dtype="<f8").reshape(3, *prob.nx)
    assert prob.matfile == path
    assert np.all(m > 0.)
    b = next(iter(prob.blocks.values()))
    # contrast across y: the top rows are stiffer and denser than the bottom ones
    for c, base in enumerate((b.rho, b.lam, b.g)):
        assert m[c, :, -1].mean() > base > m[c, :, 0].mean()
    with pytest.raises(ValueError):
        P.write_material(path, m[0], m[1], -m[2])
