"""The project's .in writer produces what the reference's Python module writes."""

import os
import sys

import pytest

from fdfault_b200 import problems as P

import oracle

REF_PY = os.path.join(oracle.reference_dir(), "python")


@pytest.mark.skipif(not os.path.isdir(REF_PY), reason="reference Python module not present")
def test_writer_matches_reference_module(tmp_path):
    sys.path.insert(0, REF_PY)
    try:
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            import fdfault
    finally:
        sys.path.remove(REF_PY)
    os.chdir(tmp_path)
    r = fdfault.problem("cmp")
    r.set_rkorder(3); r.set_sbporder(4); r.set_nt(100); r.set_cfl(0.3); r.set_ninfo(1000000)
    r.set_ndim(2); r.set_mode(2)
    r.set_nblocks((1, 2, 1)); r.set_nx_block(([401], [201, 201], [1]))
    r.set_block_lx((0, 0, 0), (40., 20.)); r.set_block_lx((0, 1, 0), (40., 20.))
    r.set_domain_xm((0., 0.))
    r.set_bounds((0, 0, 0), ["absorbing", "absorbing", "absorbing", "none"])
    r.set_bounds((0, 1, 0), ["absorbing", "absorbing", "none", "absorbing"])
    r.set_material(fdfault.material("elastic", P.RHO, P.LAM, P.G))
    r.set_iftype(0, "slipweak")
    r.add_pert(fdfault.swparam("constant", 0., 0., 0., 0., 0., 0.4, 0.677, 0.525))
    r.add_load(fdfault.load("constant", 0., 0., 0., 0., 0., -120., 70., 0.))
    r.add_load(fdfault.load("boxcar", 0., 20., 1.5, 0., 0., 0., 11.6, 0.))
    r.write_input()
    mine = P.mode2_rupture(nx=401, ny=201, h=0.1, nt=100, name="cmp")
    mine.ninfo = 1000000
    ref_tokens = open(tmp_path / "cmp.in").read().split()
    my_tokens = mine.text().split()
    # compare token streams numerically where both parse as numbers
    assert len(ref_tokens) == len(my_tokens)
    for a, b in zip(ref_tokens, my_tokens):
        try:
            assert float(a) == float(b), (a, b)
        except ValueError:
            assert a == b, (a, b)


def test_lognormal_field_statistics():
    f = P.lognormal_field(401, 201, 0.1, 0.677, 0.03, 2.0, seed=7)
    assert f.shape == (401, 201)
    assert abs(f.mean() - 0.677) < 0.01
    assert 0.02 < f.std() < 0.04
    assert (f > 0).all()


@pytest.mark.skipif(not os.path.isdir(REF_PY), reason="reference Python module not present")
def test_material_file_matches_reference_module(tmp_path):
    """A heterogeneous material file written by problems.write_material has the
    bytes the reference's Python module writes for the same arrays
    (python/fdfault/fields.py set_het_material / write_input)."""
    import numpy as np
    sys.path.insert(0, REF_PY)
    try:
        import warnings
        with warnings.catch_warnings():
            warnings.simplefilter("ignore")
            import fdfault
    finally:
        sys.path.remove(REF_PY)
    os.chdir(tmp_path)
    nx, ny = 21, 11
    rng = np.random.default_rng(3)
    mat = np.stack([base * (1. + 0.1 * rng.uniform(-1., 1., (nx, ny, 1))) for base in (P.RHO, P.LAM, P.G)])
    r = fdfault.problem("matcmp")
    r.set_ndim(2); r.set_mode(2)
    r.set_nblocks((1, 1, 1)); r.set_nx_block(([nx], [ny], [1]))
    r.set_block_lx((0, 0, 0), (2., 1.))
    r.set_nt(1); r.set_cfl(0.3)
    r.set_material(fdfault.material("elastic", P.RHO, P.LAM, P.G))
    r.set_het_material(mat[..., 0])   # 2D: (3, nx, ny)
    r.write_input()
    mine = P.write_material(str(tmp_path / "mine.mat"), mat[0], mat[1], mat[2])
    assert open(mine, "rb").read() == open(tmp_path / "matcmp.mat", "rb").read()
    # the .in line names the file where the fields section expects it
    assert str(tmp_path / "matcmp.mat") in open(tmp_path / "matcmp.in").read() or \
        "matcmp.mat" in open(tmp_path / "matcmp.in").read()
