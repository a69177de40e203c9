"""Shared helpers: emulate the reference's output units from in-memory state."""

from __future__ import annotations

import os
from typing import Dict

import numpy as np

import cases

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

VOL3 = ["vx", "vy", "vz", "sxx", "sxy", "sxz", "syy", "syz", "szz", "lambda", "gammap",
        "epxx", "epxy", "epxz", "epyy", "epyz", "epzz"]
VOL2M2 = ["vx", "vy", "sxx", "sxy", "syy", "szz", "lambda", "gammap", "epxx", "epxy", "epxz", "epyy", "epyz", "epzz"]
VOL2M3 = ["vz", "sxz", "syz", "lambda", "gammap", "epxx", "epxy", "epxz", "epyy", "epyz", "epzz"]


def load_golden(name: str) -> Dict[str, np.ndarray]:
    with np.load(os.path.join(GOLDEN, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def vol_comp(prob, field: str) -> int:
    if prob.ndim == 3:
        return VOL3.index(field)
    return (VOL2M2 if prob.mode == 2 else VOL2M3).index(field)


def unit_slice(prob, o):
    """Index expression selecting the unit's points from a (nx, ny, nz) array."""
    nx = prob.nx
    sl = []
    for d in range(3):
        xm = max(o.xm[d], 0)
        xp = nx[d] - 1 if o.xp[d] >= nx[d] else o.xp[d] - (o.xp[d] - o.xm[d]) % o.xs[d]
        sl.append(slice(xm, xp + 1, o.xs[d]))
    return tuple(sl)


def fault_sel(prob, o, field, arrays_getter):
    """Fault unit values at one step from fault arrays (iface index from unit name)."""
    n = int(o.name[1:o.name.index("_")])
    itf = prob.interfaces[n]
    base, comp = cases.fault_fields(prob, n)
    compk = dict(comp)
    key = {"V": "v", "U": "u", "S": "s", "Sn": "sn", "state": "state"}
    if field in compk:
        arr = arrays_getter(n, {"V": "vx", "U": "ux", "S": "sx"}[field[0]])
        nn = arr.size // (prob.ndim - 1)
        return arr[compk[field] * nn:(compk[field] + 1) * nn]
    return arrays_getter(n, key[field])
