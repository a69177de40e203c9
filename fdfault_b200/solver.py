"""ctypes binding of the C ABI (include/fdfault_b200.h) and a host-side mirror
of the reference's problem / domain interface.

``Problem(infile)`` stands for ``problem::problem`` (src/problem.cpp:16),
``Problem.solve()`` for ``problem::solve`` (src/problem.cpp:136) and
``Problem.do_rk_stage(dt, stage, t)`` for ``domain::do_rk_stage``
(src/domain.cpp:228).  Errors raise ``FdfaultError`` with the library's
message, the way the reference aborts with a message.

The native library must be present: importing this module on a machine where
``libfdfault_b200.so`` has not been built raises instead of falling back to
any other implementation.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfdfault_b200.so")

FP64, FP32 = 0, 1
GEOM_X, GEOM_METRIC, GEOM_JAC = 0, 1, 2
(U, DU, V, S, SN, UX, DUX, VX, SX, STATE, DSTATE, DSTATEDT, TFRONT) = range(13)


class FdfaultError(RuntimeError):
    pass


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FdfaultError("native library %s is missing; build it with fdfault_b200/build.py" % path)
    L = ctypes.CDLL(path)
    c_int, c_double, c_ll = ctypes.c_int, ctypes.c_double, ctypes.c_longlong
    P = ctypes.POINTER
    dp = P(c_double)
    L.fdf_create.argtypes = [ctypes.c_char_p, c_int, c_int, P(ctypes.c_void_p)]
    L.fdf_destroy.argtypes = [ctypes.c_void_p]
    L.fdf_destroy.restype = None
    L.fdf_get_info.argtypes = [ctypes.c_void_p, P(c_int), dp]
    L.fdf_do_rk_stage.argtypes = [ctypes.c_void_p, c_double, c_int, c_double]
    L.fdf_step.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_solve.argtypes = [ctypes.c_void_p]
    L.fdf_get_step.argtypes = [ctypes.c_void_p, P(c_int)]
    L.fdf_set_step.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_get_field.argtypes = [ctypes.c_void_p, c_int, c_int, dp]
    L.fdf_get_field_noalloc.argtypes = [ctypes.c_void_p, c_int, c_int, dp]
    L.fdf_set_field.argtypes = [ctypes.c_void_p, c_int, dp]
    L.fdf_get_rate.argtypes = [ctypes.c_void_p, c_int, dp]
    L.fdf_set_rate.argtypes = [ctypes.c_void_p, c_int, dp]
    L.fdf_get_geometry.argtypes = [ctypes.c_void_p, c_int, c_int, dp]
    L.fdf_fault_count.argtypes = [ctypes.c_void_p, c_int, c_int, P(c_ll)]
    L.fdf_get_fault.argtypes = [ctypes.c_void_p, c_int, c_int, dp]
    L.fdf_get_fault_async.argtypes = [ctypes.c_void_p, c_int, c_int, dp]
    L.fdf_set_fault.argtypes = [ctypes.c_void_p, c_int, c_int, dp]
    L.fdf_synchronize.argtypes = [ctypes.c_void_p]
    L.fdf_time_steps.argtypes = [ctypes.c_void_p, c_int, dp]
    L.fdf_profile.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_profile_read.argtypes = [ctypes.c_void_p, c_int, dp, P(c_ll)]
    L.fdf_use_fast_kernel.argtypes = [ctypes.c_void_p, c_int, P(c_int)]
    L.fdf_set_volume_kernel.argtypes = [ctypes.c_void_p, c_int, P(c_int)]
    L.fdf_set_wait_limit.argtypes = [ctypes.c_void_p, ctypes.c_longlong]
    L.fdf_set_plastic_rule.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_energy.argtypes = [ctypes.c_void_p, c_int, P(ctypes.c_double)]
    L.fdf_use_graphs.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_bytes_per_node_stage.argtypes = [ctypes.c_void_p, P(c_ll)]
    fp = P(ctypes.c_float)
    L.fdf_stz_set_learned.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_stz_set_start.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_stz_set_counting.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_stz_read_counts.argtypes = [ctypes.c_void_p, P(c_ll), c_int]
    L.fdf_stz_collect.argtypes = [ctypes.c_void_p, c_ll]
    L.fdf_stz_samples.argtypes = [ctypes.c_void_p, fp, c_ll, P(c_ll)]
    L.fdf_mlp_init.argtypes = [ctypes.c_void_p, ctypes.c_ulonglong]
    L.fdf_mlp_set_params.argtypes = [ctypes.c_void_p, fp]
    L.fdf_mlp_get_params.argtypes = [ctypes.c_void_p, fp]
    L.fdf_mlp_infer.argtypes = [ctypes.c_void_p, fp, c_ll, fp, c_int]
    L.fdf_mlp_gradients.argtypes = [ctypes.c_void_p, fp, fp, c_ll, fp, dp]
    L.fdf_mlp_train.argtypes = [ctypes.c_void_p, c_int, c_int, ctypes.c_float, ctypes.c_ulonglong, dp, dp]
    vp = ctypes.c_void_p
    L.fdf_ensemble_create.argtypes = [P(ctypes.c_char_p), c_int, c_int, P(vp)]
    L.fdf_ensemble_destroy.argtypes = [vp]
    L.fdf_ensemble_destroy.restype = None
    L.fdf_ensemble_size.argtypes = [vp, P(c_int)]
    L.fdf_ensemble_member.argtypes = [vp, c_int, P(vp)]
    L.fdf_ensemble_run.argtypes = [vp, c_int]
    L.fdf_ensemble_time_steps.argtypes = [vp, c_int, dp]
    L.fdf_ensemble_autotune.argtypes = [vp, c_int, P(c_int), P(c_ll)]
    L.fdf_ensemble_set_config.argtypes = [vp, c_int, c_ll]
    L.fdf_ensemble_use_graph.argtypes = [vp, c_int]
    L.fdf_ensemble_node_stages.argtypes = [vp, P(c_ll)]
    L.fdf_ensemble_check_status.argtypes = [vp]
    L.fdf_ensemble_last_error.argtypes = [vp]
    L.fdf_ensemble_last_error.restype = ctypes.c_char_p
    L.fdf_step_stage.argtypes = [ctypes.c_void_p, c_int]
    L.fdf_set_x_range.argtypes = [ctypes.c_void_p, c_int, c_int]
    L.fdf_ghost_info.argtypes = [ctypes.c_void_p, P(c_int), P(c_ll), P(c_int)]
    L.fdf_pack_ghosts.argtypes = [ctypes.c_void_p, c_int, vp]
    L.fdf_unpack_ghosts.argtypes = [ctypes.c_void_p, c_int, vp]
    L.fdf_get_block.argtypes = [ctypes.c_void_p, c_int, P(c_int), P(c_int)]
    L.fdf_set_stream.argtypes = [ctypes.c_void_p, c_int, vp]
    L.fdf_get_interface.argtypes = [ctypes.c_void_p, c_int, P(c_int), P(c_int), P(c_int)]
    L.fdf_last_error.argtypes = [ctypes.c_void_p]
    L.fdf_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


MLP_NPARAM = 4673   # W1[64][6], b1[64], W2[64][64], b2[64], W3[64], b3


class Problem:
    """One fdfault problem held on a GPU."""

    def __init__(self, infile: Optional[str], precision: int = FP64, device: int = 0, _handle=None, _owner=None):
        self._L = load_library()
        if _handle is None:
            h = ctypes.c_void_p()
            rc = self._L.fdf_create(infile.encode(), precision, device, ctypes.byref(h))
            if rc:
                raise FdfaultError(self._L.fdf_last_error(None).decode())
        else:
            h = _handle   # a member of an Ensemble (which owns the solver)
        self._h = h
        self._owner = _owner
        self.precision = precision
        self.device = device
        ints = (ctypes.c_int * 16)()
        dbls = (ctypes.c_double * 3)()
        self._check(self._L.fdf_get_info(self._h, ints, dbls))
        v = list(ints)
        self.ndim, self.mode = v[0], v[1]
        self.nx: Tuple[int, int, int] = (v[2], v[3], v[4])
        self.nfields, self.nfieldsp, self.nifaces, self.nstages, self.nt = v[5], v[6], v[7], v[8], v[9]
        self.sbporder = v[10]
        self.nblocks = (v[11], v[12], v[13])
        self.is_plastic = bool(v[14])
        self.rkorder = v[15]
        self.dt, self.ttot, self.cfl = list(dbls)
        self.nxyz = self.nx[0] * self.nx[1] * self.nx[2]

    def _check(self, rc: int) -> None:
        if rc:
            raise FdfaultError(self._L.fdf_last_error(self._h).decode())

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._L.fdf_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- time stepping -------------------------------------------------
    def do_rk_stage(self, dt: float, stage: int, t: float) -> None:
        self._check(self._L.fdf_do_rk_stage(self._h, dt, stage, t))

    def step(self, nsteps: int = 1) -> None:
        self._check(self._L.fdf_step(self._h, nsteps))

    def solve(self) -> None:
        self._check(self._L.fdf_solve(self._h))

    def step_stage(self, stage: int) -> None:
        """Stage `stage` of the current step as step() runs it; the last stage
        advances the step counter."""
        self._check(self._L.fdf_step_stage(self._h, stage))

    # --- x slabs (one process per GPU; fdfault_b200.slabs drives them) ----
    def set_x_range(self, x0: int, x1: int) -> None:
        """Update only the global x planes [x0, x1) (cartesian.cpp:88-165 splits
        the reference's domain across MPI ranks)."""
        self._check(self._L.fdf_set_x_range(self._h, x0, x1))

    def ghost_info(self) -> Tuple[int, int, int]:
        """(ghost planes per side, elements of one side's exchange, bytes per element)."""
        g, n, e = ctypes.c_int(), ctypes.c_longlong(), ctypes.c_int()
        self._check(self._L.fdf_ghost_info(self._h, ctypes.byref(g), ctypes.byref(n), ctypes.byref(e)))
        return g.value, n.value, e.value

    def pack_ghosts(self, side: int, dst_ptr: int) -> None:
        """Side 0: the slab's first planes; side 1: its last ones, into the device buffer at dst_ptr."""
        self._check(self._L.fdf_pack_ghosts(self._h, side, ctypes.c_void_p(dst_ptr)))

    def unpack_ghosts(self, side: int, src_ptr: int) -> None:
        """Side 0: the ghost planes below the slab; side 1: those above it, from the device buffer."""
        self._check(self._L.fdf_unpack_ghosts(self._h, side, ctypes.c_void_p(src_ptr)))

    def block(self, b: int) -> Tuple[Tuple[int, int, int], Tuple[int, int, int]]:
        """(first global node, node counts) of block b."""
        lo, n = (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        self._check(self._L.fdf_get_block(self._h, b, lo, n))
        return tuple(lo), tuple(n)

    def interface(self, iface: int) -> Tuple[int, Tuple[int, int, int], Tuple[int, int]]:
        """(normal direction, first global node of the minus-side face, face node counts)."""
        d, lo, n = ctypes.c_int(), (ctypes.c_int * 3)(), (ctypes.c_int * 2)()
        self._check(self._L.fdf_get_interface(self._h, iface, ctypes.byref(d), lo, n))
        return d.value, tuple(lo), tuple(n)

    @property
    def torch_device(self):
        """The torch device that holds this problem's buffers."""
        import torch

        return torch.device("cuda", self.device)

    def set_stream(self, stream: Optional[int]) -> None:
        """Launch on the CUDA stream handle `stream` (an int, 0 the legacy
        default stream), or on the problem's own stream when None."""
        if stream is None:
            self._check(self._L.fdf_set_stream(self._h, 1, None))
        else:
            self._check(self._L.fdf_set_stream(self._h, 0, ctypes.c_void_p(stream)))

    @property
    def step_index(self) -> int:
        v = ctypes.c_int()
        self._check(self._L.fdf_get_step(self._h, ctypes.byref(v)))
        return v.value

    @step_index.setter
    def step_index(self, i: int) -> None:
        self._check(self._L.fdf_set_step(self._h, i))

    def synchronize(self) -> None:
        self._check(self._L.fdf_synchronize(self._h))

    def time_steps(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        self._check(self._L.fdf_time_steps(self._h, nsteps, ctypes.byref(ms)))
        return ms.value

    def profile(self, on: bool) -> None:
        self._check(self._L.fdf_profile(self._h, int(on)))

    def profile_read(self, kernel: int) -> Tuple[float, int]:
        ms, n = ctypes.c_double(), ctypes.c_longlong()
        self._check(self._L.fdf_profile_read(self._h, kernel, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    # --- STZ friction: learned Newton start ------------------------------
    def stz_learned(self, on: bool) -> None:
        self._check(self._L.fdf_stz_set_learned(self._h, int(on)))

    STZ_MIDPOINT, STZ_LEARNED, STZ_WARM, STZ_EXACT_DERIVATIVE = 0, 1, 2, 3

    def stz_start(self, mode: int) -> None:
        """Start of the STZ Newton solve: 0 bracket midpoint (reference), 1
        learned, 2 warm start from each node's previous root, 3 midpoint with
        the exact derivative."""
        self._check(self._L.fdf_stz_set_start(self._h, mode))

    def stz_counting(self, on: bool) -> None:
        self._check(self._L.fdf_stz_set_counting(self._h, int(on)))

    def stz_counts(self, reset: bool = True) -> Tuple[int, int, int]:
        """(Newton solves, iterations, solves started at the bracket midpoint)."""
        c = (ctypes.c_longlong * 3)()
        self._check(self._L.fdf_stz_read_counts(self._h, c, int(reset)))
        return c[0], c[1], c[2]

    def stz_collect(self, capacity: int) -> None:
        self._check(self._L.fdf_stz_collect(self._h, capacity))

    def stz_sample_count(self) -> int:
        n = ctypes.c_longlong()
        self._check(self._L.fdf_stz_samples(self._h, None, 0, ctypes.byref(n)))
        return n.value

    def stz_samples(self, max_rows: Optional[int] = None) -> np.ndarray:
        """Collected rows [n][8]: 6 network inputs, target t = logit(s)/20, converged mu."""
        n = ctypes.c_longlong()
        self._check(self._L.fdf_stz_samples(self._h, None, 0, ctypes.byref(n)))
        k = n.value if max_rows is None else min(n.value, max_rows)
        out = np.zeros((k, 8), dtype=np.float32)
        if k:
            self._check(self._L.fdf_stz_samples(self._h, _fptr(out), k, ctypes.byref(n)))
        return out

    def mlp_init(self, seed: int) -> None:
        self._check(self._L.fdf_mlp_init(self._h, seed))

    def mlp_set_params(self, p: np.ndarray) -> None:
        a = np.ascontiguousarray(p, dtype=np.float32).reshape(-1)
        assert a.size == MLP_NPARAM
        self._check(self._L.fdf_mlp_set_params(self._h, _fptr(a)))

    def mlp_params(self) -> np.ndarray:
        out = np.empty(MLP_NPARAM, dtype=np.float32)
        self._check(self._L.fdf_mlp_get_params(self._h, _fptr(out)))
        return out

    def mlp_infer(self, x: np.ndarray, force_thread: bool = False) -> np.ndarray:
        a = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 6)
        y = np.empty(a.shape[0], dtype=np.float32)
        self._check(self._L.fdf_mlp_infer(self._h, _fptr(a), a.shape[0], _fptr(y), int(force_thread)))
        return y

    def mlp_gradients(self, x: np.ndarray, t: np.ndarray) -> Tuple[np.ndarray, float]:
        a = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, 6)
        tt = np.ascontiguousarray(t, dtype=np.float32).reshape(-1)
        g = np.empty(MLP_NPARAM, dtype=np.float32)
        loss = ctypes.c_double()
        self._check(self._L.fdf_mlp_gradients(self._h, _fptr(a), _fptr(tt), a.shape[0], _fptr(g),
                                              ctypes.byref(loss)))
        return g, loss.value

    def mlp_train(self, epochs: int, batch: int = 8192, lr: float = 1e-3, seed: int = 0) -> Tuple[float, float]:
        """Adam on the collected samples; returns (last-epoch training loss, held-out loss)."""
        tr, va = ctypes.c_double(), ctypes.c_double()
        self._check(self._L.fdf_mlp_train(self._h, epochs, batch, lr, seed, ctypes.byref(tr), ctypes.byref(va)))
        return tr.value, va.value

    def use_graphs(self, on: bool) -> None:
        """Replay pairs of steps from a captured CUDA graph (default on)."""
        self._check(self._L.fdf_use_graphs(self._h, int(on)))

    def set_volume_kernel(self, kind: int) -> int:
        """FP32 volume kernel: 0 reference order, 1 tiled (3D, or 2D elastic), 2 staged (3D),
        3 register window (3D); returns the kind that runs."""
        act = ctypes.c_int()
        self._check(self._L.fdf_set_volume_kernel(self._h, kind, ctypes.byref(act)))
        return act.value

    def energy(self, rate: bool = True) -> dict:
        """FP64 energy diagnostics (elastic problems): kinetic and strain energy
        in the SBP norm, with `rate` their rate under the semi-discrete operator
        at the current state (the state does not move; the rate register is left
        holding dt L(f)) and the rate terms' magnitude sum, and the interfaces'
        frictional power."""
        out = (ctypes.c_double * 8)()
        self._check(self._L.fdf_energy(self._h, int(rate), out))
        return {"kinetic": out[0], "strain": out[1], "total": out[0] + out[1], "rate": out[2],
                "rate_scale": out[3], "friction_power": out[4]}

    PLASTIC_REFERENCE, PLASTIC_EVERY_NODE = 0, 1

    def set_plastic_rule(self, rule: int) -> None:
        """Return-map rule of plastic problems: 0 the reference's loop
        (block.cpp:442-589; trunc(lambda + 2/3 G) as bulk modulus, in 3D the
        first z node of each block column), 1 every node with the exact
        modulus."""
        self._check(self._L.fdf_set_plastic_rule(self._h, rule))

    def set_wait_limit(self, polls: int) -> None:
        """Polls of each bounded wait for staged data in volume kernels 2 and 3
        (0: the built-in limit); 1 makes every wait a single immediate test,
        a negative value makes every such wait give up at once."""
        self._check(self._L.fdf_set_wait_limit(self._h, polls))

    def use_fast_kernel(self, on: bool) -> bool:
        act = ctypes.c_int()
        self._check(self._L.fdf_use_fast_kernel(self._h, int(on), ctypes.byref(act)))
        return bool(act.value)

    def bytes_per_node_stage(self) -> int:
        b = ctypes.c_longlong()
        self._check(self._L.fdf_bytes_per_node_stage(self._h, ctypes.byref(b)))
        return b.value

    # --- state access --------------------------------------------------
    def field(self, comp: int, absolute: bool = False, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.nxyz)
        elif out.dtype != np.float64 or out.size != self.nxyz or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of %d values" % self.nxyz)
        self._check(self._L.fdf_get_field(self._h, comp, int(absolute), _dptr(out)))
        return out

    def field_noalloc(self, comp: int, absolute: bool = False) -> np.ndarray:
        """As field(), through the allocation-free entry point (fixed device buffer)."""
        out = np.empty(self.nxyz)
        self._check(self._L.fdf_get_field_noalloc(self._h, comp, int(absolute), _dptr(out)))
        return out

    def set_field(self, comp: int, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        assert a.size == self.nxyz
        self._check(self._L.fdf_set_field(self._h, comp, _dptr(a)))

    def rate(self, comp: int) -> np.ndarray:
        out = np.empty(self.nxyz)
        self._check(self._L.fdf_get_rate(self._h, comp, _dptr(out)))
        return out

    def set_rate(self, comp: int, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        assert a.size == self.nxyz
        self._check(self._L.fdf_set_rate(self._h, comp, _dptr(a)))

    def geometry(self, which: int, comp: int = 0) -> np.ndarray:
        out = np.empty(self.nxyz)
        self._check(self._L.fdf_get_geometry(self._h, which, comp, _dptr(out)))
        return out

    def fault_count(self, iface: int, which: int) -> int:
        n = ctypes.c_longlong()
        self._check(self._L.fdf_fault_count(self._h, iface, which, ctypes.byref(n)))
        return n.value

    def fault(self, iface: int, which: int, out: Optional[np.ndarray] = None) -> Optional[np.ndarray]:
        """Fault array `which` of interface `iface`; written into `out` (a
        contiguous float64 array of the right size, e.g. a view of pinned host
        memory) when given."""
        n = self.fault_count(iface, which)
        if n == 0:
            return None
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of %d values" % n)
        self._check(self._L.fdf_get_fault(self._h, iface, which, _dptr(out)))
        return out

    def fault_async(self, iface: int, which: int, out: np.ndarray) -> None:
        """Queue the copy of fault array `which` of interface `iface` into
        `out` behind the work already queued and return at once; `out` holds the
        values after the next synchronize() and must stay alive until then
        (page-locked memory, e.g. a pinned torch tensor's numpy view, lets the
        copy overlap host work)."""
        n = self.fault_count(iface, which)
        if out.dtype != np.float64 or out.size != n or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of %d values" % n)
        self._check(self._L.fdf_get_fault_async(self._h, iface, which, _dptr(out)))

    def set_fault(self, iface: int, which: int, values: np.ndarray) -> None:
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        assert a.size == self.fault_count(iface, which)
        self._check(self._L.fdf_set_fault(self._h, iface, which, _dptr(a)))


class Ensemble:
    """Independent FP32 problems advanced together by batched launches
    (one volume and one interface launch per stage for all members, chunks
    of steps replayed from a CUDA graph).  ``member(i)`` gives a Problem view
    of member i for reading its fields and fault arrays."""

    def __init__(self, infiles: Sequence[str], device: int = 0):
        self._L = load_library()
        arr = (ctypes.c_char_p * len(infiles))(*[f.encode() for f in infiles])
        h = ctypes.c_void_p()
        rc = self._L.fdf_ensemble_create(arr, len(infiles), device, ctypes.byref(h))
        if rc:
            raise FdfaultError(self._L.fdf_ensemble_last_error(None).decode())
        self._h = h
        self.device = device
        self._members = {}
        n = ctypes.c_int()
        self._check(self._L.fdf_ensemble_size(self._h, ctypes.byref(n)))
        self.size = n.value

    def _check(self, rc: int) -> None:
        if rc:
            raise FdfaultError(self._L.fdf_ensemble_last_error(self._h).decode())

    def member(self, i: int) -> Problem:
        if i not in self._members:
            h = ctypes.c_void_p()
            self._check(self._L.fdf_ensemble_member(self._h, i, ctypes.byref(h)))
            self._members[i] = Problem(None, FP32, device=self.device, _handle=h, _owner=self)
        return self._members[i]

    def run(self, nsteps: int) -> None:
        self._check(self._L.fdf_ensemble_run(self._h, nsteps))

    def time_steps(self, nsteps: int) -> float:
        ms = ctypes.c_double()
        self._check(self._L.fdf_ensemble_time_steps(self._h, nsteps, ctypes.byref(ms)))
        return ms.value

    def autotune(self, steps: int = 2) -> Tuple[int, int]:
        th, tl = ctypes.c_int(), ctypes.c_longlong()
        self._check(self._L.fdf_ensemble_autotune(self._h, steps, ctypes.byref(th), ctypes.byref(tl)))
        return th.value, tl.value

    def set_config(self, threads: int, tile: int) -> None:
        self._check(self._L.fdf_ensemble_set_config(self._h, threads, tile))

    def use_graph(self, on: bool) -> None:
        self._check(self._L.fdf_ensemble_use_graph(self._h, int(on)))

    def node_stages_per_step(self) -> int:
        n = ctypes.c_longlong()
        self._check(self._L.fdf_ensemble_node_stages(self._h, ctypes.byref(n)))
        return n.value

    def check_status(self) -> None:
        self._check(self._L.fdf_ensemble_check_status(self._h))

    def close(self) -> None:
        for m in self._members.values():
            m.close()
        self._members = {}
        if getattr(self, "_h", None):
            self._L.fdf_ensemble_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
