"""B200-native implementation of the fdfault time-stepping hot path.

The solver state lives on the GPU and each Runge-Kutta stage runs as
hand-written sm_100a CUDA kernels behind the C-ABI in ``include/fdfault_b200.h``
(library ``fdfault_b200/libfdfault_b200.so``).  The Python layer here is a
thin host-side mirror of the reference's ``problem``/``domain`` interface
(``problem.solve()``, ``domain.do_rk_stage(dt, stage, t)``) over that C-ABI.
"""

from .problems import (Block, Interface, Output, Pert, Problem, load, mode2_rupture, planar3d,  # noqa: F401
                       stzparam, swparam)
