"""B200 external-mode (barotropic) solver for the ocean model pyOM2.

The package replaces pyOM2's ``solve_streamfunction`` / ``solve_pressure``
path (for_src/external/*.f90) with hand-written sm_100a CUDA kernels behind
a C ABI (include/pyomgpu.h, ``libpyomgpu.so``), driven from Python with the
same routine names and the same Fortran-ordered model arrays.
"""
from .model import ModelState  # noqa: F401
from ._abi import PyOMGPUError  # noqa: F401
from .external import (  # noqa: F401
    ExternalMode,
    congrad_streamfunction,
    congrad_surf_press,
    isleperim,
    solve_pressure,
    solve_streamfunction,
    streamfunction_init,
)

__version__ = "0.1.0"
