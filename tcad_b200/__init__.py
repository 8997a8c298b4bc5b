"""tcad_b200 -- PyTCAD's structured drift-diffusion solve path on B200 (sm_100a).

The reference's device API (Device2D / Device3D, Mesh2D / Mesh3D, Models,
NewtonOptions, linsolve.solve_linear) backed by hand-written CUDA kernels in
``libtcad_b200.so`` (C ABI: include/tcad_b200.h).  No CPU fallback: the
solve methods raise when the library or a CUDA device is missing.
"""
from .options import Models, NewtonOptions  # noqa: F401
from .physics import (SILICON, Semiconductor, Mesh2D, Mesh3D, graded_nodes,  # noqa: F401
                      flatband_voltage, thermal_voltage)
from .linsolve import LinearSolveError, solve_linear  # noqa: F401
from .device import Device2D, Device3D  # noqa: F401

__version__ = "0.1"
