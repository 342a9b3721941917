"""coffee_b200: B200-native field update of COFFEE's force-free EZ solver.

The CUDA kernels and the C ABI live in libcoffee_b200.so (sources in
coffee_b200/csrc, API in include/coffee_b200.h).  This package holds the
host-side helpers around that ABI: the ctypes binding (_lib), the mirror of
the reference's sim_environment / sim_data / field_solver_EZ objects
(solver), the sim_params mirror and TOML keys (config), the field-file
format (fld) and the problem set-ups (problems).
"""
from .config import Grid, SimParams  # noqa: F401

__all__ = ["Grid", "SimParams"]
