"""B200-native drop-in for the hot path of Fast-GPR-FWI.

The 2-D TMz FDTD Maxwell solver (Ez/Hx/Hy leapfrog, Ca/Cb coefficients from
eps_r and sigma, HORIPML CPML, Hertzian-dipole Ricker source, receiver
sampling) and its adjoint, behind the reference's own entry points:

    compute(...)            reference src/compute.py:33
    apply_filter(...)       reference src/multiscale.py:19
    design_fir_filter(...)  reference src/multiscale.py:4
    total_variation(...)    reference src/tv.py:135

The package directory name is not a Python identifier; import it with
``importlib.import_module("fast-gpr-fwi_b200")`` (or alias it, e.g.
``sys.modules["src"] = ...`` for code written against the reference).
"""
from . import fwi, grid, shots, workloads
from .compute import GPRFWI, Solve, compute
from .multiscale import apply_filter, design_fir_filter
from .tv import total_variation
from .fwi import Inversion

__all__ = ["compute", "GPRFWI", "Solve", "apply_filter", "design_fir_filter", "total_variation", "Inversion"]
