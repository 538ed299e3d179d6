"""nhflood: B200-native local-inertial step of the nh-flood-2d compact solver.

The step runs in hand-written sm_100a CUDA kernels (libnhflood.so, C ABI in
include/nhflood.h); this package is the host side: configs, NE/NS
preprocessing, forcing, the batch time loop and the outputs.
"""
from .input import DomainConfig, ForceConfig, load_domain_config, load_force_config  # noqa: F401
from .solver_compact import run_simulation, solver, warmup_solver  # noqa: F401

__version__ = '0.1.0'
