"""funlbm_b200: the per-step lattice-Boltzmann path of funlbm on B200 GPUs.

Drop-in for funlbm's solver / config API (``LBMD3``, ``Config``,
``create_flow``, ``FlowD3Q13/15/19/27``, ``Sphere``, ``Ellipsoid``,
``ParticleSwarm``); every step runs in the hand-written sm_100a kernels of
``liblbm_b200.so`` (C ABI in ``include/funlbm_b200.h``).  There is no CPU
path: without a CUDA device or without the library the calls raise.
"""
from .config import Boundary, BoundaryCondition, BoundaryConfig, FileConfig  # noqa: F401
from .flow import (Flow, FlowConfig, FlowD3, FlowD3Q13, FlowD3Q15, FlowD3Q19,  # noqa: F401
                   FlowD3Q27, Param, create_flow)
from .lattice import Lattice  # noqa: F401
from .lbm import (Config, LBMBase, LBMD3, LBMD3Q13, LBMD3Q15, LBMD3Q19,  # noqa: F401
                  LBMD3Q27, create_lbm_config)
from .particle import (CoordConfig, Coordinate, Ellipsoid, Particle,  # noqa: F401
                       ParticleConfig, ParticleSwarm, Sphere, create_particle,
                       create_particle_swarm)

__version__ = "0.1.0"
