"""B200-native implementation of ProtoMol 3's nonbonded cutoff / PME force path.

The product is libpmb200.so (CUDA kernels for sm_100a behind the C ABI of include/pmb200.h);
this package holds its in-tree build, the ctypes host mirror of ProtoMol's force plugin surface
(``forces``) and the seeded synthetic water-box generator (``waterbox``).
"""
from . import _lib  # noqa: F401
from .forces import (BondedSystemForce, ForceFactory, Integrator,  # noqa: F401
                     NonbondedCutoffSystemForce, NonbondedPMEwaldSystemForce, ScalarStructure,
                     Topology, evaluate_all)
from .waterbox import pme_grid_for, water_box  # noqa: F401

__all__ = ["Topology", "ScalarStructure", "NonbondedCutoffSystemForce",
           "NonbondedPMEwaldSystemForce", "BondedSystemForce", "ForceFactory", "Integrator",
           "evaluate_all", "water_box", "pme_grid_for"]
