"""dmff_b200: B200-native ADMP / PME energy-force path with DMFF's generator API.

Public entry points mirror deepmodeling/DMFF: ``Hamiltonian``, ``NeighborList``,
``ADMPPmeForce``; the compute runs in ``libdmffb200.so`` (hand-written sm_100a kernels behind
the C ABI in include/dmffb200.h).
"""
from .api.hamiltonian import Hamiltonian, Potential  # noqa: F401
from .api.paramset import ParamSet  # noqa: F401
from .api.topology import DMFFTopology, PDBFile  # noqa: F401


def __getattr__(name):
    if name in ("NeighborList", "NeighborListFreud"):
        from .common import nblist
        return getattr(nblist, name)
    if name == "ADMPPmeForce":
        from .admp.pme import ADMPPmeForce
        return ADMPPmeForce
    raise AttributeError(name)
