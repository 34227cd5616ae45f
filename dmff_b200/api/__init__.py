"""Front end with the names of dmff/api: Hamiltonian, DMFFTopology (api/__init__.py)."""
from .hamiltonian import Hamiltonian  # noqa: F401
from .topology import DMFFTopology  # noqa: F401
