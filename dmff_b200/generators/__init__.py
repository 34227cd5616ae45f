"""Generator registry: importing this package registers every force-field generator by XML tag
and exports the generator classes under the reference's names (generators/__init__.py)."""
from . import admp, classical, disp, qeq, slater  # noqa: F401
from .admp import ADMPPmeGenerator  # noqa: F401
from .classical import (CoulombGenerator, HarmonicAngleGenerator, HarmonicBondGenerator,  # noqa: F401
                        LennardJonesGenerator, NonbondedGenerator, PeriodicTorsionGenerator)
from .disp import ADMPDispGenerator, ADMPDispPmeGenerator  # noqa: F401
from .qeq import ADMPQeqGenerator  # noqa: F401
from .slater import (QqTtDampingGenerator, SlaterDampingGenerator, SlaterDhfGenerator, SlaterExGenerator,  # noqa: F401
                     SlaterSrDispGenerator, SlaterSrEsGenerator, SlaterSrPolGenerator)
