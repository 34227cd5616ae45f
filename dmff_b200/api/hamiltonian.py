"""Hamiltonian / Potential: the drop-in front end (dmff/api/hamiltonian.py:14-137).

``Hamiltonian(*xml)`` instantiates one generator per force tag found in the XML from the
``_DMFFGenerators`` registry (same tag names as the reference); ``createPotential`` types the
topology from the XML residue templates and returns a ``Potential`` whose
``getPotentialFunc(names)`` sums the generators' ``potential_fn(positions, box, pairs, params)``.
Nonbonded methods are accepted as OpenMM constants or their names ("PME", "CutoffPeriodic",
"NoCutoff", "CutoffNonPeriodic").
"""
import numpy as np

from .paramset import ParamSet
from .topology import DMFFTopology, covalent_rows
from .xmlio import XMLIO

_DMFFGenerators = {}


def build_covalent_map(data, max_neighbor):
    """Dense [n, n] matrix of shortest bond-path lengths 1 .. max_neighbor (0 otherwise) for a
    topology record with ``atoms`` and ``bonds`` (bond.atom1 / bond.atom2 as indices or atoms),
    the breadth-first map of hamiltonian.py:17-35."""
    n = len(data.atoms)
    idx = lambda a: int(getattr(a, "index", a))
    rows = covalent_rows(n, [(idx(b.atom1), idx(b.atom2)) for b in data.bonds], max_neighbor)
    cm = np.zeros((n, n), dtype=int)
    if len(rows):
        cm[rows[:, 0], rows[:, 1]] = rows[:, 2]
        cm[rows[:, 1], rows[:, 0]] = rows[:, 2]
    return cm


def method_name(m):
    if isinstance(m, str):
        return m
    n = getattr(m, "__name__", None) or str(m)
    for k in ("CutoffNonPeriodic", "CutoffPeriodic", "NoCutoff", "PME", "LJPME", "Ewald"):
        if k in n:
            return k
    return n


class Potential:
    def __init__(self, topology, has_aux=False):
        self.dmff_potentials = {}
        self.meta = {}
        self.topology = topology
        self.meta["cov_map"] = topology.buildCovMat()
        for key in topology._meta:
            self.meta[key] = topology._meta[key]
        self.has_aux = has_aux

    def add(self, name, func):
        self.dmff_potentials[name] = func

    def getPotentialFunc(self, names=()):
        if isinstance(names, str):
            names = [names]
        names = list(names) or list(self.dmff_potentials.keys())
        if not self.has_aux:
            def efunc(positions, box, pairs, prms):
                return sum(self.dmff_potentials[n](positions, box, pairs, prms) for n in names)
        else:
            def efunc(positions, box, pairs, prms, aux):
                energy, aux = self.dmff_potentials[names[0]](positions, box, pairs, prms, aux)
                for n in names[1:]:
                    e, aux = self.dmff_potentials[n](positions, box, pairs, prms, aux)
                    energy = energy + e
                return energy, aux
        return efunc


class Hamiltonian:
    def __init__(self, *args):
        from .. import generators  # noqa: F401  (registers the generator classes)
        self._xmlio = XMLIO()
        self.generators = {}
        self.paramset = ParamSet()
        for xml in [a for a in args if isinstance(a, str)]:
            self._xmlio.loadXML(xml)
        self.ffinfo = self._xmlio.parseXML()
        for key in self.ffinfo["Forces"].keys():
            if key not in _DMFFGenerators:
                print(f"Generator for {key} is not implemented.")
            else:
                self.generators[key] = _DMFFGenerators[key](self.ffinfo, self.paramset)

    def getGenerators(self):
        return list(self.generators.values())

    def createPotential(self, topdata, nonbondedMethod="NoCutoff", nonbondedCutoff=1.0, **kwargs):
        if not isinstance(topdata, DMFFTopology):
            raise TypeError("createPotential expects a dmff_b200 DMFFTopology (e.g. PDBFile(...).topology)")
        topdata.apply_templates(self.ffinfo)
        potential = Potential(topdata, has_aux=bool(kwargs.get("has_aux", False)))
        for key, gen in self.generators.items():
            potential.add(gen.getName(), gen.createPotential(topdata, nonbondedMethod, nonbondedCutoff, **kwargs))
        potential.meta.update({k: v for k, v in topdata._meta.items()})
        return potential

    def getParameters(self):
        return self.paramset
