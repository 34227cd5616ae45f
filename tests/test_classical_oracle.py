"""Classical terms: the float64 oracle, driven by this package's XML/PDB front end and term
enumeration, against the reference's classical goldens (tests/test_classical/test_bonded.py,
test_lj.py, test_coul.py of deepmodeling/DMFF)."""
import json
import math
import os

import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200 import Hamiltonian, PDBFile
from helpers import classical_oracle

HERE = os.path.join(os.path.dirname(__file__), "golden")
GOLD = json.load(open(os.path.join(HERE, "energies.json")))["classical"]


def _data(name):
    return os.path.join(HERE, "data", name)


# generators each reference test sums (getPotentialFunc(names=...)); None = all of them
NAMES = {"test_harmonic_bond_force": ["HarmonicBondForce"], "test_coul_force": ["NonbondedForce"],
         "test_coul_pme": ["NonbondedForce"]}


def golden_case(c, with_potential=False, **kw):
    """(Hamiltonian, pdb, box nm, pairs[, potential]) set up as the reference test does."""
    pdb = PDBFile(_data(c["pdb"]))
    H = Hamiltonian(_data(c["xml"]))
    if c["test"] == "test_coul_pme":
        rc, box = 0.5, np.eye(3) * 1.2
        pot = H.createPotential(pdb.topology, nonbondedMethod="PME", nonbondedCutoff=rc, PmeCoeffMethod="gromacs",
                                PmeSpacing=0.10, **kw)
    else:
        rc, box = 4.0, np.eye(3) * 10.0
        pot = H.createPotential(pdb.topology, nonbondedMethod="NoCutoff", nonbondedCutoff=rc, **kw)
    pos = pdb.positions
    if c["test"].startswith(("test_harmonic", "test_periodic")):
        pairs = np.zeros((0, 3), dtype=np.int64)
    else:
        cov = pdb.topology.buildCovMat()
        pairs = R.brute_force_pairs(pos, box, rc, lambda i, j: int(cov.lookup(i, j)))
    if with_potential:
        return H, pdb, box, pairs, pot
    return H, pdb, box, pairs


@pytest.mark.parametrize("c", GOLD, ids=[f"{c['test']}-{c['xml']}" for c in GOLD])
def test_classical_goldens(c):
    H, pdb, box, pairs = golden_case(c)
    E, _, _ = classical_oracle(H, pdb.positions, box, pairs, names=NAMES.get(c["test"]))
    if "atol" in c:
        assert abs(E.item() - c["value"]) < c["atol"]
    else:
        np.testing.assert_almost_equal(E.item(), c["value"], decimal=c["decimal"])


def test_term_enumeration_counts():
    # impr1: one improper with centre N1 third, amber order (N2, N3, N1, N4); proper2: two propers x 4 terms
    pdb = PDBFile(_data("impr1.pdb"))
    H = Hamiltonian(_data("impr1.xml"))
    H.createPotential(pdb.topology, nonbondedMethod="NoCutoff", nonbondedCutoff=1.0)
    g = H.generators["PeriodicTorsionForce"]
    assert g.torsion_idx.tolist() == [[1, 2, 0, 3]]
    pdb = PDBFile(_data("proper2.pdb"))
    H = Hamiltonian(_data("proper2.xml"))
    H.createPotential(pdb.topology, nonbondedMethod="NoCutoff", nonbondedCutoff=1.0)
    g = H.generators["PeriodicTorsionForce"]
    assert g.torsion_idx.shape == (8, 4) and g.n_proper == 8


def test_angle_formula_on_angle1():
    # no golden in the reference suite: the harmonic angle at arccos(1/sqrt 3) against the closed form
    pdb = PDBFile(_data("angle1.pdb"))
    H = Hamiltonian(_data("angle1.xml"))
    H.createPotential(pdb.topology, nonbondedMethod="NoCutoff", nonbondedCutoff=1.0)
    E, _, _ = classical_oracle(H, pdb.positions, np.eye(3) * 10, np.zeros((0, 3)))
    ref = 0.5 * 836.8 * (math.acos(1 / math.sqrt(3)) - 1.8242181341844732) ** 2
    assert abs(E.item() - ref) < 1e-9 * ref


def test_methane_water_topology_from_conect_and_water_names():
    pdb = PDBFile(_data("methane_water.pdb"))
    H = Hamiltonian(_data("methane_water_coul.xml"))
    H.createPotential(pdb.topology, nonbondedMethod="PME", nonbondedCutoff=0.5, PmeCoeffMethod="gromacs",
                      PmeSpacing=0.1)
    top = pdb.topology
    assert top.getNumAtoms() == 11 and len(list(top.bonds())) == 8
    assert [a.meta["type"] for a in top.atoms()][:6] == ["C1", "H1", "H2", "H3", "H4", "OW"]
    g = H.generators["NonbondedForce"]
    assert g.K == (12, 12, 12)
    np.testing.assert_allclose(g.charges[:2], [-0.1068, 0.0267])
