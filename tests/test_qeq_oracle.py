"""The charge-equilibration oracle (oracle/qeq_ref.py, a direct solve of the stationary point of
dmff/admp/qeq.py's E_full) against the reference's golden energies (tests/test_admp/test_qeq.py):
the 144-atom slab with one residue constraint, and the 147-atom slab with two explicit
constraint groups from zero initial charges.  Inputs are read as the reference's test reads
them (residue templates for charges and types, a cell-list neighbour set at rc 0.6 nm)."""
import json
import os

import numpy as np
import pytest
import torch

import oracle.admp_ref as R
import oracle.qeq_ref as Q
from dmff_b200 import Hamiltonian, PDBFile

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "golden", "data")
GOLD = json.load(open(os.path.join(HERE, "golden", "energies.json")))


def qeq_case(key, zero_charges=False):
    """(gold, Hamiltonian, topology, pos nm, box nm, pairs with nbond, per-atom type index)."""
    g = GOLD[key]
    pdb = PDBFile(os.path.join(DATA, g["pdb"]))
    top = pdb.topology
    H = Hamiltonian(os.path.join(DATA, g["xml"]))
    # types and charges by atom order from the XML's residue templates, as the reference's test
    # assigns them (its water residue is named differently in the PDB and the XML)
    parts = [p for r in H.ffinfo["Residues"] for p in r["particles"]]
    for a, p in zip(top.atoms(), parts):
        a.meta["type"] = p["type"]
        a.meta["charge"] = 0.0 if zero_charges else float(p["charge"])
    pos = np.asarray(pdb.positions, dtype=np.float64)
    box = np.asarray(top.getPeriodicBoxVectors(), dtype=np.float64)
    cov = top.buildCovMat()
    pairs = R.brute_force_pairs(pos, box, g["rc_nm"], lambda i, j: int(cov.lookup(i, j)))
    return g, H, top, pos, box, pairs


def oracle_force(g, H, top, box, **kw):
    gen = H.generators["ADMPQeqForce"]
    kappa, K1, K2, K3 = R.setup_ewald_parameters(g["rc_nm"], g["ethresh"], box)
    atoms = list(top.atoms())
    init_q = np.array([float(a.meta["charge"]) for a in atoms])
    if "groups" in g:
        const_list = [list(range(a, b)) for a, b in g["groups"]]
        const_vals = g["group_vals"]
    else:
        const_list = [[a.index for a in r.atoms()] for r in top.residues()]
        const_vals = [float(init_q[c].sum()) for c in const_list]
    opts = dict(damp_mod=gen.damp_mod, neutral_flag=True, slab_flag=True, constQ=True, pbc_flag=True)
    opts.update(kw)
    f = Q.ADMPQeqForce(init_q, g["rc_nm"], kappa, (K1, K2, K3), const_list=const_list, const_vals=const_vals,
                       **opts)
    idx = {k: i for i, k in enumerate(gen.atom_keys)}
    m = torch.as_tensor([idx[a.meta[gen.key_type]] for a in atoms])
    p = H.paramset["ADMPQeqForce"]
    mscales = [0.0, 0.0, gen.coulomb14scale, 1.0, 1.0, 1.0]
    return f, p["eta"][m], p["chi"][m], p["J"][m], mscales


@pytest.mark.parametrize("key,zero", [("qeq", False), ("qeq2", True)])
def test_qeq_oracle_golden(key, zero):
    g, H, top, pos, box, pairs = qeq_case(key, zero)
    f, eta, chi, J, ms = oracle_force(g, H, top, box)
    E, q, lam = f.get_energy(torch.tensor(pos), torch.tensor(box), pairs, ms, eta, chi, J)
    np.testing.assert_almost_equal(E.item(), g["value"], decimal=g["decimal"])
    # the solution satisfies the group constraints
    for c, v in zip(f.groups.tolist(), f.const_vals.tolist()):
        idx = [i for i in c if i < len(q)]
        assert abs(float(q[idx].sum()) - v) < 1e-9
