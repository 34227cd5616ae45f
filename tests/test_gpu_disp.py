"""GPU parity of dispersion PME and Tang-Toennies damping against the float64 oracle, and the
996-water goldens of examples/water_fullpol through the drop-in API."""
import json
import os

import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.engine import DispEngine
from dmff_b200.synthetic import disp_params, water_box
from tests.helpers import oracle_pairs, rel_force_rms

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(__file__), "golden")


def disp_oracle(s, d, pairs):
    pos = torch.tensor(s["pos"], requires_grad=True)
    box = torch.tensor(s["box"], requires_grad=True)
    c = torch.tensor(d["c_list"])
    ms = torch.tensor(d["mscales"])
    f = R.ADMPDispPmeForce(s["box"], s["rc"], s["ethresh"], 10)
    Elr = f.get_energy(pos, box, pairs, c, ms)
    Esr = R.pairwise_energy(R.TT_damping_qq_c6_kernel, pos, box, pairs, ms, torch.tensor(d["a"]),
                            torch.tensor(d["b"]), torch.tensor(d["q"]), c[:, 0])
    glr = torch.autograd.grad(Elr, (pos, box), retain_graph=True)
    gsr = torch.autograd.grad(Esr, (pos, box))
    return dict(Elr=Elr.item(), Esr=Esr.item(), Flr=-glr[0].numpy(), Fsr=-gsr[0].numpy(), Blr=glr[1].numpy(),
                Bsr=gsr[1].numpy())


@pytest.fixture(scope="module")
def disp_case():
    s = water_box(64, 12.4, seed=21, lmax=2, pol=False, rc=6.0)
    d = disp_params(64, seed=2)
    pr = oracle_pairs(s)
    return s, d, pr, disp_oracle(s, d, pr)


@pytest.mark.parametrize("prec,te,tf", [("fp64", 1e-10, 1e-8), ("fp32", 1e-5, 1e-4)])
def test_dispersion_pme_and_tt_match_oracle(disp_case, prec, te, tf):
    s, d, pr, ref = disp_case
    eng = DispEngine(s["n_atoms"], 10, True, s["rc"], s["kappa"], s["K"], s["cov_rows"], d["mscales"], tt=True,
                     precision=prec)
    eng.set_params(d["c_list"], d["a"], d["b"], d["q"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    res, (Flr, Fsr) = eng.compute(pos, s["box"], pairs=torch.tensor(pr, dtype=torch.int32, device="cuda"))
    assert abs(res.energy - ref["Elr"]) <= te * abs(ref["Elr"])
    assert abs(res.e_sr - ref["Esr"]) <= te * abs(ref["Esr"])
    assert rel_force_rms(Flr.cpu().numpy(), ref["Flr"]) <= tf
    assert rel_force_rms(Fsr.cpu().numpy(), ref["Fsr"]) <= tf
    assert np.abs(np.array(res.box_grad[:]).reshape(3, 3) - ref["Blr"]).max() <= tf * np.abs(ref["Blr"]).max()
    assert np.abs(np.array(res.box_grad_sr[:]).reshape(3, 3) - ref["Bsr"]).max() <= tf * np.abs(ref["Bsr"]).max()


@pytest.mark.parametrize("prec,te,tf", [("fp64", 1e-10, 1e-8), ("fp32", 1e-5, 1e-4)])
def test_dispersion_triclinic_box(prec, te, tf):
    """Dispersion PME + TT on a sheared box (K from the box diagonal, as the reference)."""
    from tests.test_gpu_edges import _sheared
    s = _sheared(water_box(64, 12.4, seed=22, lmax=2, pol=False, rc=5.0), (0.2, -0.12, 0.15))
    d = disp_params(64, seed=3)
    pr = oracle_pairs(s)
    ref = disp_oracle(s, d, pr)
    eng = DispEngine(s["n_atoms"], 10, True, s["rc"], s["kappa"], s["K"], s["cov_rows"], d["mscales"], tt=True,
                     precision=prec)
    eng.set_params(d["c_list"], d["a"], d["b"], d["q"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    res, (Flr, Fsr) = eng.compute(pos, s["box"], pairs=torch.tensor(pr, dtype=torch.int32, device="cuda"))
    assert abs(res.energy - ref["Elr"]) <= te * abs(ref["Elr"])
    assert abs(res.e_sr - ref["Esr"]) <= te * abs(ref["Esr"])
    assert rel_force_rms(Flr.cpu().numpy(), ref["Flr"]) <= tf
    assert rel_force_rms(Fsr.cpu().numpy(), ref["Fsr"]) <= tf
    assert np.abs(np.array(res.box_grad[:]).reshape(3, 3) - ref["Blr"]).max() <= tf * np.abs(ref["Blr"]).max()


def _waterbox():
    from tests.test_oracle_golden import _waterbox_topology
    return _waterbox_topology()


@pytest.mark.parametrize("force,key,rtol,kw", [
    ("ADMPDispForce", "waterbox996_disp_damp", 3e-5, {}),
    ("ADMPPmeForce", "waterbox996_es_pol", 2e-6, {"pol_solver": "cg", "cg_tol": 1e-8}),
])
def test_dropin_waterbox_996_goldens(force, key, rtol, kw):
    """examples/water_fullpol/run.py through Hamiltonian / NeighborList / potential_fn on the GPU."""
    from dmff_b200 import Hamiltonian, NeighborList
    gold = json.load(open(os.path.join(HERE, "energies.json")))[key]["value"]
    top, pos, box = _waterbox()
    H = Hamiltonian(os.path.join(HERE, "data", "waterbox_forcefield.xml"))
    pots = H.createPotential(top, nonbondedMethod="PME", nonbondedCutoff=0.6, ethresh=5e-4, has_aux=True, **kw)
    nbl = NeighborList(box, 0.6, pots.meta["cov_map"])
    nbl.allocate(pos)
    pot = pots.dmff_potentials[force]
    p = torch.tensor(pos, requires_grad=True)
    E, aux = pot(p, torch.tensor(box), nbl.pairs, H.getParameters(), {})
    assert abs(E.item() - gold) <= rtol * abs(gold)
    (g,) = torch.autograd.grad(E, p)
    assert torch.isfinite(g).all()
