"""Classical terms on the GPU (LJ + Coulomb PME / reaction field / 1/r, bonds, angles, torsions)
against the float64 oracle and the reference's classical goldens, through the drop-in generator
API and through the engine directly."""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from helpers import classical_oracle, rel_force_rms
from test_classical_oracle import GOLD, NAMES, golden_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("c", GOLD, ids=[f"{c['test']}-{c['xml']}" for c in GOLD])
def test_classical_goldens_drop_in(c, precision):
    H, pdb, box, pairs, pot = golden_case(c, with_potential=True, precision=precision)
    names = NAMES.get(c["test"])
    efunc = pot.getPotentialFunc(names=names or ())
    pos = torch.tensor(pdb.positions, requires_grad=True)
    E = efunc(pos, torch.tensor(box), pairs if len(pairs) else np.array([[]], dtype=int), H.paramset)
    E = torch.as_tensor(E).reshape(())
    if "atol" in c:
        assert abs(E.item() - c["value"]) < c["atol"]
    else:
        np.testing.assert_almost_equal(E.item(), c["value"], decimal=c["decimal"])
    Eo, po, _ = classical_oracle(H, pdb.positions, box, pairs, names=names)
    # FP32: relative to the largest energy term (for tiny PME boxes the total is a residual of
    # real, reciprocal and self terms a few hundred times larger)
    scale = max(1.0, abs(Eo.item()))
    for g in H.generators.values():
        r = getattr(getattr(g, "pme_force", None), "last_result", None)
        if r is not None:
            scale = max(scale, abs(r.e_coul_real), abs(r.e_coul_recip), abs(r.e_coul_self))
    tol = 1e-9 if precision == "fp64" else 1e-6
    assert abs(E.item() - Eo.item()) <= tol * scale
    if E.requires_grad:
        (g,) = torch.autograd.grad(E, pos)
        (go,) = torch.autograd.grad(Eo, po)
        assert rel_force_rms(g.numpy(), go.numpy()) < (1e-9 if precision == "fp64" else 1e-5)


def _synthetic(n_chains=4, n_beads=20, n_waters=500, L=24.6):
    from dmff_b200.synthetic import polymer_water_box
    return polymer_water_box(n_chains, n_beads, n_waters, L, seed=4)


def _oracle_synth(s, pairs, coulomb="pme"):
    pos = torch.tensor(s["pos"], requires_grad=True)
    box = torch.tensor(s["box"], requires_grad=True)
    q = torch.tensor(s["charges"], requires_grad=True)
    sig = torch.tensor(s["sigma"], requires_grad=True)
    eps = torch.tensor(s["epsilon"], requires_grad=True)
    bp = torch.tensor(s["bond_prm"], requires_grad=True)
    ap = torch.tensor(s["angle_prm"], requires_grad=True)
    tp = torch.tensor(s["torsion_prm"], requires_grad=True)
    if coulomb == "pme":
        Ec = R.coulomb_pme_energy(pos / 10, box / 10, pairs, q, s["mscales_coul"], s["kappa"] * 10, s["K"])
    else:
        Ec = R.coul_rf_energy(pos / 10, box / 10, pairs, q, s["mscales_coul"], s["rc"] / 10)
    El = R.lj_energy(pos, box, pairs, eps, sig, s["types"], s["mscales_lj"])
    b, a, t = (torch.as_tensor(s[k]).long() for k in ("bonds", "angles", "torsions"))
    Eb = R.bond_energy(pos, b[:, 0], b[:, 1], bp[:, 0], bp[:, 1])
    Ea = R.angle_energy(pos, a[:, 0], a[:, 1], a[:, 2], ap[:, 0], ap[:, 1])
    Et = R.torsion_energy(pos, t[:, 0], t[:, 1], t[:, 2], t[:, 3], tp[:, 0], tp[:, 1], tp[:, 2].detach())
    E = Ec + El + Eb + Ea + Et
    grads = torch.autograd.grad(E, (pos, box, q, sig, eps, bp, ap, tp))
    return dict(E=E.item(), Ec=Ec.item(), El=El.item(), Eb=Eb.item(), Ea=Ea.item(), Et=Et.item(),
                F=-grads[0].numpy(), box_grad=grads[1].numpy(), dq=grads[2].numpy(), dsig=grads[3].numpy(),
                deps=grads[4].numpy(), dbond=grads[5].numpy(), dangle=grads[6].numpy(), dtors=grads[7].numpy())


def _engine(s, precision, coulomb="pme"):
    from dmff_b200.engine import ClassicalEngine
    eng = ClassicalEngine(s["n_atoms"], n_types=len(s["sigma"]), coulomb=coulomb, pbc=True, rc=s["rc"],
                          kappa=s["kappa"], K=s["K"], cov_rows=s["cov_rows"], mscales_coul=s["mscales_coul"],
                          mscales_lj=s["mscales_lj"], precision=precision)
    eng.set_params(s["charges"], s["types"], s["sigma_tt"], s["eps_tt"])
    eng.set_terms("bond", s["bonds"], s["bond_prm"])
    eng.set_terms("angle", s["angles"], s["angle_prm"])
    eng.set_terms("torsion", s["torsions"], s["torsion_prm"])
    return eng


@pytest.mark.parametrize("coulomb", ["pme", "rf"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_polymer_water_parity(precision, coulomb):
    s = _synthetic()
    cov = s["cov_rows"]
    from dmff_b200.synthetic import pairs_nbond
    pairs = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pairs[:, 2] = pairs_nbond(pairs, cov, s["n_atoms"])
    ref = _oracle_synth(s, pairs, coulomb)
    eng = _engine(s, precision, coulomb)
    pos = torch.tensor(s["pos"], device="cuda")
    res, F = eng.compute(pos, s["box"], torch.tensor(pairs, dtype=torch.int32, device="cuda"))
    tol_e = 1e-10 if precision == "fp64" else 1e-5
    assert abs(res.energy - ref["E"]) <= tol_e * abs(ref["E"])
    assert abs(res.e_bond - ref["Eb"]) <= 1e-10 * abs(ref["Eb"])
    assert abs(res.e_angle - ref["Ea"]) <= 1e-10 * abs(ref["Ea"])
    assert abs(res.e_torsion - ref["Et"]) <= 1e-10 * max(1.0, abs(ref["Et"]))
    assert abs(res.e_lj - ref["El"]) <= tol_e * abs(ref["El"])
    assert rel_force_rms(F.cpu().numpy(), ref["F"]) < (1e-10 if precision == "fp64" else 1e-4)
    bg = np.array(res.box_grad).reshape(3, 3)
    assert np.abs(bg - ref["box_grad"]).max() <= (1e-8 if precision == "fp64" else 1e-4) * np.abs(ref["box_grad"]).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_polymer_water_triclinic_box(precision):
    """The same system on a sheared (reduced, OpenMM-style) box: all coordinates mapped linearly,
    so bonds and images stay consistent; engine-built neighbour list and given rows both."""
    s = _synthetic()
    L = s["box"][0, 0]
    box = np.array([[L, 0.0, 0.0], [0.1 * L, L, 0.0], [-0.08 * L, 0.06 * L, L]])
    s = dict(s, pos=(s["pos"] / L) @ box, box=box)
    from dmff_b200.synthetic import pairs_nbond
    pairs = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    ref = _oracle_synth(s, pairs, "pme")
    eng = _engine(s, precision, "pme")
    pos = torch.tensor(s["pos"], device="cuda")
    res, F = eng.compute(pos, s["box"], torch.tensor(pairs, dtype=torch.int32, device="cuda"))
    tol_e = 1e-10 if precision == "fp64" else 1e-5
    assert abs(res.energy - ref["E"]) <= tol_e * abs(ref["E"])
    assert rel_force_rms(F.cpu().numpy(), ref["F"]) < (1e-10 if precision == "fp64" else 1e-4)
    bg = np.array(res.box_grad).reshape(3, 3)
    assert np.abs(bg - ref["box_grad"]).max() <= (1e-8 if precision == "fp64" else 1e-4) * np.abs(ref["box_grad"]).max()
    r2, _ = eng.compute(pos, s["box"], None)
    assert r2.n_pairs == len(pairs)


def test_polymer_water_internal_neighbour_list_matches():
    s = _synthetic()
    eng = _engine(s, "fp64")
    pos = torch.tensor(s["pos"], device="cuda")
    from dmff_b200.synthetic import pairs_nbond
    pairs = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    r1, _ = eng.compute(pos, s["box"], torch.tensor(pairs, dtype=torch.int32, device="cuda"))
    r2, _ = eng.compute(pos, s["box"], None)
    assert r2.n_pairs == len(pairs)
    assert abs(r1.energy - r2.energy) <= 1e-9 * abs(r1.energy)


def test_polymer_water_parameter_gradients():
    s = _synthetic()
    from dmff_b200.synthetic import pairs_nbond
    from dmff_b200.classical.forces import ClassicalForce
    from dmff_b200.generators.classical import _lb_tables
    pairs = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    ref = _oracle_synth(s, pairs)
    f = ClassicalForce(s["n_atoms"], n_types=len(s["sigma"]), coulomb="pme", rc=s["rc"], kappa=s["kappa"], K=s["K"],
                       cov_rows=s["cov_rows"], mscales_coul=s["mscales_coul"], mscales_lj=s["mscales_lj"],
                       precision="fp64")
    q = torch.tensor(s["charges"], requires_grad=True)
    sig = torch.tensor(s["sigma"], requires_grad=True)
    eps = torch.tensor(s["epsilon"], requires_grad=True)
    bp = torch.tensor(s["bond_prm"], requires_grad=True)
    ap = torch.tensor(s["angle_prm"], requires_grad=True)
    tp = torch.tensor(s["torsion_prm"], requires_grad=True)
    pos = torch.tensor(s["pos"], requires_grad=True)
    box = torch.tensor(s["box"], requires_grad=True)
    sig_tt, eps_tt = _lb_tables(sig, eps)
    E = f.energy(pos, box, pairs, charges=q, atom_type=s["types"], sigma_tt=sig_tt, eps_tt=eps_tt,
                 bond_idx=s["bonds"], bond_prm=bp, angle_idx=s["angles"], angle_prm=ap, torsion_idx=s["torsions"],
                 torsion_prm=tp)
    g = torch.autograd.grad(E, (pos, box, q, sig, eps, bp, ap, tp))
    assert abs(E.item() - ref["E"]) <= 1e-10 * abs(ref["E"])
    for got, want in [(g[0], -ref["F"]), (g[1], ref["box_grad"]), (g[2], ref["dq"]), (g[3], ref["dsig"]),
                      (g[4], ref["deps"]), (g[5], ref["dbond"]), (g[6], ref["dangle"]), (g[7][:, :2], ref["dtors"][:, :2])]:
        got = got.detach().numpy()
        assert np.abs(got - want).max() <= 1e-7 * max(np.abs(want).max(), 1e-12), (got.ravel()[:4], want.ravel()[:4])
