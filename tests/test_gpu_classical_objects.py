"""The dmff/classical/inter.py and intra.py force objects (``dmff_b200.classical.inter`` /
``.intra``), built directly as a caller of the reference would, against the float64 oracle on a
polymer-in-water box: energies, dE/dpositions and the parameter gradients (charges through bcc,
epsilon / sigma / NBFix, bond / angle / torsion k and equilibria)."""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from helpers import rel_force_rms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def system():
    from dmff_b200.synthetic import pairs_nbond, polymer_water_box
    s = polymer_water_box(4, 20, 500, 24.6, seed=4)
    pairs = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    # nm units, as the reference's force objects are called by its generators
    return dict(s, pos_nm=s["pos"] / 10, box_nm=s["box"] / 10, rc_nm=s["rc"] / 10, kappa_nm=s["kappa"] * 10,
                sigma_nm=s["sigma"] / 10, pairs=pairs)


def _leaf(x):
    return torch.tensor(np.asarray(x, dtype=np.float64), requires_grad=True)


def _close(got, want, tol):
    got, want = np.asarray(got), np.asarray(want)
    assert np.abs(got - want).max() <= tol * max(np.abs(want).max(), 1e-12), (got.ravel()[:3], want.ravel()[:3])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_lennard_jones_force_with_nbfix(system, precision):
    from dmff_b200.classical.inter import LennardJonesForce
    s = system
    # two NBFix rows over type pairs that occur in the box, values near the mixed ones
    t = np.unique(s["types"])
    nbfix = np.array([[t[0], t[1], 0], [t[2], t[5], 1]])
    eps, sig = s["epsilon"], s["sigma_nm"]
    epsfix = [1.3 * np.sqrt(eps[a] * eps[b]) for a, b, _ in nbfix]
    sigfix = [1.05 * 0.5 * (sig[a] + sig[b]) for a, b, _ in nbfix]
    f = LennardJonesForce(0.0, s["rc_nm"], s["types"], nbfix, isPBC=True, precision=precision)
    efn = f.generate_get_energy()
    args = [_leaf(s["pos_nm"]), _leaf(s["box_nm"])]
    prm = [_leaf(eps), _leaf(sig), _leaf(epsfix), _leaf(sigfix)]
    E = efn(args[0], args[1], s["pairs"], *prm, s["mscales_lj"])
    g = torch.autograd.grad(E, args + prm)
    args_o = [_leaf(s["pos_nm"]), _leaf(s["box_nm"])]
    prm_o = [_leaf(eps), _leaf(sig), _leaf(epsfix), _leaf(sigfix)]
    Eo = R.lj_energy(args_o[0], args_o[1], s["pairs"], prm_o[0], prm_o[1], s["types"], s["mscales_lj"],
                     map_nbfix=nbfix, epsfix=prm_o[2], sigfix=prm_o[3])
    go = torch.autograd.grad(Eo, args_o + prm_o)
    tol = 1e-10 if precision == "fp64" else 1e-5
    assert abs(E.item() - Eo.item()) <= tol * abs(Eo.item())
    assert rel_force_rms(g[0].numpy(), go[0].numpy()) <= (1e-10 if precision == "fp64" else 1e-4)
    for k in range(1, 6):
        _close(g[k].numpy(), go[k].numpy(), 1e-8 if precision == "fp64" else 1e-4)
    E2, aux = efn(args[0], args[1], s["pairs"], *prm, s["mscales_lj"], aux={"tag": 1})
    assert aux == {"tag": 1} and abs(E2.item() - E.item()) <= 1e-12 * abs(E.item())


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_coulomb_pme_force_with_bcc(system, precision):
    from dmff_b200.classical.inter import CoulombPMEForce
    s = system
    rng = np.random.default_rng(3)
    n = s["n_atoms"]
    top = np.zeros((n, 4))
    top[rng.integers(0, n, 40), rng.integers(0, 4, 40)] = 1.0
    top[rng.integers(0, n, 40), rng.integers(0, 4, 40)] = -1.0
    f = CoulombPMEForce(s["rc_nm"], s["charges"], s["kappa_nm"], tuple(s["K"]), topology_matrix=top,
                        precision=precision)
    efn = f.generate_get_energy()
    pos, box, bcc = _leaf(s["pos_nm"]), _leaf(s["box_nm"]), _leaf([0.05, -0.02, 0.01, 0.03])
    E = efn(pos, box, s["pairs"], bcc, s["mscales_coul"])
    g = torch.autograd.grad(E, (pos, box, bcc))
    pos_o, box_o, bcc_o = _leaf(s["pos_nm"]), _leaf(s["box_nm"]), _leaf([0.05, -0.02, 0.01, 0.03])
    q = torch.as_tensor(s["charges"]) + (torch.as_tensor(top) @ bcc_o).reshape(-1)
    Eo = R.coulomb_pme_energy(pos_o, box_o, s["pairs"], q, s["mscales_coul"], s["kappa_nm"], s["K"])
    go = torch.autograd.grad(Eo, (pos_o, box_o, bcc_o))
    r = f._forces[(n, tuple(float(x) for x in s["mscales_coul"]))].last_result
    scale = abs(Eo.item()) if precision == "fp64" else max(abs(r.e_coul_real), abs(r.e_coul_recip),
                                                            abs(r.e_coul_self))
    assert abs(E.item() - Eo.item()) <= (1e-10 if precision == "fp64" else 1e-5) * scale
    assert rel_force_rms(g[0].numpy(), go[0].numpy()) <= (1e-9 if precision == "fp64" else 1e-4)
    _close(g[1].numpy(), go[1].numpy(), 1e-8 if precision == "fp64" else 1e-4)
    _close(g[2].numpy(), go[2].numpy(), 1e-8 if precision == "fp64" else 1e-4)


def test_reaction_field_and_no_cutoff_forces(system):
    from dmff_b200.classical.inter import CoulNoCutoffForce, CoulReactionFieldForce
    s = system
    q = s["charges"]
    rf = CoulReactionFieldForce(s["rc_nm"], q, epsilon_1=2.0, epsilon_solv=50.0, isPBC=True,
                                precision="fp64").generate_get_energy()
    nc = CoulNoCutoffForce(q, epsilon_1=1.5, precision="fp64").generate_get_energy()
    for efn, oracle in ((rf, lambda p, b: R.coul_rf_energy(p, b, s["pairs"], torch.as_tensor(q), s["mscales_coul"],
                                                          s["rc_nm"], eps_1=2.0, eps_solv=50.0)),
                        (nc, lambda p, b: R.coul_nocutoff_energy(p, s["pairs"], torch.as_tensor(q),
                                                                 s["mscales_coul"], eps_1=1.5))):
        pos = _leaf(s["pos_nm"])
        E = efn(pos, torch.tensor(s["box_nm"]), s["pairs"], s["mscales_coul"])
        (g,) = torch.autograd.grad(E, pos)
        pos_o = _leaf(s["pos_nm"])
        Eo = oracle(pos_o, torch.tensor(s["box_nm"]))
        (go,) = torch.autograd.grad(Eo, pos_o)
        assert abs(E.item() - Eo.item()) <= 1e-10 * abs(Eo.item())
        assert rel_force_rms(g.numpy(), go.numpy()) <= 1e-9


def test_bonded_force_objects(system):
    from dmff_b200.classical.intra import HarmonicAngleJaxForce, HarmonicBondJaxForce, PeriodicTorsionJaxForce
    s = system
    pos_nm = s["pos_nm"]
    b, a, t = (torch.as_tensor(s[k]).long() for k in ("bonds", "angles", "torsions"))
    # per-type parameters picked through prmidx, as the reference's generators enumerate them
    bpi, api, tpi = (torch.arange(len(x)) % m for x, m in ((b, 5), (a, 4), (t, 7)))
    kb, lb = _leaf(s["bond_prm"][:5, 0] * 100), _leaf(s["bond_prm"][:5, 1] / 10)
    ka, ta = _leaf(s["angle_prm"][:4, 0]), _leaf(s["angle_prm"][:4, 1])
    kt, pt = _leaf(s["torsion_prm"][:7, 0]), _leaf(s["torsion_prm"][:7, 1])
    order = torch.as_tensor(s["torsion_prm"][:, 2])
    cases = [
        (HarmonicBondJaxForce(b[:, 0].numpy(), b[:, 1].numpy(), bpi.numpy()), (kb, lb),
         lambda p, k, x: R.bond_energy(p, b[:, 0], b[:, 1], k[bpi], x[bpi])),
        (HarmonicAngleJaxForce(a[:, 0].numpy(), a[:, 1].numpy(), a[:, 2].numpy(), api.numpy()), (ka, ta),
         lambda p, k, x: R.angle_energy(p, a[:, 0], a[:, 1], a[:, 2], k[api], x[api])),
        (PeriodicTorsionJaxForce(*(t[:, c].numpy() for c in range(4)), tpi.numpy(), order.numpy()), (kt, pt),
         lambda p, k, x: R.torsion_energy(p, t[:, 0], t[:, 1], t[:, 2], t[:, 3], k[tpi], x[tpi], order)),
    ]
    box = torch.tensor(s["box_nm"])
    for force, prm, oracle in cases:
        pos = _leaf(pos_nm)
        E = force.get_energy(pos, box, None, *prm)
        g = torch.autograd.grad(E, (pos, *prm))
        prm_o = [_leaf(x.detach().numpy()) for x in prm]
        pos_o = _leaf(pos_nm)
        Eo = oracle(pos_o, *prm_o)
        go = torch.autograd.grad(Eo, (pos_o, *prm_o))
        assert abs(E.item() - Eo.item()) <= 1e-10 * max(1.0, abs(Eo.item()))
        for x, y in zip(g, go):
            _close(x.numpy(), y.numpy(), 1e-8)
        E2, dpos = force.get_forces(pos_nm, box, None, *[x.detach() for x in prm])
        assert abs(E2.item() - E.item()) <= 1e-12 * max(1.0, abs(E.item()))
        _close(dpos.numpy(), go[0].numpy(), 1e-8)
    # update_env swaps the term list and rebuilds the closures
    f = cases[0][0]
    f.update_env("p1idx", b[:10, 0].numpy())
    f.update_env("p2idx", b[:10, 1].numpy())
    f.update_env("prmidx", bpi[:10].numpy())
    E = f.get_energy(torch.tensor(pos_nm), box, None, kb.detach(), lb.detach())
    Eo = R.bond_energy(torch.tensor(pos_nm), b[:10, 0], b[:10, 1], kb.detach()[bpi[:10]], lb.detach()[bpi[:10]])
    assert abs(E.item() - Eo.item()) <= 1e-10 * abs(Eo.item())
