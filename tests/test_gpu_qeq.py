"""ADMPQeqForce on the GPU engines (dmff_b200.admp.qeq: MINRES on the constraint null space with
charge-only PME and Gaussian-charge pair evaluations as the matrix-vector product) against the
float64 oracle's direct solve and the reference's golden energies (tests/test_admp/test_qeq.py):
energies, equilibrated charges and multipliers, position / box / parameter gradients, the
drop-in generator with residue constraints and with explicit groups through ``aux``, the
constant-potential form, DampMod 2 and the non-periodic (no cutoff) Coulomb form."""
import numpy as np
import pytest
import torch

import oracle.qeq_ref as Q
from dmff_b200.admp.qeq import ADMPQeqForce
from tests.test_qeq_oracle import oracle_force, qeq_case

pytestmark = pytest.mark.gpu


def _ours(g, H, top, box, f_oracle, **over):
    """The GPU force built from the same inputs as the oracle's."""
    kw = dict(damp_mod=f_oracle.damp_mod, neutral_flag=True, slab_flag=f_oracle.slab_flag, constQ=True,
              pbc_flag=f_oracle.pbc_flag)
    kw.update(over)
    const_vals = f_oracle.const_vals.numpy()
    groups = [[i for i in row if i < f_oracle.init_q.shape[0]] for row in f_oracle.groups.tolist()]
    return ADMPQeqForce(f_oracle.init_q.numpy(), g["rc_nm"], f_oracle.kappa, f_oracle._K, const_list=groups,
                        const_vals=const_vals, **kw)


def _grads(E, xs):
    return torch.autograd.grad(E, xs)


@pytest.mark.parametrize("key,zero", [("qeq", False), ("qeq2", True)])
def test_qeq_matches_oracle_and_golden(key, zero):
    g, H, top, pos, box, pairs = qeq_case(key, zero)
    fo, eta, chi, J, ms = oracle_force(g, H, top, box)
    pos_t = torch.tensor(pos, requires_grad=True)
    box_t = torch.tensor(box, requires_grad=True)
    params = [t.clone().requires_grad_(True) for t in (eta, chi, J)]
    Eo, qo, lo = fo.get_energy(pos_t, box_t, pairs, ms, *params)
    go = _grads(Eo, [pos_t, box_t] + params)
    f = _ours(g, H, top, box, fo)
    energy = f.generate_get_energy()
    pos_g = torch.tensor(pos, device="cuda", requires_grad=True)
    box_g = torch.tensor(box, device="cuda", requires_grad=True)
    pg = [t.detach().clone().cuda().requires_grad_(True) for t in (eta, chi, J)]
    f.has_aux = True
    E, aux = energy(pos_g, box_g, pairs, ms, *pg)
    np.testing.assert_almost_equal(E.item(), g["value"], decimal=g["decimal"])
    assert abs(E.item() - Eo.item()) <= 1e-8 * max(1.0, abs(Eo.item())), (E.item(), Eo.item())
    assert (aux["q"].cpu() - qo).abs().max().item() <= 1e-6 * max(1.0, qo.abs().max().item())
    if len(lo):
        assert (aux["lagmt"].cpu() - lo).abs().max().item() <= 1e-6 * max(1.0, lo.abs().max().item())
    gg = _grads(E, [pos_g, box_g] + pg)
    for name, a, b in zip(["pos", "box", "eta", "chi", "J"], gg, go):
        a = a.detach().cpu()
        # the box gradient is a small sum of large cancelling terms (the reciprocal virial): its
        # error is bounded by the energy scale
        atol = 1e-9 * max(1.0, abs(Eo.item())) if name == "box" else 0.0
        assert (a - b).abs().max() <= atol + 1e-5 * max(b.abs().max().item(), 1e-12), (name, (a - b).abs().max(),
                                                                                        b.abs().max())


def test_qeq_generator_drop_in():
    """Hamiltonian.createPotential(..., PME, ethresh=1e-3, neutral, slab, constQ) on qeq.pdb."""
    g, H, top, pos, box, pairs = qeq_case("qeq")
    pot = H.createPotential(top, nonbondedCutoff=g["rc_nm"], nonbondedMethod="PME", ethresh=g["ethresh"],
                            neutral=True, slab=True, constQ=True)
    efunc = pot.getPotentialFunc()
    E = efunc(torch.tensor(pos, device="cuda"), torch.tensor(box, device="cuda"), pairs, H.paramset.parameters)
    np.testing.assert_almost_equal(float(E), g["value"], decimal=g["decimal"])


@pytest.mark.parametrize("variant", ["constP", "damp2", "nocutoff"])
def test_qeq_variants_match_oracle(variant):
    g, H, top, pos, box, pairs = qeq_case("qeq")
    kw = {}
    if variant == "constP":
        kw = dict(constQ=False)
    elif variant == "damp2":
        kw = dict(damp_mod=2)
    else:
        kw = dict(pbc_flag=False, slab_flag=False)
    fo, eta, chi, J, ms = oracle_force(g, H, top, box, **kw)
    pos_t = torch.tensor(pos, requires_grad=True)
    Eo, qo, _ = fo.get_energy(pos_t, torch.tensor(box), pairs, ms, eta, chi, J)
    (gpo,) = torch.autograd.grad(Eo, [pos_t])
    f = _ours(g, H, top, box, fo, **kw)
    pos_g = torch.tensor(pos, device="cuda", requires_grad=True)
    f.has_aux = True
    E, aux = f.generate_get_energy()(pos_g, torch.tensor(box, device="cuda"), pairs, ms, eta.cuda(), chi.cuda(),
                                     J.cuda())
    assert abs(E.item() - Eo.item()) <= 1e-8 * max(1.0, abs(Eo.item())), (variant, E.item(), Eo.item())
    assert (aux["q"].cpu() - qo).abs().max().item() <= 1e-6 * max(1.0, qo.abs().max().item())
    (gp,) = torch.autograd.grad(E, [pos_g])
    # the charges agree to ~1e-7 relative (iterative vs direct solve); the gradient is linear in
    # them, summed over every pair
    assert (gp.cpu() - gpo).abs().max() <= 1e-5 * gpo.abs().max()
