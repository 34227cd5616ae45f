"""Parameter gradients on the GPU (the differentiation workload): per-atom dE/dQ_local, dE/dpol,
dE/dthole of polarizable ADMP and dE/dc (C6/C8/C10), dE_sr/d(A, B, Q) of dispersion + Tang-Toennies,
against the float64 oracle's autograd at the same converged dipoles, and per-type gradients
through the drop-in autograd path against central finite differences (h = 1e-5, FP64)."""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.engine import DispEngine
from dmff_b200.synthetic import disp_params, water_box
from helpers import make_engine, oracle_pairs, oracle_reference

pytestmark = pytest.mark.gpu


def _relmax(got, want):
    got, want = np.asarray(got), np.asarray(want)
    return float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-300))


def admp_oracle_pgrad(s, pairs):
    ref = oracle_reference(s, pairs, tol=1e-10)
    f = R.ADMPPmeForce(s["box"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], s["lmax"], s["lpol"],
                       kappa=s["kappa"], K=s["K"])
    Ql = torch.tensor(s["Q_local"], requires_grad=True)
    pos, box = torch.tensor(s["pos"]), torch.tensor(s["box"])
    ms, ps, ds = (torch.tensor(s[k]) for k in ("mscales", "pscales", "dscales"))
    if s["lpol"]:
        pol = torch.tensor(s["pol"], requires_grad=True)
        th = torch.tensor(s["thole"], requires_grad=True)
        E = f.energy_fn(pos, box, pairs, Ql, torch.tensor(ref["U"]), pol, th, ms, ps, ds)
        gQ, gp, gt = torch.autograd.grad(E, (Ql, pol, th))
        return dict(E=E.item(), Q=gQ.numpy(), pol=gp.numpy(), thole=gt.numpy())
    E = f.energy_fn(pos, box, pairs, Ql, None, None, None, ms, ps, ds)
    (gQ,) = torch.autograd.grad(E, (Ql,))
    return dict(E=E.item(), Q=gQ.numpy())


@pytest.fixture(scope="module")
def pol_case():
    s = water_box(64, 12.4, seed=22, lmax=2, pol=True, rc=6.0)
    pr = oracle_pairs(s)
    return s, pr, admp_oracle_pgrad(s, pr)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-7), ("fp32", 2e-4)])
def test_admp_param_grads_match_oracle(pol_case, prec, tol):
    s, pr, ref = pol_case
    eng = make_engine(s, precision=prec, cg_tol=1e-10 if prec == "fp64" else 1e-6)
    eng.set_param_grads(True)
    pos = torch.tensor(s["pos"], device="cuda")
    res, F, U = eng.compute(pos, s["box"], torch.tensor(pr, dtype=torch.int32, device="cuda"))
    pg = eng.param_grads()
    assert _relmax(pg["Q_local"].cpu().numpy(), ref["Q"]) < tol
    assert _relmax(pg["pol"].cpu().numpy(), ref["pol"]) < tol
    assert _relmax(pg["thole"].cpu().numpy(), ref["thole"]) < tol
    # switching the adjoints off leaves energy and forces as they were
    eng.set_param_grads(False)
    res2, F2, _ = eng.compute(pos, s["box"], torch.tensor(pr, dtype=torch.int32, device="cuda"))
    assert abs(res2.energy - res.energy) <= 1e-6 * abs(res.energy)


def test_admp_nonpol_multipole_grads_match_oracle():
    s = water_box(64, 12.4, seed=23, lmax=2, pol=False, rc=6.0)
    pr = oracle_pairs(s)
    ref = admp_oracle_pgrad(s, pr)
    eng = make_engine(s, precision="fp64")
    eng.set_param_grads(True)
    eng.compute(torch.tensor(s["pos"], device="cuda"), s["box"], torch.tensor(pr, dtype=torch.int32, device="cuda"))
    assert _relmax(eng.param_grads()["Q_local"].cpu().numpy(), ref["Q"]) < 1e-8


def test_admp_per_type_grads_vs_finite_differences():
    """dE/d(per-type Q_local, pol, thole) through ADMPPmeForce.get_energy + torch autograd against
    central differences of the FP64 engine energy (CG to 1e-12)."""
    from dmff_b200.admp.pme import ADMPPmeForce
    s = water_box(27, 9.3, seed=24, lmax=2, pol=True, rc=4.6)
    types = torch.as_tensor(s["types"])
    f = ADMPPmeForce(s["box"], s["types"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], 2, True, True,
                     cov_rows=s["cov_rows"], precision="fp64", cg_tol=1e-12, max_iter=2000)
    pr = oracle_pairs(s)
    Qt = torch.tensor(s["Q_type"], requires_grad=True)
    pt = torch.tensor([1.0, 0.5], dtype=torch.float64, requires_grad=True)
    tt = torch.tensor([0.33, 0.33], dtype=torch.float64, requires_grad=True)
    ms, ps, ds = (torch.tensor(s[k]) for k in ("mscales", "pscales", "dscales"))
    pos, box = torch.tensor(s["pos"]), torch.tensor(s["box"])

    def energy(Q, p, t):
        return f.get_energy(pos, box, pr, Q[types], p[types], t[types], ms, ps, ds,
                            U_init=torch.zeros((s["n_atoms"], 3)))

    E = energy(Qt, pt, tt)
    gQ, gp, gt = torch.autograd.grad(E, (Qt, pt, tt))
    h = 1e-5
    with torch.no_grad():
        for tensor, grad, idx in [(Qt, gQ, (0, 0)), (Qt, gQ, (0, 2)), (Qt, gQ, (1, 5)), (pt, gp, (0,)), (pt, gp, (1,)),
                                  (tt, gt, (0,))]:
            base = tensor[idx].item()
            args = [Qt.detach().clone(), pt.detach().clone(), tt.detach().clone()]
            k = 0 if tensor is Qt else (1 if tensor is pt else 2)
            args[k][idx] = base + h
            ep = energy(*args).item()
            args[k][idx] = base - h
            em = energy(*args).item()
            fd = (ep - em) / (2 * h)
            assert abs(fd - grad[idx].item()) <= 1e-5 * max(abs(fd), 1.0), (idx, fd, grad[idx].item())


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-8), ("fp32", 1e-4)])
def test_dispersion_param_grads_match_oracle(prec, tol):
    s = water_box(64, 12.4, seed=21, lmax=2, pol=False, rc=6.0)
    d = disp_params(64, seed=2)
    pr = oracle_pairs(s)
    pos, box = torch.tensor(s["pos"]), torch.tensor(s["box"])
    c = torch.tensor(d["c_list"], requires_grad=True)
    a, b, q = (torch.tensor(d[k], requires_grad=True) for k in ("a", "b", "q"))
    ms = torch.tensor(d["mscales"])
    f = R.ADMPDispPmeForce(s["box"], s["rc"], s["ethresh"], 10)
    Elr = f.get_energy(pos, box, pr, c, ms)
    Esr = R.pairwise_energy(R.TT_damping_qq_c6_kernel, pos, box, pr, ms, a, b, q, c[:, 0])
    (gc_lr,) = torch.autograd.grad(Elr, (c,))
    gsr = torch.autograd.grad(Esr, (a, b, q, c))
    eng = DispEngine(s["n_atoms"], 10, True, s["rc"], s["kappa"], s["K"], s["cov_rows"], d["mscales"], tt=True,
                     precision=prec)
    eng.set_params(d["c_list"], d["a"], d["b"], d["q"])
    eng.set_param_grads(True)
    eng.compute(torch.tensor(s["pos"], device="cuda"), s["box"], pairs=torch.tensor(pr, dtype=torch.int32, device="cuda"))
    pg = eng.param_grads()
    assert _relmax(pg["c"].cpu().numpy(), gc_lr.numpy()) < tol
    assert _relmax(pg["a"].cpu().numpy(), gsr[0].numpy()) < tol
    assert _relmax(pg["b"].cpu().numpy(), gsr[1].numpy()) < tol
    assert _relmax(pg["q"].cpu().numpy(), gsr[2].numpy()) < tol
    assert _relmax(pg["c6"].cpu().numpy(), gsr[3][:, 0].numpy()) < tol
