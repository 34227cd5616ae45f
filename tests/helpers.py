"""Shared test helpers: oracle references for synthetic systems and comparison metrics."""
import numpy as np
import torch

import oracle.admp_ref as R
from dmff_b200.synthetic import pairs_nbond


def oracle_pairs(sysd, rc=None):
    cov = sysd["cov_rows"]
    n = sysd["n_atoms"]
    pr = R.brute_force_pairs(sysd["pos"], sysd["box"], rc if rc is not None else sysd["rc"])
    pr[:, 2] = pairs_nbond(pr, cov, n)
    return pr


def oracle_reference(sysd, pairs, solver="cg", tol=1e-8, steps_pol=None, want_box=True):
    """Energy, forces (-dE/dpos), dE/dbox and dipoles from the float64 oracle."""
    pos = torch.tensor(sysd["pos"], dtype=torch.float64, requires_grad=True)
    box = torch.tensor(sysd["box"], dtype=torch.float64, requires_grad=True)
    f = R.ADMPPmeForce(sysd["box"], sysd["axis_types"], sysd["axis_indices"], sysd["rc"], sysd["ethresh"],
                       sysd["lmax"], sysd["lpol"], lpme=sysd.get("lpme", True), steps_pol=steps_pol,
                       kappa=sysd["kappa"], K=sysd["K"])
    Ql = torch.tensor(sysd["Q_local"], dtype=torch.float64)
    ms = torch.tensor(sysd["mscales"])
    if sysd["lpol"]:
        E, U, flag, n = f.get_energy(pos, box, pairs, Ql, torch.tensor(sysd["pol"]), torch.tensor(sysd["thole"]),
                                     ms, torch.tensor(sysd["pscales"]), torch.tensor(sysd["dscales"]),
                                     solver=solver, tol=tol)
    else:
        E, U, flag, n = f.get_energy(pos, box, pairs, Ql, mScales=ms)
    gp, gb = torch.autograd.grad(E, (pos, box))
    return dict(E=E.item(), F=-gp.numpy(), box_grad=gb.numpy(), U=None if U is None else U.numpy(), n_iter=n)


def rel_force_rms(F, Fref):
    return float(np.sqrt(np.mean((F - Fref) ** 2)) / np.sqrt(np.mean(Fref ** 2)))


def make_engine(sysd, precision="fp32", solver="cg", cg_tol=1e-8, steps_pol=None, lpme=True):
    from dmff_b200.engine import AdmpEngine
    eng = AdmpEngine(sysd["n_atoms"], sysd["lmax"], sysd["lpol"], lpme, sysd["rc"], sysd["kappa"], sysd["K"],
                     sysd["axis_types"], sysd["axis_indices"], sysd["cov_rows"], sysd["mscales"],
                     sysd["pscales"], sysd["dscales"], precision=precision, solver=solver, cg_tol=cg_tol,
                     steps_pol=steps_pol)
    eng.set_params(sysd["Q_local"], sysd.get("pol"), sysd.get("thole"))
    return eng
