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


def classical_oracle(H, pos_nm, box_nm, pairs, names=None):
    """Float64 oracle energy of a Hamiltonian's classical generators (dmff/classical/*.py formulas),
    using the term lists / maps the generators enumerated in createPotential.  Returns
    (E, positions tensor, box tensor) with autograd attached."""
    pos = torch.tensor(np.asarray(pos_nm, dtype=np.float64), requires_grad=True)
    box = torch.tensor(np.asarray(box_nm, dtype=np.float64), requires_grad=True)
    E = torch.zeros((), dtype=torch.float64)
    for name, g in H.generators.items():
        if names is not None and name not in names:
            continue
        P = H.paramset[name]
        if name == "HarmonicBondForce" and len(g.bond_idx):
            i, pi = torch.as_tensor(g.bond_idx).long(), g.bond_prm_idx
            E = E + R.bond_energy(pos, i[:, 0], i[:, 1], P["k"][pi], P["length"][pi])
        elif name == "HarmonicAngleForce" and len(g.angle_idx):
            i, pi = torch.as_tensor(g.angle_idx).long(), g.angle_prm_idx
            E = E + R.angle_energy(pos, i[:, 0], i[:, 1], i[:, 2], P["k"][pi], P["angle"][pi])
        elif name == "PeriodicTorsionForce" and getattr(g, "torsion_idx", np.zeros((0, 4))).shape[0]:
            i = torch.as_tensor(g.torsion_idx).long()
            k = torch.cat([P["proper_k"][g.sel_proper], P["improper_k"][g.sel_improper]])
            ph = torch.cat([P["proper_phase"][g.sel_proper], P["improper_phase"][g.sel_improper]])
            E = E + R.torsion_energy(pos, i[:, 0], i[:, 1], i[:, 2], i[:, 3], k, ph, g.torsion_per)
        elif name in ("NonbondedForce", "CoulombForce"):
            q = torch.as_tensor(np.asarray(g.charges, dtype=np.float64))
            if g.coul_mode == "pme":
                E = E + R.coulomb_pme_energy(pos, box, pairs, q, g.mscales_coul, g.kappa_nm, g.K)
            elif g.coul_mode == "rf":
                E = E + R.coul_rf_energy(pos, box, pairs, q, g.mscales_coul, g.r_cut, pbc=g.pbc)
            elif g.coul_mode == "nocutoff":
                E = E + R.coul_nocutoff_energy(pos, pairs, q, g.mscales_coul)
            if name == "NonbondedForce":
                E = E + R.lj_energy(pos, box, pairs, P["epsilon"], P["sigma"], g.map_prm, g.mscales_lj, pbc=g.pbc)
                if g.disp_corr is not None:
                    E = E + R.lj_dispersion_correction(box, P["epsilon"], P["sigma"], g.map_prm,
                                                       g.disp_corr.count, g.r_cut)
        elif name == "LennardJonesForce":
            E = E + R.lj_energy(pos, box, pairs, P["epsilon"], P["sigma"], g.map_prm, g.mscales_lj, pbc=g.pbc,
                                map_nbfix=g.nbfix, epsfix=P["epsilon_nbfix"], sigfix=P["sigma_nbfix"])
    return E, pos, box


def oracle_force_loss_grads(sysd, pairs, w, tol=1e-12):
    """Exact derivatives of L = <w, dE/dpos> with respect to positions, Q_local, pol and thole, the
    converged induced dipoles following, by implicit differentiation through the float64 oracle
    (double autograd): with E_U(z, U*) = 0 and A = d2E/dU2,
        dL/dz = d/dz <w, E_x>|_U - d/dz <lam, E_U>|_U,   A lam = d/dU <w, E_x>,
    lam solved by CG on exact A-products (E is quadratic in U)."""
    import oracle.admp_ref as R
    f = R.ADMPPmeForce(sysd["box"], sysd["axis_types"], sysd["axis_indices"], sysd["rc"], sysd["ethresh"],
                       sysd["lmax"], True, kappa=sysd["kappa"], K=sysd["K"])
    pos = torch.tensor(sysd["pos"], dtype=torch.float64, requires_grad=True)
    box = torch.tensor(sysd["box"], dtype=torch.float64)
    Q = torch.tensor(sysd["Q_local"], dtype=torch.float64, requires_grad=True)
    pol = torch.tensor(sysd["pol"], dtype=torch.float64, requires_grad=True)
    th = torch.tensor(sysd["thole"], dtype=torch.float64, requires_grad=True)
    sc = tuple(torch.tensor(sysd[k]) for k in ("mscales", "pscales", "dscales"))
    Ustar, ok, _ = f.solve_Uind_cg(pos.detach(), box, pairs, Q.detach(), pol.detach(), th.detach(), *sc, tol=tol)
    assert ok
    U = Ustar.detach().clone().requires_grad_(True)
    E = f.energy_fn(pos, box, pairs, Q, U, pol, th, *sc)
    gx, gU = torch.autograd.grad(E, (pos, U), create_graph=True)
    w = torch.as_tensor(w, dtype=torch.float64)
    Lx = (w * gx).sum()
    (rhs,) = torch.autograd.grad(Lx, U, retain_graph=True)

    def Ap(p):
        (r,) = torch.autograd.grad((gU * p).sum(), U, retain_graph=True)
        return r

    Minv = (torch.clamp(pol.detach(), min=1e-8) / R.DIELECTRIC)[:, None]
    lam = torch.zeros_like(rhs)
    r = rhs.clone()
    z = Minv * r
    p = z.clone()
    rz = (r * z).sum()
    for _ in range(500):
        if float(torch.sqrt((r * r).mean())) < 1e-13 * max(float(torch.sqrt((rhs * rhs).mean())), 1e-300):
            break
        q = Ap(p)
        alpha = rz / (p * q).sum()
        lam = lam + alpha * p
        r = r - alpha * q
        z = Minv * r
        rz_new = (r * z).sum()
        p = z + (rz_new / rz) * p
        rz = rz_new
    total = Lx - (lam.detach() * gU).sum()
    gpos, gQ, gpol, gth = torch.autograd.grad(total, (pos, Q, pol, th))
    return dict(L=float(Lx.detach()), pos=gpos.numpy(), Q=gQ.numpy(), pol=gpol.numpy(), thole=gth.numpy())
