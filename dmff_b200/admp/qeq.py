"""Charge equilibration, ADMPQeqForce, with the names and call of dmff/admp/qeq.py.

``ADMPQeqForce(init_q, r_cut, kappa, K, damp_mod, const_list, const_vals, neutral_flag,
slab_flag, constQ, pbc_flag, has_aux).generate_get_energy()`` returns
``get_energy(positions, box, pairs, mscales, eta, chi, J, aux=None)`` (nm, kJ/mol), the energy
E_full(q*, lambda*) at the charges q* and multipliers lambda* where E_full is stationary
(qeq.py:310-405):

    E_full = E_constraint + E_sr + E_site + E_coul [+ E_corr]

E_coul is the charge-only PME energy (qeq.py:275-299; point charges over the pair rows with
mscales[nbond - 1] without PBC), E_sr the Gaussian-charge short range (DampMod 2 / 3,
qeq.py:85-112), E_site the on-site chi q + J q^2 (qeq.py:120-129), E_corr the slab correction
(qeq.py:132-152) and E_constraint the group-charge constraint (constQ, qeq.py:66-69) or the
constant-potential term (qeq.py:72-75).

Every term is quadratic in q, so the reference's root finding (MINPACK hybr on the gradient,
qeq.py:375-381) is the linear saddle-point problem  A q + g + C^T lambda = 0,  C q = c  (constQ;
no constraint rows for the constant-potential form).  Here it is solved matrix-free on the GPU:
A v is one charge-only PME evaluation of the ADMP engine (the charge gradient of E_coul at
charges v; E_coul has no linear part) plus one evaluation of the engine's short-range pair
kernel (its q adjoint for the QEq kinds), plus the diagonal self and site terms and the slab
term.  A may be indefinite (negative J), so the solver is MINRES (Paige and Saunders, 1975) on
the constraint null space: the start satisfies C q = c, and every preconditioned residual is
projected back onto C z = 0 with the diagonal metric M = |self + site diagonal| (the constraint
groups are disjoint, which makes the projection a per-group weighted mean removal).  lambda is
read off the converged gradient.  The energy and its gradients (positions, box, chi, J, eta)
are evaluated at (q*, lambda*) held fixed, as the reference's stop_gradient does (qeq.py:395).
"""
import math

import numpy as np
import torch

from .. import _lib as L
from ..engine import AdmpEngine, PairwiseEngine

DIELECTRIC = 1389.35455846


def _f64(x, device):
    return torch.as_tensor(x, dtype=torch.float64).to(device)


class ADMPQeqForce:
    """dmff/admp/qeq.py:217-405.  ``precision`` of the engines ('fp64' by default), ``tol`` the
    relative residual of the linear solve, ``max_iter`` its iteration limit."""

    def __init__(self, init_q, r_cut, kappa, K, damp_mod=3, const_list=(), const_vals=(), neutral_flag=True,
                 slab_flag=False, constQ=True, pbc_flag=True, has_aux=False, precision="fp64", tol=1e-12,
                 max_iter=2000):
        if damp_mod not in (1, 2, 3):
            raise ValueError("damp_mod must be 1, 2 or 3")
        const_vals = np.asarray(const_vals, dtype=np.float64)
        assert len(const_list) == len(const_vals), "const_list and const_vals must have the same length"
        if neutral_flag and len(const_vals):
            const_vals = const_vals - np.sum(const_vals) / len(const_vals)
        self.n = len(init_q)
        self.init_q = np.asarray(init_q, dtype=np.float64)
        self.const_vals = const_vals
        self.group = np.full(self.n, -1, dtype=np.int64)
        for g, members in enumerate(const_list):
            for i in members:
                i = int(i)
                if not 0 <= i < self.n:
                    continue
                if self.group[i] >= 0 and self.group[i] != g:
                    raise NotImplementedError("constraint groups sharing an atom are not supported")
                self.group[i] = g
        self.n_const = len(const_list)
        self.r_cut, self.kappa, self.K = float(r_cut), float(kappa) if pbc_flag else 0.0, tuple(int(k) for k in K)
        self.damp_mod, self.neutral_flag, self.slab_flag = damp_mod, neutral_flag, slab_flag
        self.constQ, self.pbc_flag, self.has_aux = constQ, pbc_flag, has_aux
        self.precision, self.tol, self.max_iter = precision, tol, max_iter
        self._coul = {}
        self._sr = None
        self.last_iters = 0

    # --------------------------------------------------------------------------- engines
    def _coul_engine(self, mscales, device):
        key = (tuple(float(x) for x in mscales), str(device))
        eng = self._coul.get(key)
        if eng is None:
            n = self.n
            if self.pbc_flag:
                eng = AdmpEngine(n, 0, False, True, self.r_cut * 10, self.kappa / 10, self.K,
                                 np.full(n, 5, dtype=np.int32), None, np.zeros((0, 3)), list(key[0]),
                                 precision=self.precision, device=device)
            else:  # point charges over the rows, no Ewald split
                eng = AdmpEngine(n, 0, False, False, 1e4, 0.0, (0, 0, 0), np.full(n, 5, dtype=np.int32), None,
                                 np.zeros((0, 3)), list(key[0]), precision=self.precision, device=device)
            eng.set_param_grads(True)
            self._coul[key] = eng
        return eng

    def _sr_engine(self, device):
        if self._sr is None and self.damp_mod in (2, 3):
            kind = L.DMFFB_SR_QEQ_GAUSS3 if self.damp_mod == 3 else L.DMFFB_SR_QEQ_GAUSS2
            self._sr = PairwiseEngine(self.n, kind, rc=max(self.r_cut * 10, 1.0), mscales=[1.0] * 6,
                                      precision=self.precision, device=device)
            self._sr.set_param_grads(True)
        return self._sr

    # --------------------------------------------------------------------------- pieces
    def _site_coefs(self, chi, J):
        """(linear, diagonal quadratic) coefficients of E_site: E_site = sum lin q + quad q^2."""
        if self.damp_mod == 3:
            return chi * 4.184, J * DIELECTRIC * 2 * math.pi
        if self.damp_mod == 2:
            return chi * 96.4869, 0.5 * J * 96.4869
        return torch.zeros_like(chi), torch.zeros_like(chi)

    def _self_coef(self, eta):
        """E_sr self term pre_self q^2, pre_self = D / (eta sqrt(2 pi)) for eta > 1e-4."""
        if self.damp_mod == 1:
            return torch.zeros_like(eta)
        inv = torch.where(eta > 1e-4, 1.0 / torch.where(eta > 1e-4, eta, torch.ones_like(eta)), torch.zeros_like(eta))
        return inv / math.sqrt(2 * math.pi) * DIELECTRIC

    def _slab(self, q, posA, boxA, want_grad=False):
        """E_corr (Angstrom inputs) and, with want_grad, its charge gradient."""
        kap = self.kappa / 10
        V = torch.linalg.det(boxA)
        pre = 2 * math.pi / V * DIELECTRIC
        z = posA[:, 2]
        Mz, Qt, Sz2 = torch.sum(q * z), torch.sum(q), torch.sum(q * z * z)
        Lz = torch.linalg.norm(boxA[2])  # the reference's box[3] clamps to the last row
        e = pre * (Mz ** 2 - Qt * Sz2 - Qt ** 2 * Lz ** 2 / 12)
        pre_non = -math.pi / (2 * V * kap ** 2) * DIELECTRIC if self.neutral_flag else 0.0
        e = e + pre_non * Qt ** 2
        if not want_grad:
            return e
        g = pre * (2 * Mz * z - Sz2 - Qt * z * z - 2 * Qt * Lz ** 2 / 12) + 2 * pre_non * Qt
        return e, g

    def _engines_at(self, q, ctx):
        """One evaluation of both engines at charges q: (E_coul, dE_coul/dq, E_sr_pair,
        dE_sr_pair/dq, coul result, sr result, forces)."""
        dev = ctx["dev"]
        eng = ctx["coul"]
        eng.set_params(q.detach().cpu().numpy().reshape(-1, 1))
        res, F, _ = eng.compute(ctx["posA"], ctx["boxA"], pairs=ctx["rows"])
        gq = eng.param_grads()["Q_global"][:, 0].clone()
        out = {"e_coul": res.energy, "g_coul": gq, "res_coul": res, "F_coul": F.clone()}
        sr = ctx["sr"]
        if sr is not None:
            sr.set_params(torch.stack([q.detach(), ctx["eta"]]))
            r2, F2 = sr.compute(ctx["posA"], ctx["boxA"], pairs=ctx["rows"])
            pg = sr.param_grads()
            out.update(e_sr=r2.energy, g_sr=pg[0].clone(), d_eta=pg[1].clone(), res_sr=r2, F_sr=F2.clone())
        else:
            out.update(e_sr=0.0, g_sr=torch.zeros(self.n, dtype=torch.float64, device=dev), d_eta=None, res_sr=None,
                       F_sr=None)
        return out

    def _matvec(self, v, ctx):
        """A v: the charge Hessian of E_full (no constraint rows) times v."""
        ev = self._engines_at(v, ctx)
        y = ev["g_coul"] + ev["g_sr"] + 2 * (ctx["self"] + ctx["quad"]) * v
        if self.slab_flag:
            _, gs = self._slab(v, ctx["posA"], ctx["boxA"], want_grad=True)
            y = y + gs
        return y

    # --------------------------------------------------------------------------- solve
    def _project(self, r, ctx):
        """z = M^-1 r with the group components removed in the M metric (C z = 0)."""
        z = r * ctx["minv"]
        if self.constQ and self.n_const:
            gid, w = ctx["gid"], ctx["minv"]
            num = torch.zeros(self.n_const + 1, dtype=torch.float64, device=r.device).index_add_(0, gid, z)
            den = torch.zeros(self.n_const + 1, dtype=torch.float64, device=r.device).index_add_(0, gid, w)
            mu = num / torch.where(den > 0, den, torch.ones_like(den))
            mu[-1] = 0.0  # ungrouped atoms
            z = z - w * mu[gid]
        return z

    def _feasible(self, q0, ctx):
        """q0 moved onto C q = c: each group shifted uniformly to its target sum."""
        if not (self.constQ and self.n_const):
            return q0
        gid = ctx["gid"]
        cnt = torch.zeros(self.n_const + 1, dtype=torch.float64, device=q0.device).index_add_(
            0, gid, torch.ones_like(q0))
        s = torch.zeros(self.n_const + 1, dtype=torch.float64, device=q0.device).index_add_(0, gid, q0)
        c = torch.cat([_f64(self.const_vals, q0.device), torch.zeros(1, dtype=torch.float64, device=q0.device)])
        shift = (c - s) / torch.where(cnt > 0, cnt, torch.ones_like(cnt))
        shift[-1] = 0.0
        return q0 + shift[gid]

    def _minres(self, b, x0, ctx):
        """MINRES (Paige-Saunders recurrences) for A x = b from x0, preconditioned by the
        projected diagonal metric; returns (x, iterations)."""
        r1 = b - self._matvec(x0, ctx)
        y = self._project(r1, ctx)
        beta1 = float(torch.dot(r1, y))
        if beta1 <= 0.0:
            return x0, 0
        beta1 = math.sqrt(beta1)
        x = x0.clone()
        oldb, beta, dbar, epsln, phibar = 0.0, beta1, 0.0, 0.0, beta1
        cs, sn = -1.0, 0.0
        w = torch.zeros_like(b)
        w2 = torch.zeros_like(b)
        r2 = r1.clone()
        it = 0
        for it in range(1, self.max_iter + 1):
            v = y / beta
            y = self._matvec(v, ctx)
            if it >= 2:
                y = y - (beta / oldb) * r1
            alfa = float(torch.dot(v, y))
            y = y - (alfa / beta) * r2
            r1, r2 = r2, y
            y = self._project(r2, ctx)
            oldb = beta
            bb = float(torch.dot(r2, y))
            beta = math.sqrt(max(bb, 0.0))
            oldeps = epsln
            delta = cs * dbar + sn * alfa
            gbar = sn * dbar - cs * alfa
            epsln = sn * beta
            dbar = -cs * beta
            gamma = max(math.hypot(gbar, beta), 1e-300)
            cs, sn = gbar / gamma, beta / gamma
            phi = cs * phibar
            phibar = sn * phibar
            w1, w2 = w2, w
            w = (v - oldeps * w1 - delta * w2) / gamma
            x = x + phi * w
            if phibar <= self.tol * beta1 or beta == 0.0:
                break
        return x, it

    # --------------------------------------------------------------------------- energy
    def generate_get_energy(self):
        force = self

        def get_energy(positions, box, pairs, mscales, eta, chi, J, aux=None):
            pos = torch.as_tensor(positions, dtype=torch.float64)
            dev = pos.device if pos.is_cuda else torch.device("cuda", torch.cuda.current_device())
            if not torch.cuda.is_available():
                raise RuntimeError("ADMPQeqForce runs on the GPU engines; no CUDA device is available")
            boxt = torch.as_tensor(box, dtype=torch.float64)
            eta_t, chi_t, J_t = (torch.as_tensor(x, dtype=torch.float64) for x in (eta, chi, J))
            if aux is not None and force.has_aux:
                q0 = torch.as_tensor(aux["q"], dtype=torch.float64).to(dev)
                lam0 = torch.as_tensor(aux["lagmt"], dtype=torch.float64).to(dev)
            else:
                q0 = _f64(force.init_q, dev)
                lam0 = torch.ones(force.n_const, dtype=torch.float64, device=dev)
            E, q, lam = _QeqEnergy.apply(pos, boxt, eta_t, chi_t, J_t,
                                         {"force": force, "pairs": pairs, "mscales": mscales, "q0": q0, "lam0": lam0,
                                          "dev": dev})
            if force.has_aux:
                aux = {} if aux is None else dict(aux)
                aux["q"], aux["lagmt"] = q, lam
                return E, aux
            return E

        return get_energy

    def _context(self, pos, box, pairs, mscales, eta, dev):
        n = self.n
        rows = pairs if torch.is_tensor(pairs) else torch.as_tensor(np.asarray(pairs))
        rows = rows.to(device=dev, dtype=torch.int64)
        keep = (rows[:, 0] < rows[:, 1]) & (rows[:, 1] < n) & (rows[:, 0] >= 0)
        rows = rows[keep]
        nb = rows[:, 2] if rows.shape[1] > 2 else torch.zeros_like(rows[:, 0])
        rows3 = torch.stack([rows[:, 0], rows[:, 1], nb], dim=1).to(torch.int32).contiguous()
        posA = (pos.detach().to(dev) * 10).contiguous()
        boxA = box.detach().to(dev) * 10
        if not self.pbc_flag:
            boxA = torch.eye(3, dtype=torch.float64, device=dev) * 1e4  # no image ever nearer
        eta_d = eta.detach().to(dev)
        ctx = {"dev": dev, "rows": rows3, "posA": posA, "boxA": boxA, "eta": eta_d,
               "coul": self._coul_engine(mscales, dev), "sr": self._sr_engine(dev)}
        ctx["self"] = self._self_coef(eta_d)
        gid = torch.as_tensor(self.group, device=dev)
        ctx["gid"] = torch.where(gid >= 0, gid, torch.full_like(gid, self.n_const))
        return ctx

    def solve(self, pos, box, pairs, mscales, eta, chi, J, q0, lam0, dev):
        """(q*, lambda*, ctx) of the stationary point."""
        ctx = self._context(pos, box, pairs, mscales, eta, dev)
        lin, quad = self._site_coefs(chi.detach().to(dev), J.detach().to(dev))
        ctx["quad"] = quad
        dg = (ctx["self"] + quad).abs()
        floor = max(float(dg.max()) * 1e-6, 1e-12) if dg.numel() else 1.0
        ctx["minv"] = 1.0 / torch.clamp(dg, min=floor)
        g = lin.clone()
        if not self.constQ and self.n_const:  # E_constP: sum_g (sum_{i in g} q_i) c_g
            c = torch.cat([_f64(self.const_vals, dev), torch.zeros(1, dtype=torch.float64, device=dev)])
            g = g + c[ctx["gid"]]
        x0 = self._feasible(q0, ctx)
        q, it = self._minres(-g, x0, ctx)
        self.last_iters = it
        lam = lam0.clone()
        if self.constQ and self.n_const:
            # A q + g = -C^T lambda on the groups: lambda_g from the M-weighted group mean
            grad = self._matvec(q, ctx) + g
            w = ctx["minv"]
            num = torch.zeros(self.n_const + 1, dtype=torch.float64, device=dev).index_add_(0, ctx["gid"], grad * w)
            den = torch.zeros(self.n_const + 1, dtype=torch.float64, device=dev).index_add_(0, ctx["gid"], w)
            lam = -(num / torch.where(den > 0, den, torch.ones_like(den)))[: self.n_const]
        ctx["lin"] = lin
        return q, lam, ctx


class _QeqEnergy(torch.autograd.Function):
    """E_full at the stationary point; gradients with (q*, lambda*) held fixed."""

    @staticmethod
    def forward(ctx, pos, box, eta, chi, J, cfg):
        f = cfg["force"]
        dev = cfg["dev"]
        q, lam, c = f.solve(pos, box, cfg["pairs"], cfg["mscales"], eta, chi, J, cfg["q0"], cfg["lam0"], dev)
        ev = f._engines_at(q, c)
        e = ev["e_coul"] + ev["e_sr"] + float(torch.sum(c["self"] * q * q))
        e += float(torch.sum(c["lin"] * q + c["quad"] * q * q))
        if f.constQ and f.n_const:
            s = torch.zeros(f.n_const + 1, dtype=torch.float64, device=dev).index_add_(0, c["gid"], q)[: f.n_const]
            e += float(torch.sum((s - _f64(f.const_vals, dev)) * lam))
        elif f.n_const:
            s = torch.zeros(f.n_const + 1, dtype=torch.float64, device=dev).index_add_(0, c["gid"], q)[: f.n_const]
            e += float(torch.sum(s * _f64(f.const_vals, dev)))
        # position / box gradients (nm): engines in Angstrom, x10
        gpos = -(ev["F_coul"] + (ev["F_sr"] if ev["F_sr"] is not None else 0.0)) * 10
        gbox = torch.tensor(list(ev["res_coul"].box_grad), dtype=torch.float64, device=dev).reshape(3, 3)
        if ev["res_sr"] is not None:
            gbox = gbox + torch.tensor(list(ev["res_sr"].box_grad), dtype=torch.float64, device=dev).reshape(3, 3)
        gbox = gbox * 10
        if f.slab_flag:
            with torch.enable_grad():  # autograd of the closed-form slab term inside forward
                p_ = (pos.detach().to(dev) * 10).requires_grad_(True)
                b_ = (box.detach().to(dev) * 10).requires_grad_(True)
                es = f._slab(q, p_, b_)
                gp, gb = torch.autograd.grad(es, [p_, b_])
            e += float(es)
            gpos = gpos + gp * 10
            gbox = gbox + gb * 10
        if not f.pbc_flag:
            gbox = torch.zeros_like(gbox)
        # parameter gradients
        if f.damp_mod == 3:
            g_chi, g_J = 4.184 * q, DIELECTRIC * 2 * math.pi * q * q
        elif f.damp_mod == 2:
            g_chi, g_J = 96.4869 * q, 0.5 * 96.4869 * q * q
        else:
            g_chi, g_J = torch.zeros_like(q), torch.zeros_like(q)
        eta_d = c["eta"]
        g_eta = torch.zeros_like(q)
        if f.damp_mod in (2, 3):
            keep = eta_d > 1e-4
            g_eta = ev["d_eta"] - torch.where(keep, DIELECTRIC / math.sqrt(2 * math.pi) * q * q /
                                              torch.where(keep, eta_d, torch.ones_like(eta_d)) ** 2,
                                              torch.zeros_like(q))
        ctx.grads = (gpos.to(pos.device), gbox.to(box.device), g_eta.to(eta.device), g_chi.to(chi.device),
                     g_J.to(J.device))
        out = torch.tensor(e, dtype=torch.float64, device=pos.device)
        ctx.mark_non_differentiable(q, lam)
        return out, q, lam

    @staticmethod
    def backward(ctx, g, gq, glam):
        gp, gb, ge, gc, gj = ctx.grads
        return gp * g, gb * g, ge * g, gc * g, gj * g, None
