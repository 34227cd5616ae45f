"""ADMPDispPmeForce backed by the B200 engine (drop-in for dmff/admp/disp_pme.py:13-77).

``get_energy(positions, box, pairs, c_list, mScales)`` returns the dispersion PME energy E_lr
(real + three reciprocal passes with the k = 0 term + self, disp_pme.py:80-130) as a torch
scalar with autograd to positions and box.  With ``tt=(a_list, b_list, q_list)`` it returns
E_sr - E_lr, E_sr the Tang-Toennies damped short-range term of ADMPDispForce
(pairwise.py:100-118, admp.py:183-208), evaluated in the same pair pass.
"""
import numpy as np
import torch

from .pme import setup_ewald_parameters


class ADMPDispPmeForce:
    def __init__(self, box, rc, ethresh, pmax, lpme=True, cov_rows=None, tt_damping=False, precision="fp32",
                 device=None):
        self.rc, self.ethresh, self.pmax, self.lpme = rc, ethresh, pmax, lpme
        if lpme:
            self.kappa, self.K1, self.K2, self.K3 = setup_ewald_parameters(rc, ethresh, box)
        else:
            self.kappa, self.K1, self.K2, self.K3 = 0.0, 0, 0, 0
        self.pme_order = 6
        self.cov_rows = np.zeros((0, 3), np.int32) if cov_rows is None else np.asarray(cov_rows)
        self.tt = tt_damping
        self.precision = precision
        self.device = device
        self._engine = None
        self._key = None
        self.last_result = None
        self.refresh_calculators()

    def generate_get_energy(self):
        """The energy closure of disp_pme.py:45-51, get_energy(positions, box, pairs, c_list,
        mScales) (with the optional ``tt`` triple of this engine's fused short-range term)."""
        return ADMPDispPmeForce.get_energy.__get__(self)

    def update_env(self, attr, val):
        """Set one attribute (kappa, K1, pmax, ...) and rebuild the calculators
        (disp_pme.py:54-59)."""
        setattr(self, attr, val)
        self.refresh_calculators()

    def refresh_calculators(self):
        """Drop the engine so that the next call builds one from the current attributes, and
        regenerate ``get_forces`` = value_and_grad(get_energy) w.r.t. positions
        (disp_pme.py:62-77)."""
        self._engine = None
        energy = self.generate_get_energy()

        def get_forces(positions, *args, **kwargs):
            with torch.enable_grad():
                p = torch.as_tensor(positions, dtype=torch.float64).detach().requires_grad_(True)
                E = energy(p, *args, **kwargs)
                (g,) = torch.autograd.grad(E, p)
            return E.detach(), g

        self.get_forces = get_forces

    def _eng(self, n, mScales):
        from ..engine import DispEngine
        ms = tuple(float(x) for x in np.asarray(torch.as_tensor(mScales).detach().cpu()))
        if self._engine is None or self._engine.n != n or self._engine.mscales != ms:
            self._engine = DispEngine(n, self.pmax, self.lpme, self.rc, self.kappa, (self.K1, self.K2, self.K3),
                                      self.cov_rows, ms, tt=self.tt, precision=self.precision, device=self.device)
        return self._engine

    def second_order(self, point, pairs, with_tt, cot):
        """Vector-Jacobian product through the first derivatives at ``point`` = (positions, box,
        c_list, a, b, q) with cotangents ``cot``: central differences of the engine's analytic
        first derivatives along ``cot`` (``_hvp.central_hvp``), on an FP64 engine of the same
        system with its pair list built at the evaluation's positions."""
        from .._hvp import central_hvp
        from ..engine import DispEngine
        eng0 = self._engine
        if self.precision == "fp64":
            eng = eng0
        else:
            if getattr(self, "_engine64", None) is None or self._engine64.n != eng0.n:
                self._engine64 = DispEngine(eng0.n, self.pmax, self.lpme, self.rc, self.kappa,
                                            (self.K1, self.K2, self.K3), self.cov_rows, eng0.mscales, tt=self.tt,
                                            precision="fp64", device=self.device)
            eng = self._engine64
        pos0, box0 = point[0], point[1]
        dev = eng.device
        eng.rebuild_internal_pairs(pos0.detach().to(dev, torch.float64).contiguous(), box0.detach())
        want_p = any(t is not None for t in point[2:])

        def grad_at(z):
            pos, box, c, a, b, q = z
            eng.set_params(c.detach(), *((a.detach(), b.detach(), q.detach()) if with_tt else (None, None, None)))
            _, first = _disp_first(eng, pos.detach().to(dev, torch.float64).contiguous(), box.detach(), pairs,
                                   with_tt, want_p)
            return [first[0].to(pos.device), first[1].to(box.device)] + [
                None if t is None else (torch.zeros_like(t) if v is None else v.to(t.device))
                for v, t in zip(first[2:], z[2:])]

        scales = [1.0, 1.0] + [1.0 if t is None else float(t.detach().abs().max()) for t in point[2:]]
        direction = [None if c is None else c.detach() for c in cot]
        hv, step = central_hvp(grad_at, [None if t is None else t.detach().to(torch.float64) for t in point],
                               direction, scales)
        self.last_second_order = {"step": step}
        return hv

    def get_energy(self, positions, box, pairs, c_list, mScales, tt=None):
        from .pme import _as_cuda_pairs
        positions = torch.as_tensor(positions, dtype=torch.float64)
        if not torch.is_tensor(box):
            box = torch.as_tensor(np.asarray(box), dtype=torch.float64)
        eng = self._eng(positions.shape[0], mScales)
        eng.set_params(c_list, *(tt if tt is not None else (None, None, None)))
        c_list = torch.as_tensor(c_list, dtype=torch.float64)
        a, b, q = (None, None, None) if tt is None else (torch.as_tensor(x, dtype=torch.float64) for x in tt)
        return _DispEnergy.apply(positions, box, c_list, a, b, q, eng, _as_cuda_pairs(pairs, eng.device), self,
                                 tt is not None)


class _DispEnergy(torch.autograd.Function):
    """E_lr, or E_sr - E_lr with TT damping, of (positions, box, c_list, a, b, q); backward gives
    position / box gradients and, when the parameter tensors require grad, the engine's
    parameter adjoints.  The first derivatives come out of ``_DispFirstDerivs``, so that they are
    differentiable in turn (``create_graph=True``)."""

    @staticmethod
    def forward(ctx, positions, box, c_list, a, b, q, eng, pairs, force, with_tt):
        pos = positions.detach().to(device=eng.device, dtype=torch.float64).contiguous()
        want_p = any(ctx.needs_input_grad[2:6])
        res, first = _disp_first(eng, pos, box, pairs, with_tt, want_p)
        force.last_result = res
        E = (res.e_sr - res.energy) if with_tt else res.energy
        ctx.payload = {"force": force, "pairs": pairs, "with_tt": with_tt, "first": first, "want_p": want_p}
        ctx.save_for_backward(positions, box, c_list, a, b, q)
        return torch.tensor(E, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, g):
        saved = ctx.saved_tensors
        d = _DispFirstDerivs.apply(*saved, ctx.payload)
        outs = []
        for k, t in enumerate(d):
            if t is None or (k >= 2 and not (ctx.payload["want_p"] and ctx.needs_input_grad[k])):
                outs.append(None)
            else:
                outs.append(t * g.to(t.device))
        return (*outs, None, None, None, None)


def _disp_first(eng, pos, box, pairs, with_tt, want_p):
    """One engine evaluation; returns (result, [dE/dpos, dE/dbox, dE/dc [n, 3], dE/da, dE/db, dE/dq])
    of E = E_lr, or E_sr - E_lr with TT (parameter blocks None without adjoints)."""
    eng.set_param_grads(want_p)
    res, F = eng.compute(pos, box, pairs=pairs)
    g_sr = torch.tensor(list(res.box_grad_sr), dtype=torch.float64).reshape(3, 3)
    g_lr = torch.tensor(list(res.box_grad), dtype=torch.float64).reshape(3, 3)
    # forces from the engine are -dE_lr/dpos (disp) and -dE_sr/dpos (TT) separately
    Flr, Fsr = F
    first = [(-(Fsr - Flr)) if with_tt else (-Flr).clone(), (g_sr - g_lr) if with_tt else g_lr, None, None, None, None]
    if want_p:
        pg = eng.param_grads()
        if with_tt:
            dc = -pg["c"].clone()
            dc[:, 0] += pg["c6"]
            first[2:] = [dc, pg["a"].clone(), pg["b"].clone(), pg["q"].clone()]
        else:
            first[2] = pg["c"].clone()
    return res, first


class _DispFirstDerivs(torch.autograd.Function):
    """(dE/dpositions, dE/dbox, dE/dc_list, dE/da, dE/db, dE/dq) of the forward's evaluation as a
    function of those inputs; its backward is the Hessian-vector product by central differences
    of the engine's analytic first derivatives (``_hvp.central_hvp``)."""

    @staticmethod
    def forward(ctx, positions, box, c_list, a, b, q, payload):
        ctx.payload = payload
        ctx.save_for_backward(positions, box, c_list, a, b, q)
        like = (positions, box, c_list, a, b, q)
        out = []
        for v, t in zip(payload["first"], like):
            if t is None:
                out.append(None)
            elif v is None:
                out.append(torch.zeros_like(t, dtype=torch.float64))
            else:
                out.append(v.to(t.device).clone())
        return tuple(out)

    @staticmethod
    def backward(ctx, *cot):
        saved = ctx.saved_tensors
        p = ctx.payload
        sec = p["force"].second_order(saved, p["pairs"], p["with_tt"], cot)
        return (*[None if t is None else g.to(t.device) for g, t in zip(sec, saved)], None)
