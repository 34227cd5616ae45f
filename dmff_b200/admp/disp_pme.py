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
    parameter adjoints."""

    @staticmethod
    def forward(ctx, positions, box, c_list, a, b, q, eng, pairs, force, with_tt):
        pos = positions.detach().to(device=eng.device, dtype=torch.float64).contiguous()
        want_p = any(ctx.needs_input_grad[2:6])
        eng.set_param_grads(want_p)
        res, F = eng.compute(pos, box, pairs=pairs)
        force.last_result = res
        E = (res.e_sr - res.energy) if with_tt else res.energy
        g_sr = torch.tensor(list(res.box_grad_sr), dtype=torch.float64).reshape(3, 3)
        g_lr = torch.tensor(list(res.box_grad), dtype=torch.float64).reshape(3, 3)
        # forces from the engine are -dE_lr/dpos (disp) and -dE_sr/dpos (TT) separately
        Flr, Fsr = F
        grad = (-(Fsr - Flr)) if with_tt else (-Flr)
        ctx.save_for_backward(grad.clone())
        ctx.box_grad = (g_sr - g_lr) if with_tt else g_lr
        ctx.devs = (positions.device, box.device)
        ctx.pdevs = [None if t is None else t.device for t in (c_list, a, b, q)]
        ctx.with_tt = with_tt
        ctx.pg = None
        if want_p:
            pg = eng.param_grads()
            if with_tt:
                dc = -pg["c"].clone()
                dc[:, 0] += pg["c6"]
                ctx.pg = (dc, pg["a"], pg["b"], pg["q"])
            else:
                ctx.pg = (pg["c"], None, None, None)
        return torch.tensor(E, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        outs = [None] * 4
        if ctx.pg is not None:
            for k, t in enumerate(ctx.pg):
                if t is not None and ctx.pdevs[k] is not None:
                    outs[k] = (t * g.to(t.device)).to(ctx.pdevs[k])
        return ((grad * g.to(grad.device)).to(ctx.devs[0]), (ctx.box_grad.to(ctx.devs[1]) * g.to(ctx.devs[1])),
                *outs, None, None, None, None)
