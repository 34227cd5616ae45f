"""ADMPPmeForce backed by the B200 engine (drop-in for dmff/admp/pme.py:36-423).

``get_energy`` keeps the reference's signature (positions and box in Angstrom, Q_local per
atom, pol, tholes, m/p/dScales, U_init, aux) and returns a torch scalar whose autograd yields
dE/dpositions and dE/dbox (the reference's jax.value_and_grad over those arguments).  The
induced dipoles are solved on the GPU: by CG to ``cg_tol`` (default) or with the reference's
fixed-step iteration (``pol_solver='reference'``); as in the reference (pme.py:212-213) the
gradients treat the converged dipoles as constants (Hellmann-Feynman).
"""
import math

import numpy as np
import torch

from ..engine import AdmpEngine
from .settings import MAX_N_POL, POL_CONV

DIELECTRIC = 1389.35455846


def setup_ewald_parameters(rc, ethresh, box=None, spacing=None, method="openmm"):
    """dmff/admp/pme.py:426-492 (float64 host arithmetic)."""
    if method == "openmm":
        kappa = math.sqrt(-math.log(2 * ethresh)) / rc
        box = np.asarray(box, dtype=np.float64)
        K = [int(math.ceil(2 * kappa * box[d, d] / 3 / ethresh ** 0.2)) for d in range(3)]
        return kappa, K[0], K[1], K[2]
    if method == "gromacs":
        kappa, i = 5.0, 0
        while math.erfc(kappa * rc) > ethresh:
            i += 1
            kappa *= 2
        low, high = 0.0, kappa
        for _ in range(i + 60):
            kappa = (low + high) / 2
            if math.erfc(kappa * rc) > ethresh:
                low = kappa
            else:
                high = kappa
        box = np.asarray(box, dtype=np.float64)
        K = [int(math.ceil(box[d, d] / spacing)) for d in range(3)]
        return kappa, K[0], K[1], K[2]
    raise ValueError(f"Invalid method: {method}.Valid methods: 'openmm', 'gromacs'")


def _as_cuda_pairs(pairs, device):
    if pairs is None:
        return None
    if torch.is_tensor(pairs):
        p = pairs
    else:
        p = torch.as_tensor(np.asarray(pairs))
    p = p[:, :3].to(device=device, dtype=torch.int32)
    return p.contiguous()


class _AdmpEnergy(torch.autograd.Function):
    """E(positions, box, Q_local, pol, tholes); backward returns dE/dpositions (-forces), dE/dbox
    and, when the parameter tensors require grad, the engine's parameter adjoints (dE/dQ_local,
    dE/dpol, dE/dthole at the converged dipoles, where E is stationary in U).  Those first
    derivatives come out of ``_AdmpFirstDerivs``, so that with ``create_graph=True`` they are
    differentiable in turn (a loss on forces or on the virial, force matching)."""

    @staticmethod
    def forward(ctx, positions, box, Q_local, pol, tholes, force, pairs, U0, aux):
        eng = force.engine
        dev = eng.device
        pos = positions.detach().to(device=dev, dtype=torch.float64).contiguous()
        want = [t is not None and torch.is_tensor(t) and t.requires_grad for t in (Q_local, pol, tholes)]
        want_p = any(ctx.needs_input_grad[2:5]) and any(want)
        eng.set_param_grads(want_p)
        U = None
        if force.lpol:
            U = (U0.detach().to(device=dev, dtype=torch.float64).contiguous().clone() if U0 is not None
                 else torch.zeros((force.n_atoms, 3), dtype=torch.float64, device=dev))
        res, forces, U = eng.compute(pos, box, pairs=pairs, U=U)
        force.last_result = res
        if aux is not None:
            aux["U_ind"] = U * 0.1  # Angstrom -> nm, as pme.py:225
            aux["lconverg"] = bool(res.converged)
            aux["n_cycle"] = int(res.n_iter)
        pg = eng.param_grads() if want_p else None
        z = lambda t: None if t is None else torch.zeros_like(t, dtype=torch.float64)
        first = {"pos": -forces.clone(), "box": torch.tensor(list(res.box_grad), dtype=torch.float64).reshape(3, 3),
                 "Q_local": pg["Q_local"] if pg is not None else None,
                 "pol": pg["pol"] if pg is not None else None, "thole": pg["thole"] if pg is not None else None}
        ctx.payload = {"force": force, "pairs": pairs, "U": None if U is None else U.clone(), "first": first,
                       "zero": (z(Q_local), z(pol), z(tholes))}
        ctx.save_for_backward(positions, box, Q_local, pol, tholes)
        return torch.tensor(res.energy, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, g):
        positions, box, Q_local, pol, tholes = ctx.saved_tensors
        d = _AdmpFirstDerivs.apply(positions, box, Q_local, pol, tholes, ctx.payload)
        gpos = d[0] * g.to(d[0].device)
        gbox = d[1] * g.to(d[1].device)
        gq = gp = gt = None
        if ctx.payload["first"]["Q_local"] is not None:
            gq = d[2] * g.to(d[2].device) if ctx.needs_input_grad[2] else None
            gp = d[3] * g.to(d[3].device) if ctx.needs_input_grad[3] and d[3] is not None else None
            gt = d[4] * g.to(d[4].device) if ctx.needs_input_grad[4] and d[4] is not None else None
        return gpos, gbox, gq, gp, gt, None, None, None, None


class _AdmpFirstDerivs(torch.autograd.Function):
    """(dE/dpositions, dE/dbox, dE/dQ_local, dE/dpol, dE/dthole) of the forward's evaluation, as
    a function of (positions, box, Q_local, pol, tholes) with the induced dipoles following.  Its
    backward is the engine's second-order pass (dmffb_admp_backward): one adjoint CG solve for the
    dipole response instead of differentiating through the iteration."""

    @staticmethod
    def forward(ctx, positions, box, Q_local, pol, tholes, payload):
        ctx.payload = payload
        ctx.save_for_backward(positions, box, Q_local, pol, tholes)
        f, zero = payload["first"], payload["zero"]

        def out(v, like, zz):
            if like is None:
                return None
            if v is None:
                return zz.clone()
            v = v[:, : like.shape[1]] if like.dim() == 2 and v.dim() == 2 else v
            return v.to(like.device).clone()

        return (f["pos"].to(positions.device).clone(), f["box"].to(box.device).clone(),
                out(f["Q_local"], Q_local, zero[0]), out(f["pol"], pol, zero[1]), out(f["thole"], tholes, zero[2]))

    @staticmethod
    def backward(ctx, c_pos, c_box, c_Q, c_pol, c_th):
        positions, box, Q_local, pol, tholes = ctx.saved_tensors
        p = ctx.payload
        sec = p["force"].second_order(positions, box, Q_local, pol, tholes, p["pairs"], p["U"], c_pos, c_box, c_Q,
                                      c_pol, c_th)
        gQ = None if Q_local is None else sec["Q_local"][:, : Q_local.shape[1]].to(Q_local.device)
        gp = None if pol is None else sec["pol"].to(pol.device)
        gt = None if tholes is None else sec["thole"].to(tholes.device)
        return sec["pos"].to(positions.device), sec["box"].to(box.device), gQ, gp, gt, None


class ADMPPmeForce:
    def __init__(self, box, map_atomtype, axis_type, axis_indices, rc, ethresh, lmax, lpol=False, lpme=True,
                 steps_pol=None, has_aux=False, cov_rows=None, precision="fp32", pol_solver="cg", cg_tol=1e-6,
                 max_iter=500, device=None):
        self.map_atomtype = np.asarray(map_atomtype)
        self.axis_type = np.asarray(axis_type)
        self.axis_indices = None if axis_indices is None else np.asarray(axis_indices)
        self.rc = rc
        self.ethresh = ethresh
        self.lmax = int(lmax)
        self.lpme = lpme
        if lpme:
            self.kappa, self.K1, self.K2, self.K3 = setup_ewald_parameters(rc, ethresh, box)
        else:
            self.kappa, self.K1, self.K2, self.K3 = 0.0, 0, 0, 0
        self.pme_order = 6
        self.lpol = lpol
        self.steps_pol = steps_pol
        self.n_atoms = len(self.axis_type)
        self.has_aux = has_aux
        self.cov_rows = np.zeros((0, 3), np.int32) if cov_rows is None else np.asarray(cov_rows)
        self.precision = precision
        self.pol_solver = pol_solver if steps_pol is None else "reference"
        self.cg_tol = cg_tol if self.pol_solver == "cg" else POL_CONV
        self.max_iter = max_iter if self.pol_solver == "cg" else MAX_N_POL
        self.device = device
        self.U_ind = torch.zeros((self.n_atoms, 3), dtype=torch.float64)
        self._engine = None
        self._param_key = None
        self.last_result = None
        self.refresh_calculators()

    @property
    def engine(self):
        if self._engine is None:
            self._engine = AdmpEngine(
                self.n_atoms, self.lmax, self.lpol, self.lpme, self.rc, self.kappa, (self.K1, self.K2, self.K3),
                self.axis_type if self.lmax > 0 else None, self.axis_indices if self.lmax > 0 else None,
                self.cov_rows, [0, 0, 1, 1, 1, 1], precision=self.precision, solver=self.pol_solver,
                cg_tol=self.cg_tol, max_iter=self.max_iter, steps_pol=self.steps_pol, device=self.device)
        return self._engine

    def _sync_params(self, Q_local, pol, tholes, mScales, pScales, dScales):
        # keyed by value: a fresh tensor can reuse a freed one's address, so identity is not enough
        vals = tuple(None if t is None else torch.as_tensor(t, dtype=torch.float64).detach().cpu().clone()
                     for t in (Q_local, pol, tholes))
        scales = tuple(tuple(np.asarray(torch.as_tensor(s).detach().cpu()).tolist()) if s is not None else None
                       for s in (mScales, pScales, dScales))
        old = self._param_key
        if old is not None and old[1] == scales and all(
                (a is None and b is None) or (a is not None and b is not None and a.shape == b.shape and torch.equal(a, b))
                for a, b in zip(old[0], vals)):
            return
        key = (vals, scales)
        # scales are part of the engine description: rebuild when they change
        ms = np.asarray(torch.as_tensor(mScales).detach().cpu(), np.float64)
        ps = np.asarray(torch.as_tensor(pScales).detach().cpu(), np.float64) if pScales is not None else None
        ds = np.asarray(torch.as_tensor(dScales).detach().cpu(), np.float64) if dScales is not None else None
        scales = (tuple(ms), None if ps is None else tuple(ps), None if ds is None else tuple(ds))
        if getattr(self, "_scales", None) != scales:
            self._engine = AdmpEngine(
                self.n_atoms, self.lmax, self.lpol, self.lpme, self.rc, self.kappa, (self.K1, self.K2, self.K3),
                self.axis_type if self.lmax > 0 else None, self.axis_indices if self.lmax > 0 else None,
                self.cov_rows, ms, ps, ds, precision=self.precision, solver=self.pol_solver, cg_tol=self.cg_tol,
                max_iter=self.max_iter, steps_pol=self.steps_pol, device=self.device)
            self._scales = scales
        self.engine.set_params(Q_local, pol if self.lpol else None, tholes if self.lpol else None)
        self._param_key = key

    def second_order(self, positions, box, Q_local, pol, tholes, pairs, U, c_pos, c_box, c_Q, c_pol, c_thole):
        """Vector-Jacobian product through the first derivatives of an evaluation (the backward of
        ``_AdmpFirstDerivs``), on an FP64 engine: the forward's engine when it is FP64, else an FP64
        engine of the same system kept for this purpose.  The engine is brought back to the
        evaluation's point (parameters, positions, pairs; the dipole solve restarts from the
        forward's converged dipoles) and runs dmffb_admp_backward."""
        if self.precision == "fp64":
            eng = self.engine
        else:
            if getattr(self, "_engine64", None) is None:
                ms, ps, ds = self._scales if getattr(self, "_scales", None) else ([0, 0, 1, 1, 1, 1],) * 3
                self._engine64 = AdmpEngine(
                    self.n_atoms, self.lmax, self.lpol, self.lpme, self.rc, self.kappa, (self.K1, self.K2, self.K3),
                    self.axis_type if self.lmax > 0 else None, self.axis_indices if self.lmax > 0 else None,
                    self.cov_rows, ms, ps, ds, precision="fp64", solver="cg", cg_tol=min(self.cg_tol, 1e-10),
                    max_iter=max(self.max_iter, 1000), device=self.device)
            eng = self._engine64
        self._param_key = None  # the engine's parameters are set below: the value cache is stale
        eng.set_params(Q_local.detach(), pol.detach() if self.lpol else None, tholes.detach() if self.lpol else None)
        eng.set_param_grads(False)
        pos = positions.detach().to(device=eng.device, dtype=torch.float64).contiguous()
        Ui = None if U is None else U.detach().to(device=eng.device, dtype=torch.float64).contiguous().clone()
        if pairs is None:  # the engine's own list, built at this evaluation's positions
            eng.rebuild_internal_pairs(pos, box.detach())
        eng.compute(pos, box.detach(), pairs=pairs, U=Ui)
        cQ = None
        if c_Q is not None:
            cQ = torch.zeros((self.n_atoms, 9), dtype=torch.float64, device=eng.device)
            cQ[:, : c_Q.shape[1]] = c_Q.detach().to(eng.device, torch.float64)
        out = eng.backward(c_pos, c_box, cQ, c_pol if self.lpol else None, c_thole if self.lpol else None)
        self.last_second_order = {"n_iter": out["n_iter"], "residual_rms": out["residual_rms"], "step": out["step"]}
        return out

    def get_energy(self, positions, box, pairs, Q_local, pol=None, tholes=None, mScales=None, pScales=None,
                   dScales=None, U_init=None, aux=None):
        """Energy (kJ/mol) for positions / box in Angstrom; pairs (i, j, nbond) rows or None for the
        engine's own cell-list pairs.  As in the reference (pme.py:186-232), U_init is in nm and is
        scaled to Angstrom here, and ``aux`` receives U_ind (nm), lconverg and n_cycle."""
        if not self.lpol:
            # non-polarizable signature: get_energy(positions, box, pairs, Q_local, mScales)
            if mScales is None and pol is not None:
                mScales, pol = pol, None
        self._sync_params(Q_local, pol, tholes, mScales, pScales, dScales)
        eng = self.engine
        if not torch.is_tensor(positions):
            positions = torch.as_tensor(np.asarray(positions), dtype=torch.float64)
        if not torch.is_tensor(box):
            box = torch.as_tensor(np.asarray(box), dtype=torch.float64)
        pairs_d = _as_cuda_pairs(pairs, eng.device)
        U0 = None
        if self.lpol:
            U0 = U_init if U_init is not None else self.U_ind
            U0 = torch.as_tensor(np.asarray(U0) if not torch.is_tensor(U0) else U0, dtype=torch.float64) * 10.0
        Q_local = torch.as_tensor(Q_local, dtype=torch.float64)
        if self.lpol:
            pol = torch.as_tensor(pol, dtype=torch.float64)
            tholes = torch.as_tensor(tholes, dtype=torch.float64)
        else:
            pol = tholes = None
        E = _AdmpEnergy.apply(positions, box, Q_local, pol, tholes, self, pairs_d, U0, aux)
        return E if aux is None else (E, aux)

    def generate_get_energy(self):
        """The energy closure of pme.py:116-245.  Its signature covers both of the reference's
        forms: (positions, box, pairs, Q_local, mScales) and, polarizable, (..., Q_local, pol,
        tholes, mScales, pScales, dScales, U_init, aux)."""
        return ADMPPmeForce.get_energy.__get__(self)

    def generate_esp(self):
        """``get_esp(positions, grids, Q_local[, U_ind])`` -> potential [n_grid] (kJ/mol/e) of the
        global multipoles (and induced dipoles when polarizable) at grid points, no periodic
        images (pme.py:236-293).  Charge q / r, dipoles -(d / 10 + U) . dR / r^3 and
        quadrupoles 3 dR^T (Q / 300) dR / r^5 with dR = r_site - r_grid, times DIELECTRIC / 10.
        Host torch on the input's device, 4096 grid points at a time."""

        def esp(positions, grids, Q_local, U_ind=None):
            pos = torch.as_tensor(positions, dtype=torch.float64)
            g = torch.as_tensor(grids, dtype=torch.float64).to(pos.device)
            Qg = self.Q_local_to_global(pos, torch.eye(3, dtype=torch.float64, device=pos.device) * 1000.0,
                                        torch.as_tensor(Q_local, dtype=torch.float64).to(pos.device))
            n = pos.shape[0]
            q = Qg[:, 0]
            d = Qg[:, 1:4] / 10.0 if Qg.shape[1] >= 4 else torch.zeros((n, 3), dtype=torch.float64, device=pos.device)
            if U_ind is not None:
                d = d + torch.as_tensor(U_ind, dtype=torch.float64).to(pos.device)
            quad = Qg[:, 4:10] / 300.0 if Qg.shape[1] >= 10 else None
            out = []
            for g0 in range(0, g.shape[0], 4096):
                dR = pos[None, :, :] - g[g0:g0 + 4096, None, :]  # [G, n, 3]
                r2 = (dR * dR).sum(-1) + 1e-16
                rr1 = torch.rsqrt(r2)
                rr3 = rr1 * rr1 * rr1
                v = q * rr1 - (d * dR).sum(-1) * rr3
                if quad is not None:
                    xx, yy, zz, xy, xz, yz = quad.unbind(-1)
                    x, y, z = dR.unbind(-1)
                    scq = (xx * x * x + yy * y * y + zz * z * z) + 2.0 * (xy * x * y + xz * x * z + yz * y * z)
                    v = v + scq * 3.0 * rr3 * rr1 * rr1
                out.append(v.sum(-1))
            return torch.cat(out) * DIELECTRIC * 0.1

        if self.lpol:
            def get_esp(positions, grids, Q_local, U_ind):
                return esp(positions, grids, Q_local, U_ind)
        else:
            def get_esp(positions, grids, Q_local):
                return esp(positions, grids, Q_local)
        return get_esp

    def generate_Q_global_function(self):
        """``get_Q_global(positions, box, Q_local)`` -> global Cartesian multipoles [n, 1 | 4 | 10]
        (charge; dipole; quadrupole xx yy zz xy xz yz), i.e. Q_local per type mapped to atoms,
        rotated by the local frames and converted to Cartesian (pme.py:183-196).  A host
        utility in torch; the engine keeps its own global multipoles on the GPU."""
        from .multipole import convert_harm2cart, rot_local2global
        from .spatial import generate_construct_local_frames
        lmax, mt = self.lmax, torch.as_tensor(self.map_atomtype, dtype=torch.long)
        has_frames = lmax > 0 and self.axis_indices is not None
        frames = generate_construct_local_frames(self.axis_type, self.axis_indices) if has_frames else None

        def get_Q_global(positions, box, Q_local):
            Q = torch.as_tensor(Q_local, dtype=torch.float64)[mt.to(Q_local.device if torch.is_tensor(Q_local)
                                                                      else "cpu")]
            if frames is not None:
                Q = rot_local2global(Q[:, : (lmax + 1) ** 2], frames(positions, box), lmax)
            return convert_harm2cart(Q, lmax)

        return get_Q_global

    def update_env(self, attr, val):
        """Set one attribute (kappa, K1, lmax, axis_type, ...) and rebuild the calculators
        (pme.py:198-203)."""
        setattr(self, attr, val)
        self.refresh_calculators()

    def refresh_calculators(self):
        """Drop the engine so that the next call builds one from the current attributes, and
        regenerate ``get_forces`` = value_and_grad(get_energy) w.r.t. positions (pme.py:205-224)."""
        self._engine = None
        self._param_key = None
        self._scales = None
        self.n_atoms = len(self.axis_type)
        self.U_ind = torch.zeros((self.n_atoms, 3), dtype=torch.float64)
        self.Q_local_to_global = self.generate_Q_global_function()
        if self.lmax > 0 and self.axis_indices is not None:
            from .spatial import generate_construct_local_frames
            self.construct_local_frames = generate_construct_local_frames(self.axis_type, self.axis_indices)
        else:
            self.construct_local_frames = None
        energy = self.generate_get_energy()

        def get_forces(positions, *args, **kwargs):
            with torch.enable_grad():
                p = torch.as_tensor(positions, dtype=torch.float64).detach().requires_grad_(True)
                out = energy(p, *args, **kwargs)
                E = out[0] if isinstance(out, tuple) else out
                (g,) = torch.autograd.grad(E, p)
            return (E.detach(), g) if not isinstance(out, tuple) else ((E.detach(), out[1]), g)

        self.get_forces = get_forces
