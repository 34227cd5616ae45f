"""Engine-backed classical force objects (drop-ins for dmff/classical/inter.py and intra.py).

``ClassicalForce`` holds one ``ClassicalEngine`` (libdmffb200.so) for one generator:
LJ + point-charge Coulomb in one fused pair pass (PME / reaction field / plain 1/r), the PME
reciprocal and self terms, and harmonic bond / angle / periodic torsion term lists.
``energy(...)`` takes Angstrom-unit torch tensors and returns a torch scalar whose autograd
gives dE/dpositions and dE/dbox from the engine's forward pass and, when any parameter tensor
requires grad, the parameter adjoints the kernels write (dE/dq, dE/dsigma_ij, dE/deps_ij per
type pair, dE/dk and dE/d(r0 | theta0 | psi) per term).
"""
import numpy as np
import torch


def _as_cuda_pairs(pairs, device):
    if pairs is None:
        return None
    p = pairs if torch.is_tensor(pairs) else torch.as_tensor(np.asarray(pairs))
    if p.dim() != 2 or p.shape[0] == 0 or p.shape[1] < 3:
        return torch.zeros((0, 3), dtype=torch.int32, device=device)
    return p[:, :3].to(device=device, dtype=torch.int32).contiguous()


class ClassicalForce:
    """One classical engine.  coulomb: 'pme' | 'rf' | 'nocutoff' | 'none'; n_types > 0 enables LJ."""

    def __init__(self, n_atoms, n_types=0, coulomb="none", pbc=True, rc=10.0, kappa=0.0, K=(0, 0, 0),
                 cov_rows=None, mscales_coul=(0, 0, 0, 1, 1, 1), mscales_lj=(0, 0, 0, 1, 1, 1),
                 eps_solvent=78.5, precision="fp32", device=None):
        self.cfg = dict(n_atoms=int(n_atoms), n_types=int(n_types), coulomb=coulomb, pbc=bool(pbc), rc=float(rc),
                        kappa=float(kappa), K=tuple(int(k) for k in K), cov_rows=cov_rows,
                        mscales_coul=tuple(float(x) for x in mscales_coul),
                        mscales_lj=tuple(float(x) for x in mscales_lj), eps_solvent=float(eps_solvent),
                        precision=precision, device=device)
        self.n_atoms = int(n_atoms)
        self.n_types = int(n_types)
        self.coulomb = coulomb
        self._engine = None
        self._cache = {}
        self.last_result = None

    @property
    def engine(self):
        if self._engine is None:
            from ..engine import ClassicalEngine
            self._engine = ClassicalEngine(**self.cfg)
        return self._engine

    def _changed(self, key, t):
        if t is None:
            return False
        h = t.detach().to("cpu", torch.float64).contiguous()
        old = self._cache.get(key)
        if old is not None and old.shape == h.shape and torch.equal(old, h):
            return False
        self._cache[key] = h.clone()
        return True

    def energy(self, positions, box, pairs, charges=None, atom_type=None, sigma_tt=None, eps_tt=None,
               bond_idx=None, bond_prm=None, angle_idx=None, angle_prm=None, torsion_idx=None, torsion_prm=None):
        """positions [n,3] A, box [3,3] A (rows = lattice vectors); pairs (i, j, nbond) rows or None
        (engine's own list); charges [n]; sigma_tt / eps_tt [T,T] (A, kJ/mol); *_idx int [m, 2|3|4];
        bond_prm [m,2] (k kJ/mol/A^2, r0 A), angle_prm [m,2] (k, theta0), torsion_prm [m,3] (k, psi, n)."""
        eng = self.engine
        p_changed = any([self._changed("q", charges), self._changed("sig", sigma_tt), self._changed("eps", eps_tt)])
        if p_changed or "types" not in self._cache:
            if atom_type is not None:
                self._cache["types"] = np.asarray(atom_type, dtype=np.int32)
            else:
                self._cache["types"] = None
            eng.set_params(self._cache.get("q"), self._cache["types"], self._cache.get("sig"), self._cache.get("eps"))
        terms = (("bond", bond_idx, bond_prm), ("angle", angle_idx, angle_prm), ("torsion", torsion_idx, torsion_prm))
        for kind, idx, prm in terms:
            if prm is None:
                continue
            if self._changed(kind, prm) or self._cache.get(kind + "_idx") is not idx:
                self._cache[kind + "_idx"] = idx
                eng.set_terms(kind, idx, self._cache[kind])
        params = [charges, sigma_tt, eps_tt, bond_prm, angle_prm, torsion_prm]
        want = torch.is_grad_enabled() and any(t is not None and t.requires_grad for t in params)
        eng.set_param_grads(want)
        positions = torch.as_tensor(positions, dtype=torch.float64)
        box = torch.as_tensor(box, dtype=torch.float64)
        dummy = lambda t: t if t is not None else torch.zeros(0, dtype=torch.float64)
        return _ClassicalEnergy.apply(positions, box, dummy(charges), dummy(sigma_tt), dummy(eps_tt), dummy(bond_prm),
                                      dummy(angle_prm), dummy(torsion_prm), self,
                                      _as_cuda_pairs(pairs, eng.device), want)


class _ClassicalEnergy(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, box, charges, sigma_tt, eps_tt, bond_prm, angle_prm, torsion_prm, force, pairs,
                want):
        eng = force.engine
        pos = positions.detach().to(device=eng.device, dtype=torch.float64).contiguous()
        res, F = eng.compute(pos, box, pairs=pairs)
        force.last_result = res
        ctx.grad_pos = (-F).clone()
        ctx.box_grad = torch.tensor(list(res.box_grad), dtype=torch.float64).reshape(3, 3)
        ctx.pg = eng.param_grads() if want else None
        ctx.shapes = [t.shape for t in (charges, sigma_tt, eps_tt, bond_prm, angle_prm, torsion_prm)]
        ctx.devs = [t.device for t in (positions, box, charges, sigma_tt, eps_tt, bond_prm, angle_prm, torsion_prm)]
        return torch.tensor(res.energy, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, g):
        gp = (ctx.grad_pos * g.to(ctx.grad_pos.device)).to(ctx.devs[0])
        gb = (ctx.box_grad.to(ctx.devs[1]) * g.to(ctx.devs[1]))
        outs = [None] * 6
        if ctx.pg is not None:
            pg = ctx.pg
            cand = [pg["q"], pg["sigma_tt"], pg["eps_tt"], pg["bond"], pg["angle"], None]
            if pg["torsion"].numel():
                t = pg["torsion"]
                cand[5] = torch.stack([t[:, 0], t[:, 1], torch.zeros_like(t[:, 0])], dim=1)
            for k, c in enumerate(cand):
                n_el = int(np.prod(ctx.shapes[k])) if len(ctx.shapes[k]) else 0
                if c is None or n_el == 0:
                    continue
                outs[k] = (c.reshape(ctx.shapes[k]) * g.to(c.device)).to(ctx.devs[2 + k])
        return (gp, gb, *outs, None, None, None)
