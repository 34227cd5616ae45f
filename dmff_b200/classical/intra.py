"""Drop-ins for dmff/classical/intra.py: harmonic bond, harmonic angle and periodic torsion force
objects built from index arrays and a parameter map.

Same class names, constructor arguments, ``get_energy(positions, box, pairs, k, <equilibrium>)``
closures and ``update_env`` / ``refresh_calculators`` / ``get_forces`` members as the reference
(``HarmonicBondJaxForce`` intra.py:32-62, ``HarmonicAngleJaxForce`` 65-97,
``PeriodicTorsionJaxForce`` 100-138).  ``k`` and the equilibrium values are per parameter type,
picked per term through ``prmidx`` (autograd carries the gradient back through that gather).
The terms run in the engine's FP64 term kernels (``ClassicalForce``, libdmffb200.so); positions
and lengths are handed over x10 with bond constants / 100, which leaves the energy unchanged in
whatever length unit the caller uses.  ``get_forces`` returns (energy, dE/dpositions), the
reference's ``value_and_grad(get_energy)``.
"""
import numpy as np
import torch

from .forces import ClassicalForce


def _t(x):
    return torch.as_tensor(x, dtype=torch.float64)


def _idx(*cols):
    return np.stack([np.asarray(c, dtype=np.int32).ravel() for c in cols], axis=1)


class _TermForce:
    kind = None

    def update_env(self, attr, val):
        """Set one attribute (an index array, the parameter map, ...) and rebuild the closures."""
        setattr(self, attr, val)
        self.refresh_calculators()

    def refresh_calculators(self):
        self.get_energy = self.generate_get_energy()
        self.get_forces = self._value_and_grad(self.get_energy)

    @staticmethod
    def _value_and_grad(fn):
        def value_and_grad(positions, *args):
            with torch.enable_grad():
                p = _t(positions).detach().requires_grad_(True)
                E = _t(fn(p, *args))
                if not E.requires_grad:
                    return E.detach(), torch.zeros_like(p)
                (g,) = torch.autograd.grad(E, p)
            return E.detach(), g

        return value_and_grad

    def _lists(self, cols, with_order=False):
        """Term rows, parameter indices (and torsion orders) read from the attributes at the first
        energy call of this closure, so that ``update_env`` may change them one at a time."""
        memo = []

        def lists():
            if not memo:
                pi = torch.as_tensor(np.asarray(self.prmidx, dtype=np.int64).ravel())
                order = _t(np.asarray(self.order, dtype=np.float64).ravel()) if with_order else None
                memo.append((_idx(*(getattr(self, c) for c in cols)), pi, order))
            return memo[0]

        return lists

    def _force(self, n_atoms):
        f = getattr(self, "_cf", None)
        if f is None or f.n_atoms != n_atoms:
            f = ClassicalForce(n_atoms, precision=self.precision, device=self.device)
            self._cf = f
        return f

    def _run(self, positions, prm, terms):
        positions = _t(positions)
        if terms.shape[0] == 0:
            return torch.zeros((), dtype=torch.float64, device=positions.device)
        f = self._force(positions.shape[0])
        kw = {self.kind + "_idx": terms, self.kind + "_prm": prm}
        box = torch.eye(3, dtype=torch.float64)  # bonded terms use raw coordinates (no periodic image)
        return f.energy(positions * 10.0, box * 10.0, None, **kw)


class HarmonicBondJaxForce(_TermForce):
    """E = sum k/2 (|r_p1 - r_p2| - length)^2 (intra.py:32-62)."""

    kind = "bond"

    def __init__(self, p1idx, p2idx, prmidx, precision="fp64", device=None):
        self.p1idx, self.p2idx, self.prmidx = p1idx, p2idx, prmidx
        self.precision, self.device = precision, device
        self.refresh_calculators()

    def generate_get_energy(self):
        lists = self._lists(("p1idx", "p2idx"))

        def get_energy(positions, box, pairs, k, length):
            terms, pi, _ = lists()
            prm = torch.stack([_t(k)[pi] / 100.0, _t(length)[pi] * 10.0], dim=1)
            return self._run(positions, prm, terms)

        return get_energy


class HarmonicAngleJaxForce(_TermForce):
    """E = sum k/2 (theta - theta0)^2, theta the p1-p2-p3 angle (intra.py:65-97)."""

    kind = "angle"

    def __init__(self, p1idx, p2idx, p3idx, prmidx, precision="fp64", device=None):
        self.p1idx, self.p2idx, self.p3idx, self.prmidx = p1idx, p2idx, p3idx, prmidx
        self.precision, self.device = precision, device
        self.refresh_calculators()

    def generate_get_energy(self):
        lists = self._lists(("p1idx", "p2idx", "p3idx"))

        def get_energy(positions, box, pairs, k, theta0):
            terms, pi, _ = lists()
            prm = torch.stack([_t(k)[pi], _t(theta0)[pi]], dim=1)
            return self._run(positions, prm, terms)

        return get_energy


class PeriodicTorsionJaxForce(_TermForce):
    """E = sum k (1 + cos(order * phi - psi)), phi the p1-p2-p3-p4 dihedral (intra.py:100-138);
    ``order`` is per term, k and psi per parameter type."""

    kind = "torsion"

    def __init__(self, p1idx, p2idx, p3idx, p4idx, prmidx, order, precision="fp64", device=None):
        self.p1idx, self.p2idx, self.p3idx, self.p4idx = p1idx, p2idx, p3idx, p4idx
        self.prmidx, self.order = prmidx, order
        self.precision, self.device = precision, device
        self.refresh_calculators()

    def generate_get_energy(self):
        if len(self.p1idx) == 0:
            return lambda positions, box, pairs, k, psi: 0.0
        lists = self._lists(("p1idx", "p2idx", "p3idx", "p4idx"), with_order=True)

        def get_energy(positions, box, pairs, k, psi):
            terms, pi, order = lists()
            prm = torch.stack([_t(k)[pi], _t(psi)[pi], order], dim=1)
            return self._run(positions, prm, terms)

        return get_energy
