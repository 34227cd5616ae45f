"""Trajectory-batched energies and parameter gradients for force-field fitting.

The reference's fitting consumers evaluate a potential over the frames of a trajectory and
differentiate the result with respect to the parameters: ``buildTrajEnergyFunction`` builds a
neighbour list per frame with freud and calls the potential frame by frame
(dmff/mbar.py:27-80), ``TargetState.calc_energy`` turns the energies into reduced energies
(mbar.py:83-92), and optax optimizers step on ``jax.grad`` of a loss built from them
(dmff/optimize.py:30-84).

Here the same two functions keep the reference's signatures over the drop-in potentials
(``buildTrajEnergyFunction``, ``TargetState``), and ``TrajectoryEvaluator`` is the batched path
on one engine: every frame's positions go to the device once, each frame rebuilds the engine's
cell list on the device, the induced-dipole solve of frame k starts from frame k - 1's dipoles
(consecutive frames of a trajectory are close), and the per-atom parameter adjoints of all frames
are accumulated on the device with per-frame weights; the host waits once per batch.
"""
import numpy as np
import torch

from .engine import AdmpEngine

# kJ/mol per (bar nm^3): the PV term of the NPT reduced energy (dmff/mbar.py:74)
PV_KJMOL_PER_BAR_NM3 = 0.06023


def _traj_arrays(traj):
    """(positions [F, n, 3] nm, boxes [F, 3, 3] nm, volumes [F] nm^3) of an mdtraj-like object
    (attributes xyz, unitcell_vectors, unitcell_volumes) or a dict with those keys."""
    get = (lambda k: traj[k]) if isinstance(traj, dict) else (lambda k: getattr(traj, k))
    xyz = np.asarray(get("xyz"), dtype=np.float64)
    boxes = np.asarray(get("unitcell_vectors"), dtype=np.float64)
    try:
        vols = np.asarray(get("unitcell_volumes"), dtype=np.float64)
    except (KeyError, AttributeError):
        vols = np.abs(np.linalg.det(boxes))
    return xyz, boxes, vols


def buildTrajEnergyFunction(potential_func, cov_map, cutoff, usePBC=True, useFreud=True, ensemble="nvt",
                            pressure=1.0):
    """dmff/mbar.py:27-80: ``energy_function(traj, parameters)`` -> list of per-frame energies
    (kJ/mol, torch scalars carrying autograd to the parameters).  Periodic frames take the
    potential's own cell-list pairs (the reference builds a freud list per frame); non-periodic
    ones every pair with its nbond from ``cov_map``.  NPT adds pressure * 0.06023 * V per frame."""
    if ensemble.upper() not in ("NVT", "NPT"):
        raise ValueError(f"unknown ensemble {ensemble}")
    ens = 0.0 if ensemble.upper() == "NVT" else 1.0

    def energy_function(traj, parameters):
        xyz, boxes, vols = _traj_arrays(traj)
        pairs = None
        if not usePBC:
            from .common.nblist import NoCutoffNeighborList
            nbl = NoCutoffNeighborList(cov_map, padding=False, device=None if torch.cuda.is_available() else "cpu")
            pairs = nbl.allocate(torch.as_tensor(xyz[0]))
        from .common.nblist import NeighborList
        out = []
        for f in range(xyz.shape[0]):
            pos = torch.as_tensor(xyz[f])
            box = torch.as_tensor(boxes[f])
            p = pairs
            if usePBC:
                nbl = NeighborList(boxes[f], cutoff, cov_map, padding=False)
                p = nbl.allocate(xyz[f])
            e = potential_func(pos, box, p, parameters)
            out.append(e + ens * pressure * PV_KJMOL_PER_BAR_NM3 * float(vols[f]))
        return out

    return energy_function


class TargetState:
    """dmff/mbar.py:83-92: reduced energies u = E / (R T) of a trajectory at ``temperature``."""

    def __init__(self, temperature, energy_function):
        self._temperature = temperature
        self._efunc = energy_function

    def calc_energy(self, trajectory, parameters):
        beta = 1.0 / self._temperature / 8.314 * 1000.0
        eners = self._efunc(trajectory, parameters)
        return torch.stack([beta * torch.as_tensor(e).reshape(()) for e in eners])


class TrajectoryEvaluator:
    """Energies and weighted parameter gradients of one ADMP system over many frames, batched on
    one engine.

    ``engine`` an ``AdmpEngine`` (its parameters set); ``frames`` positions [F, n, 3] and boxes
    [F, 3, 3] in Angstrom.  ``evaluate(weights)`` returns the per-frame energies [F] and, with
    ``param_grads=True``, sum_f w_f dE_f/d(Q_local [n, 9], pol [n], thole [n]) (per atom, at each
    frame's converged dipoles) -- the gradient of the fitting loss sum_f w_f E_f.  Frames run in
    order; each dipole solve starts from the previous frame's solution."""

    def __init__(self, engine: AdmpEngine, positions, boxes):
        self.eng = engine
        dev = engine.device
        self.pos = torch.as_tensor(np.asarray(positions, dtype=np.float64)).to(dev).contiguous()
        self.boxes = np.asarray(boxes, dtype=np.float64).reshape(-1, 3, 3)
        assert self.pos.shape[0] == self.boxes.shape[0] and self.pos.shape[1] == engine.n
        self.n_frames = self.pos.shape[0]
        self.last_iters = []

    def evaluate(self, weights=None, param_grads=True):
        eng, dev, n = self.eng, self.eng.device, self.eng.n
        w = np.ones(self.n_frames) if weights is None else np.asarray(weights, dtype=np.float64)
        eng.set_param_grads(param_grads)
        eng.set_zero_guess(False)
        U = torch.zeros((n, 3), dtype=torch.float64, device=dev) if eng.lpol else None
        energies = np.zeros(self.n_frames)
        acc = None
        if param_grads:
            acc = {"Q_local": torch.zeros((n, 9), dtype=torch.float64, device=dev),
                   "pol": torch.zeros(n, dtype=torch.float64, device=dev),
                   "thole": torch.zeros(n, dtype=torch.float64, device=dev)}
        self.last_iters = []
        for f in range(self.n_frames):
            pos = self.pos[f]
            eng.rebuild_internal_pairs(pos, self.boxes[f])
            res, _, Uf = eng.compute(pos, self.boxes[f], U=U)
            if eng.lpol:
                U = Uf.clone()  # warm start of the next frame
            energies[f] = res.energy
            self.last_iters.append(int(res.n_iter))
            if param_grads and w[f] != 0.0:
                pg = eng.param_grads()
                for k in acc:
                    acc[k].add_(pg[k], alpha=float(w[f]))
        return energies, acc
