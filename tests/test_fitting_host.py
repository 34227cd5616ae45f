"""The fitting front end (dmff/mbar.py:27-92 semantics) on the CPU with a stand-in potential:
per-frame energies in the frame order, the NPT pressure-volume term, reduced energies at a
temperature, and autograd from the reduced energies back to the parameters."""
import numpy as np
import torch

from dmff_b200.fitting import PV_KJMOL_PER_BAR_NM3, TargetState, buildTrajEnergyFunction


def test_traj_energy_function_and_target_state():
    rng = np.random.default_rng(0)
    F, n = 4, 5
    traj = {"xyz": rng.normal(size=(F, n, 3)), "unitcell_vectors": np.stack([np.eye(3) * (2.0 + 0.1 * f) for f in range(F)]),
            "unitcell_volumes": np.array([(2.0 + 0.1 * f) ** 3 for f in range(F)])}
    k = torch.tensor(1.7, dtype=torch.float64, requires_grad=True)
    seen = []

    def potential(pos, box, pairs, params):
        seen.append(None if pairs is None else int(len(pairs)))
        return params["k"] * (pos ** 2).sum() + box[0, 0]

    cov = np.zeros((n, n), dtype=int)
    efun = buildTrajEnergyFunction(potential, cov, 0.5, usePBC=False, ensemble="npt", pressure=2.0)
    e = efun(traj, {"k": k})
    assert len(e) == F and seen == [n * (n - 1) // 2] * F
    for f in range(F):
        want = 1.7 * (traj["xyz"][f] ** 2).sum() + traj["unitcell_vectors"][f, 0, 0] + \
            2.0 * PV_KJMOL_PER_BAR_NM3 * traj["unitcell_volumes"][f]
        assert abs(float(e[f]) - want) < 1e-12
    u = TargetState(300.0, efun).calc_energy(traj, {"k": k})
    beta = 1.0 / 300.0 / 8.314 * 1000.0
    assert torch.allclose(u, beta * torch.stack([torch.as_tensor(x) for x in e]))
    (g,) = torch.autograd.grad(u.sum(), k)
    assert abs(float(g) - beta * sum((traj["xyz"][f] ** 2).sum() for f in range(F))) < 1e-9
