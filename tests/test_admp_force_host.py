"""Host logic of ``ADMPPmeForce`` (dmff/admp/pme.py:36-245) with a stand-in engine that records
what the force hands down: the nm <-> Angstrom handling of the induced dipoles, the aux entries,
``get_forces`` and ``update_env``."""
from types import SimpleNamespace

import numpy as np
import torch

from dmff_b200.admp.pme import ADMPPmeForce


class _Recorder:
    device = torch.device("cpu")

    def __init__(self):
        self.U_in = []

    def set_param_grads(self, on):
        pass

    def set_params(self, *args):
        pass

    def compute(self, pos, box, pairs=None, U=None):
        self.U_in.append(None if U is None else U.clone())
        res = SimpleNamespace(energy=-12.5, converged=1, n_iter=7, box_grad=[0.0] * 9)
        forces = torch.ones_like(pos) * 0.25
        return res, forces, (U + 1.0 if U is not None else None)


def _force(lpol=True):
    n = 6
    f = ADMPPmeForce(np.eye(3) * 20.0, np.zeros(n, int), np.zeros(n, int), np.zeros((n, 3), int), 8.0, 5e-4, 2,
                     lpol=lpol)
    rec = _Recorder()
    f._engine = rec
    ms, ps, ds = [0, 0, 0, 1, 1, 1], [0, 0, 0, 1, 1, 1], [0, 0, 0, 1, 1, 1]
    f._scales = (tuple(np.asarray(ms, np.float64)), tuple(np.asarray(ps, np.float64)) if lpol else None,
                 tuple(np.asarray(ds, np.float64)) if lpol else None)
    return f, rec, n, ms, ps, ds


def test_induced_dipoles_are_nm_at_the_interface():
    f, rec, n, ms, ps, ds = _force()
    pos = torch.zeros((n, 3), dtype=torch.float64)
    Q = torch.zeros((1, 9), dtype=torch.float64)
    U_nm = torch.full((n, 3), 0.02, dtype=torch.float64)
    E, aux = f.get_energy(pos, torch.eye(3) * 20, None, Q, torch.ones(1), torch.ones(1), ms, ps, ds,
                          U_init=U_nm, aux={})
    assert E.item() == -12.5
    assert torch.allclose(rec.U_in[-1], U_nm * 10.0)  # pme.py:208: U_init * 10 (nm -> Angstrom)
    assert torch.allclose(aux["U_ind"], (U_nm * 10.0 + 1.0) * 0.1)  # pme.py:225: back to nm
    assert aux["lconverg"] is True and aux["n_cycle"] == 7
    E2 = f.get_energy(pos, torch.eye(3) * 20, None, Q, torch.ones(1), torch.ones(1), ms, ps, ds)
    assert torch.is_tensor(E2) and not rec.U_in[-1].any()  # default U_init: zeros


def test_get_forces_and_update_env():
    f, rec, n, ms, ps, ds = _force(lpol=False)
    pos = np.zeros((n, 3))
    Q = torch.zeros((1, 9), dtype=torch.float64)
    E, g = f.get_forces(pos, torch.eye(3) * 20, None, Q, ms)
    assert E.item() == -12.5
    assert torch.allclose(g, torch.full((n, 3), -0.25, dtype=torch.float64))  # dE/dx = -F
    assert f.generate_get_energy()(pos, torch.eye(3) * 20, None, Q, ms).item() == -12.5
    f.update_env("kappa", 0.41)
    assert f.kappa == 0.41 and f._engine is None and f._scales is None


class _DispRecorder:
    device = torch.device("cpu")

    def __init__(self, n, mscales):
        self.n, self.mscales = n, mscales

    def set_params(self, *args):
        pass

    def set_param_grads(self, on):
        pass

    def compute(self, pos, box, pairs=None):
        res = SimpleNamespace(energy=3.0, e_sr=5.0, box_grad=[0.0] * 9, box_grad_sr=[0.0] * 9)
        return res, (torch.ones_like(pos) * 0.5, torch.ones_like(pos) * 2.0)


def test_disp_force_calculators():
    from dmff_b200.admp.disp_pme import ADMPDispPmeForce
    n, ms = 4, [0.0, 0.0, 0.0, 1.0, 1.0, 1.0]
    f = ADMPDispPmeForce(np.eye(3) * 20.0, 8.0, 5e-4, 10)
    f._engine = _DispRecorder(n, tuple(ms))
    c = torch.ones((n, 3), dtype=torch.float64)
    E, g = f.get_forces(np.zeros((n, 3)), torch.eye(3) * 20, None, c, ms)
    assert E.item() == 3.0 and torch.allclose(g, torch.full((n, 3), -0.5, dtype=torch.float64))
    assert f.generate_get_energy()(torch.zeros((n, 3)), torch.eye(3) * 20, None, c, ms).item() == 3.0
    f.update_env("kappa", 0.3)
    assert f.kappa == 0.3 and f._engine is None
