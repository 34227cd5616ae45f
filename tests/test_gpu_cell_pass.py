"""The classical cell pass (pairs straight from the cell grid, no pair list) against the float64
oracle on the brute-force pair set, and against the list path of the same engine at the density of
the 100 000-atom polymer + water box (rc 10 A)."""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.synthetic import pairs_nbond, polymer_water_box
from helpers import rel_force_rms
from test_gpu_classical import _engine, _oracle_synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("coulomb", ["pme", "rf"])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cell_pass_matches_oracle(precision, coulomb):
    """4 chains x 20 beads + 500 waters, 24.6 A box, rc 8 A (6 half-width cells per axis)."""
    s = polymer_water_box(4, 20, 500, 24.6, seed=4, rc=8.0)
    pairs = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    assert np.count_nonzero(pairs[:, 2]) > 0
    ref = _oracle_synth(s, pairs, coulomb)
    eng = _engine(s, precision, coulomb)
    eng.set_cell_pass(True)
    res, F = eng.compute(torch.tensor(s["pos"], device="cuda"), s["box"])
    assert res.n_pairs == len(pairs)
    tol_e = 1e-10 if precision == "fp64" else 1e-5
    assert abs(res.energy - ref["E"]) <= tol_e * abs(ref["E"])
    assert abs(res.e_lj - ref["El"]) <= tol_e * abs(ref["El"])
    assert rel_force_rms(F.cpu().numpy(), ref["F"]) < (1e-10 if precision == "fp64" else 1e-4)
    bg = np.array(res.box_grad).reshape(3, 3)
    assert np.abs(bg - ref["box_grad"]).max() <= (1e-8 if precision == "fp64" else 1e-4) * np.abs(ref["box_grad"]).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cell_pass_matches_list_path_at_classical_box_density(precision):
    """A 40 A block at the 100k-atom box's density (~11 M pairs): the cell pass and the list path
    (build the engine's list, then compute on it) give the same pair count, energies, forces and box
    gradient; moving the atoms and computing again follows the new positions."""
    scale = (40.0 / 70.0) ** 3
    s = polymer_water_box(int(round(200 * scale)), 50, int(round(30000 * scale)), 40.0, seed=4, rc=10.0, ethresh=1e-5)
    pos = torch.tensor(s["pos"], device="cuda")
    lst = _engine(s, precision)
    cel = _engine(s, precision)
    cel.set_cell_pass(True)
    rng = np.random.default_rng(3)
    for step in range(2):
        lst.rebuild_internal_pairs(pos, s["box"])
        r1, F1 = lst.compute(pos, s["box"])
        F1 = F1.cpu().numpy().copy()
        r2, F2 = cel.compute(pos, s["box"])
        F2 = F2.cpu().numpy().copy()
        assert r2.n_pairs == r1.n_pairs > 10_000_000
        tol = 1e-11 if precision == "fp64" else 2e-6
        for k in ("e_coul_real", "e_lj", "energy"):
            assert abs(getattr(r2, k) - getattr(r1, k)) <= tol * abs(getattr(r1, k)), k
        assert rel_force_rms(F2, F1) < (1e-11 if precision == "fp64" else 1e-5)
        b1, b2 = np.array(r1.box_grad), np.array(r2.box_grad)
        assert np.abs(b2 - b1).max() <= (1e-10 if precision == "fp64" else 1e-5) * np.abs(b1).max()
        pos = pos + torch.tensor(rng.normal(0.0, 0.05, size=s["pos"].shape), device="cuda")


def test_cell_pass_matches_list_path_triclinic():
    """The same comparison in a sheared box (the cell pass's triclinic stencil bounds): 32 A block
    at the classical box's density, box rows (32, 0, 0), (5, 32, 0), (-4, 6, 32)."""
    scale = (32.0 / 70.0) ** 3
    s = polymer_water_box(int(round(200 * scale)), 50, int(round(30000 * scale)), 32.0, seed=9, rc=10.0, ethresh=1e-5)
    frac = s["pos"] @ np.linalg.inv(s["box"])
    box = np.array([[32.0, 0.0, 0.0], [5.0, 32.0, 0.0], [-4.0, 6.0, 32.0]])
    pos = torch.tensor(frac @ box, device="cuda")
    s = dict(s, box=box)
    lst = _engine(s, "fp32")
    cel = _engine(s, "fp32")
    cel.set_cell_pass(True)
    lst.rebuild_internal_pairs(pos, box)
    r1, F1 = lst.compute(pos, box)
    F1 = F1.cpu().numpy().copy()
    r2, F2 = cel.compute(pos, box)
    F2 = F2.cpu().numpy().copy()
    assert r2.n_pairs == r1.n_pairs > 1_000_000
    for k in ("e_coul_real", "e_lj", "energy"):
        assert abs(getattr(r2, k) - getattr(r1, k)) <= 2e-6 * abs(getattr(r1, k)), k
    assert rel_force_rms(F2, F1) < 1e-5
