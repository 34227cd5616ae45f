"""Edge cases of the ADMP path on the GPU against the float64 oracle: a triclinic (reduced,
OpenMM-style) box, molecules shifted by lattice vectors far outside the box, and an empty pair
list (reciprocal and self terms only)."""
import numpy as np
import pytest
import torch

from dmff_b200.synthetic import water_box
from tests.helpers import make_engine, oracle_pairs, oracle_reference, rel_force_rms

pytestmark = pytest.mark.gpu


def _sheared(s, shear):
    """Rigid molecules on a sheared lattice: each molecule is translated so that its oxygen moves
    from fractional coordinates of the cubic box to the same fractional coordinates of
    box = [[L, 0, 0], [a L, L, 0], [b L, c L, L]] (rows = lattice vectors, same volume)."""
    L = s["box"][0, 0]
    a, b, c = shear
    box = np.array([[L, 0.0, 0.0], [a * L, L, 0.0], [b * L, c * L, L]])
    mol = s["pos"].reshape(-1, 3, 3)
    o = mol[:, 0, :]
    on = (o / L) @ box
    return dict(s, pos=(mol - o[:, None, :] + on[:, None, :]).reshape(-1, 3), box=box)


def _run(eng, s, pairs=None):
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    if eng.lpol:
        eng.U.zero_()
    pr = None if pairs is None else torch.tensor(pairs, dtype=torch.int32, device="cuda")
    res, F, _ = eng.compute(pos, s["box"], pairs=pr)
    return res, F.cpu().numpy().copy()


@pytest.mark.parametrize("pol,shear", [(False, (0.25, -0.15, 0.2)), (True, (0.1, -0.08, 0.05))])
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_triclinic_box(pol, shear, prec):
    s = _sheared(water_box(216, 18.6, seed=31, lmax=2, pol=pol, rc=6.0), shear)
    pr = oracle_pairs(s)
    ref = oracle_reference(s, pr)
    eng = make_engine(s, precision=prec, cg_tol=1e-8)
    res, F = _run(eng, s)  # engine-built cell list on the sheared cells
    assert res.n_pairs == len(pr)
    tol_e, tol_f = (1e-9, 1e-7) if prec == "fp64" else (1e-5, 1e-4)
    # the total can cancel almost completely (random multipoles on a sheared lattice); the FP32
    # bound is relative to the largest of the real, reciprocal and self terms it is made of
    scale = abs(ref["E"]) if prec == "fp64" else max(abs(res.e_real), abs(res.e_recip), abs(res.e_self))
    assert abs(res.energy - ref["E"]) <= tol_e * scale
    assert rel_force_rms(F, ref["F"]) <= tol_f


@pytest.mark.parametrize("pol", [False, True])
def test_lattice_shifts_far_outside_the_box(pol):
    """Energy and forces do not change when whole molecules move by integer lattice vectors
    (up to three boxes in each direction, negative included)."""
    s = _sheared(water_box(216, 18.6, seed=32, lmax=2, pol=pol, rc=6.0), (0.2, -0.1, 0.15))
    eng = make_engine(s, precision="fp64", cg_tol=1e-10)
    res0, F0 = _run(eng, s)
    rng = np.random.default_rng(7)
    shift = rng.integers(-3, 4, size=(216, 3)) @ s["box"]
    s2 = dict(s, pos=(s["pos"].reshape(-1, 3, 3) + shift[:, None, :]).reshape(-1, 3))
    res1, F1 = _run(eng, s2)
    assert res1.n_pairs == res0.n_pairs
    assert abs(res1.energy - res0.energy) <= 1e-9 * abs(res0.energy)
    assert rel_force_rms(F1, F0) <= 1e-8


@pytest.mark.parametrize("pol", [False, True])
def test_empty_pair_list(pol):
    """Zero pair rows: the real-space kernels launch nothing and the reciprocal, self (and
    polarization) terms match the oracle given the same empty list."""
    s = water_box(64, 12.4, seed=33, lmax=2, pol=pol, rc=5.0)
    empty = np.zeros((0, 3), dtype=np.int64)
    ref = oracle_reference(s, empty)
    eng = make_engine(s, precision="fp64", cg_tol=1e-10)
    res, F = _run(eng, s, pairs=empty)
    assert res.n_pairs == 0
    assert abs(res.energy - ref["E"]) <= 1e-9 * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= 1e-7
