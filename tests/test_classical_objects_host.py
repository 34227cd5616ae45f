"""Host side of the dmff/classical/inter.py and intra.py force objects (``dmff_b200.classical.inter``
/ ``.intra``): the long-range dispersion correction (host torch arithmetic) against the oracle,
argument checks, and the closures' behaviour that needs no GPU."""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.classical.inter import (CoulNoCutoffForce, CoulombPMEForce, CoulReactionFieldForce,
                                       LennardJonesForce, LennardJonesLongRangeForce, ONE_4PI_EPS0)
from dmff_b200.classical.intra import HarmonicAngleJaxForce, HarmonicBondJaxForce, PeriodicTorsionJaxForce


def _count_matrix(map_prm, n_types):
    cnt = np.bincount(map_prm, minlength=n_types)
    cm = np.outer(cnt, cnt).astype(np.float64)
    cm[np.diag_indices(n_types)] = cnt * (cnt - 1) / 2
    return np.triu(cm)


def test_long_range_correction_matches_oracle():
    rng = np.random.default_rng(5)
    n_types, n = 4, 300
    map_prm = rng.integers(0, n_types, n)
    cm = _count_matrix(map_prm, n_types)
    eps = torch.tensor(rng.uniform(0.1, 0.9, n_types), requires_grad=True)
    sig = torch.tensor(rng.uniform(0.25, 0.35, n_types), requires_grad=True)
    box = torch.tensor(np.diag([3.1, 3.2, 3.3]) + 0.05 * rng.standard_normal((3, 3)), requires_grad=True)
    f = LennardJonesLongRangeForce(0.9, map_prm, np.zeros((0, 3), dtype=int), cm)
    E = f.generate_get_energy()(box, eps, sig, torch.zeros(0), torch.zeros(0))
    Eo = R.lj_dispersion_correction(box, eps, sig, map_prm, cm, 0.9)
    assert abs(E.item() - Eo.item()) <= 1e-14 * abs(Eo.item())
    g = torch.autograd.grad(E, (box, eps, sig))
    go = torch.autograd.grad(Eo, (box, eps, sig))
    for x, y in zip(g, go):
        np.testing.assert_allclose(x.numpy(), y.numpy(), rtol=1e-12, atol=0)


def test_long_range_correction_nbfix_sets_one_orientation():
    """An NBFix row (t1, t2, k) replaces eps/sigma of the (t1, t2) entry only, as inter.py:121-122
    does; with the upper-triangular count matrix only t1 <= t2 rows contribute."""
    map_prm = np.array([0, 0, 1, 1, 1, 2])
    cm = _count_matrix(map_prm, 3)
    f64 = lambda x: torch.tensor(x, dtype=torch.float64)
    eps, sig = f64([0.2, 0.5, 0.3]), f64([0.3, 0.32, 0.28])
    box = torch.eye(3, dtype=torch.float64) * 2.5
    base = LennardJonesLongRangeForce(1.0, map_prm, None, cm).generate_get_energy()(box, eps, sig, None, None)
    fixed = LennardJonesLongRangeForce(1.0, map_prm, np.array([[0, 1, 0]]), cm).generate_get_energy()(
        box, eps, sig, f64([0.7]), f64([0.4]))
    c6 = lambda e, s: 4 * e * s ** 6
    delta = (c6(0.7, 0.4) - c6(np.sqrt(0.2 * 0.5), 0.31)) * cm[0, 1] / cm.sum()
    scale = -2.0 / 3.0 * np.pi * 36 / 2.5 ** 3 / 1.0 ** 3
    assert abs((fixed - base).item() - scale * delta) <= 1e-12 * abs(scale * delta)
    swapped = LennardJonesLongRangeForce(1.0, map_prm, np.array([[1, 0, 0]]), cm).generate_get_energy()(
        box, eps, sig, f64([0.7]), f64([0.4]))
    assert abs((swapped - base).item()) <= 1e-15 * abs(base.item())  # lower triangle: count 0


def test_constructor_checks():
    with pytest.raises(NotImplementedError):
        LennardJonesForce(0.8, 1.0, [0, 1], [], isSwitch=True)
    with pytest.raises(ValueError):
        CoulombPMEForce(1.0, np.zeros(3), 3.0, (10, 10, 10), pme_order=4)
    rf = CoulReactionFieldForce(1.2, np.zeros(3), epsilon_solv=78.5)
    assert rf.krf == pytest.approx((78.5 - 1) / (2 * 78.5 + 1) / 1.2 ** 3)
    assert rf.crf == pytest.approx(3 * 78.5 / (2 * 78.5 + 1) / 1.2)
    assert ONE_4PI_EPS0 == pytest.approx(138.935455846)


def test_energy_closures_reject_bad_pairs_and_mscales():
    pos, box = torch.zeros((3, 3)), torch.eye(3)
    nc = CoulNoCutoffForce(np.array([0.4, -0.8, 0.4])).generate_get_energy()
    with pytest.raises(ValueError, match="pairs"):
        nc(pos, box, None, [0, 0, 0.5, 1, 1, 1])
    with pytest.raises(ValueError, match="mscales"):
        nc(pos, box, np.array([[0, 1, 1]]), [0, 0, 0.5, 1, 1])
    lj = LennardJonesForce(0.0, 1.0, [0, 1, 1], None).generate_get_energy()
    with pytest.raises(ValueError, match="pairs"):
        lj(pos, box, None, torch.ones(2), torch.ones(2), torch.zeros(0), torch.zeros(0), [0, 0, 0.5, 1, 1, 1])


def test_topology_matrix_closure_signature():
    """With a topology matrix the closure takes bcc (charges = init + T @ bcc), as inter.py:329-333."""
    top = np.array([[1.0, 0.0], [-1.0, 1.0], [0.0, -1.0]])
    f = CoulombPMEForce(1.0, np.array([0.4, -0.8, 0.4]), 3.0, (10, 10, 10), topology_matrix=top)
    q = f._charges(torch.tensor([0.1, 0.2], dtype=torch.float64))
    np.testing.assert_allclose(q.numpy(), [0.5, -0.7, 0.2])
    import inspect
    assert list(inspect.signature(f.generate_get_energy()).parameters) == ["positions", "box", "pairs", "bcc",
                                                                            "mscales"]
    f0 = CoulombPMEForce(1.0, np.array([0.4, -0.8, 0.4]), 3.0, (10, 10, 10))
    assert list(inspect.signature(f0.generate_get_energy()).parameters) == ["positions", "box", "pairs", "mscales"]


def test_bonded_closures_without_terms_and_update_env():
    pos = np.random.default_rng(1).standard_normal((6, 3))
    box = torch.eye(3)
    b = HarmonicBondJaxForce(np.zeros(0, int), np.zeros(0, int), np.zeros(0, int))
    assert float(b.get_energy(pos, box, None, torch.ones(1), torch.ones(1))) == 0.0
    E, g = b.get_forces(pos, box, None, torch.ones(1), torch.ones(1))
    assert float(E) == 0.0 and g.shape == (6, 3) and not g.any()
    t = PeriodicTorsionJaxForce([], [], [], [], [], [])
    assert t.get_energy(pos, box, None, torch.ones(1), torch.ones(1)) == 0.0
    a = HarmonicAngleJaxForce([0], [1], [2], [0])
    # attributes change one at a time; the term list is read at the next energy call
    a.update_env("p1idx", [0, 3])
    a.update_env("p2idx", [1, 4])
    a.update_env("p3idx", [2, 5])
    a.update_env("prmidx", [0, 0])
    assert a.get_energy.__name__ == "get_energy"
