"""The single-pass neighbour build (k_pairs_cell pass 2 into per-atom slots, then k_ell_compact),
which an engine uses from its second build on, against the two-pass build (count pass, scans,
fill pass) of a fresh engine: the same half rows (as a set: the order of an atom's rows follows
the cell fill's atomics in both builds), and through the CSR the same dipole solve, energy and
forces; a denser box than the slots were sized for falls back to the two passes."""
import numpy as np
import pytest
import torch

from dmff_b200.synthetic import water_box
from tests.helpers import make_engine, rel_force_rms

pytestmark = pytest.mark.gpu


def _build(eng, pos, box):
    eng.rebuild_internal_pairs(pos, box)
    rows = eng.internal_pairs().cpu().numpy().copy()
    # rows come sorted by i; within an atom the order is not fixed
    assert np.all(np.diff(rows[:, 0]) >= 0)
    return rows[np.lexsort((rows[:, 1], rows[:, 0]))]


def _compute(eng, pos, box):
    eng.set_zero_guess(True)
    res, F, U = eng.compute(pos, box)
    torch.cuda.synchronize()
    return res, F.cpu().numpy().copy()


def _fresh(s, pos, box):
    e = make_engine(s, precision="fp64", cg_tol=1e-10)
    e.set_persistent_cg(False)
    rows = _build(e, pos, box)
    return rows, _compute(e, pos, box)


def test_single_pass_matches_two_pass_build():
    s = water_box(1500, 35.5, seed=5, lmax=2, pol=True, rc=8.0)
    box = s["box"]
    pos0 = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng = make_engine(s, precision="fp64", cg_tol=1e-10)
    eng.set_persistent_cg(False)
    rows0 = _build(eng, pos0, box)  # two passes; sizes the slots
    rows1 = _build(eng, pos0, box)  # single pass
    assert rows0.shape[0] > 100_000
    assert np.array_equal(rows0, rows1)
    rng = np.random.default_rng(2)
    pos1 = pos0 + torch.tensor(rng.normal(0.0, 0.08, size=s["pos"].shape), device="cuda")
    rows2 = _build(eng, pos1, box)  # single pass at new positions
    r2, F2 = _compute(eng, pos1, box)
    ref_rows, (rr, Fr) = _fresh(s, pos1, box)
    assert np.array_equal(rows2, ref_rows)
    assert r2.n_pairs == rr.n_pairs
    assert abs(r2.energy - rr.energy) <= 1e-10 * abs(rr.energy)
    assert rel_force_rms(F2, Fr) <= 1e-9


def test_single_pass_overflow_falls_back_to_two_passes():
    s = water_box(1500, 35.5, seed=6, lmax=2, pol=True, rc=8.0)
    eng = make_engine(s, precision="fp64", cg_tol=1e-10)
    eng.set_persistent_cg(False)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    _build(eng, pos, s["box"])  # sizes the slots for this density
    # the same atoms in a box 0.92 times as wide: 1.28 times the neighbours per atom, past the slots
    box2 = s["box"] * 0.92
    pos2 = pos * 0.92
    rows = _build(eng, pos2, box2)
    r, F = _compute(eng, pos2, box2)
    ref_rows, (rr, Fr) = _fresh(s, pos2, box2)
    assert np.array_equal(rows, ref_rows)
    assert abs(r.energy - rr.energy) <= 1e-10 * abs(rr.energy)
    assert rel_force_rms(F, Fr) <= 1e-9
    # the next build at the new density takes the single pass with the resized slots
    assert np.array_equal(_build(eng, pos2, box2), ref_rows)
