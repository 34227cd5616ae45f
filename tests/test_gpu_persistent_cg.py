"""The whole CG dipole solve in one persistent cooperative launch (k_cg_solve) against the
graph-replayed per-pass solve of the same engine (cuFFT convolution) on serving-stream boxes with
composite and prime meshes, against the float64 oracle on a small box, its iteration count, and
the bounded grid-barrier wait: a barrier that waits for an arrival that never comes returns
DMFFB_TIMEOUT and leaves the engine usable."""
import numpy as np
import pytest
import torch

from dmff_b200 import _lib as L
from dmff_b200.synthetic import serving_system, water_box
from tests.helpers import make_engine, oracle_pairs, oracle_reference, rel_force_rms

pytestmark = pytest.mark.gpu


def _solve(eng, s, persistent):
    eng.set_persistent_cg(persistent)
    eng.set_zero_guess(True)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.rebuild_internal_pairs(pos, s["box"])
    res, F, U = eng.compute(pos, s["box"])
    torch.cuda.synchronize()
    return res, F.cpu().numpy().copy(), U.cpu().numpy().copy(), eng.persistent_cg_blocks()


@pytest.mark.parametrize("n_waters", [150, 300, 700, 2300, 3900])
def test_persistent_solve_matches_per_pass_solve(n_waters):
    """Meshes 17^3 (prime), 21^3, 28^3, 42^3, 49^3."""
    s = serving_system(n_waters, 700 + n_waters)
    eng = make_engine(s, precision="fp32", cg_tol=1e-7)
    r0, F0, U0, b0 = _solve(eng, s, False)
    r1, F1, U1, b1 = _solve(eng, s, True)
    assert b0 == 0 and b1 > 0, (b0, b1)
    assert r1.converged == 1
    # the persistent solve tests convergence every iteration, the per-pass one at the steps its
    # residual decay predicts
    assert r1.n_iter <= r0.n_iter
    assert abs(r1.energy - r0.energy) <= 2e-6 * abs(r0.energy), (s["K"], r1.energy, r0.energy)
    assert rel_force_rms(F1, F0) < 1e-5
    assert np.abs(U1 - U0).max() <= 1e-5 * np.abs(U0).max()


def test_persistent_solve_small_box_matches_oracle():
    s = water_box(64, 12.4, seed=62, lmax=2, pol=True, rc=6.0)
    pr = oracle_pairs(s)
    ref = oracle_reference(s, pr, solver="cg", tol=1e-9)
    eng = make_engine(s, precision="fp32", cg_tol=1e-7)
    res, F, U, b = _solve(eng, s, True)
    assert b > 0
    assert abs(res.energy - ref["E"]) <= 1e-5 * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= 1e-4
    assert np.abs(U - ref["U"]).max() <= 1e-4 * np.abs(ref["U"]).max()


def test_barrier_wait_runs_out_and_engine_stays_usable():
    """The first grid barrier waits for one arrival more than the grid has: every wait runs out
    after 20 ms, the solve returns DMFFB_TIMEOUT, and the next solve (normal barrier) succeeds."""
    s = serving_system(300, 9001)
    eng = make_engine(s, precision="fp32", cg_tol=1e-7)
    r_ok, F_ok, _, _ = _solve(eng, s, True)
    eng.set_cg_wait_limit(0.02, phantom_arrivals=1)
    with pytest.raises(L.EngineError) as e:
        _solve(eng, s, True)
    assert e.value.status == L.DMFFB_TIMEOUT
    eng.set_cg_wait_limit(2.0)
    r2, F2, _, _ = _solve(eng, s, True)
    assert r2.converged == 1
    # the same solve again (atomic accumulation order aside)
    assert abs(r2.energy - r_ok.energy) <= 1e-6 * abs(r_ok.energy)
    assert rel_force_rms(F2, F_ok) < 1e-5
