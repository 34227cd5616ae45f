"""The dipole solve's step schedule: each CG step takes the parity of its r.z slot from a step
counter on the device, so a two-step and a one-step CUDA graph are captured (on the second solve
with the same pointers and box) and mixed freely, and the last segment ends at the first step the
residual decay predicts to converge.  Three solves of one engine (direct launches, capture and
replay, replay) and a solve with graphs off agree, including solves that need an odd number of
steps (the one-step graph)."""
import numpy as np
import pytest
import torch

from dmff_b200.synthetic import serving_system
from tests.helpers import make_engine, rel_force_rms

pytestmark = pytest.mark.gpu


def _solve(eng, s, pos):
    res, F, U = eng.compute(pos, s["box"])
    torch.cuda.synchronize()
    return res, F.cpu().numpy().copy(), U.cpu().numpy().copy()


def test_graph_replay_matches_direct_launches_with_odd_step_counts():
    s = serving_system(400, 11)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    counts = []
    for tol in (1e-6, 1e-7, 1e-8, 1e-9, 1e-10):
        eng = make_engine(s, precision="fp64", cg_tol=tol)
        eng.set_persistent_cg(False)
        eng.set_zero_guess(True)
        eng.rebuild_internal_pairs(pos, s["box"])
        runs = [_solve(eng, s, pos) for _ in range(3)]
        ref = make_engine(s, precision="fp64", cg_tol=tol)
        ref.set_persistent_cg(False)
        ref.set_zero_guess(True)
        assert ref.lib.dmffb_set_graphs(ref.h, 0) == 0
        ref.rebuild_internal_pairs(pos, s["box"])
        r0, F0, U0 = _solve(ref, s, pos)
        counts.append(r0.n_iter)
        for r, F, U in runs:
            assert r.converged == 1 and r.n_iter == r0.n_iter, (tol, r.n_iter, r0.n_iter)
            assert abs(r.energy - r0.energy) <= 1e-12 * abs(r0.energy)
            assert rel_force_rms(F, F0) <= 1e-11
            assert np.abs(U - U0).max() <= 1e-11 * np.abs(U0).max()
    # the tolerances span several step counts, odd ones among them
    assert any(c % 2 == 1 for c in counts), counts
    assert len(set(counts)) >= 3, counts
