"""Trajectory-batched evaluation for fitting on the GPU: per-frame energies and the weighted sum of
per-atom parameter adjoints over the frames of a trajectory (one engine, device cell list per
frame, dipoles warm-started from the previous frame) against independent per-frame evaluations
and the float64 oracle, and the per-type gradient of the weighted loss against finite
differences (the consumer of dmff/mbar.py:27-92 and dmff/optimize.py:30-84)."""
import numpy as np
import pytest
import torch

from dmff_b200.fitting import TrajectoryEvaluator
from dmff_b200.synthetic import water_box
from tests.helpers import make_engine, oracle_pairs, oracle_reference

pytestmark = pytest.mark.gpu


def _frames(s, F, seed=4, sigma=0.03):
    rng = np.random.default_rng(seed)
    pos = [s["pos"]]
    for _ in range(F - 1):
        pos.append(pos[-1] + rng.normal(0.0, sigma, size=s["pos"].shape))
    return np.stack(pos), np.stack([s["box"]] * F)


def test_trajectory_energies_and_weighted_adjoints():
    s = water_box(216, 18.6, seed=71, lmax=2, pol=True, rc=6.0)
    # small steps between frames: each frame's solve starts close to its solution
    P, B = _frames(s, 8, sigma=0.002)
    w = np.linspace(0.5, 1.5, 8)
    eng = make_engine(s, precision="fp64", cg_tol=1e-11)
    ev = TrajectoryEvaluator(eng, P, B)
    E, acc = ev.evaluate(weights=w)
    # independent per-frame evaluations from zero dipoles
    ref = make_engine(s, precision="fp64", cg_tol=1e-11)
    ref.set_param_grads(True)
    ref.set_zero_guess(True)
    want = {k: 0.0 for k in acc}
    cold_iters = []
    for f in range(8):
        pos = torch.tensor(P[f], device="cuda")
        ref.rebuild_internal_pairs(pos, B[f])
        r, _, _ = ref.compute(pos, B[f])
        cold_iters.append(int(r.n_iter))
        assert abs(E[f] - r.energy) <= 1e-9 * abs(r.energy)
        pg = ref.param_grads()
        for k in want:
            want[k] = want[k] + w[f] * pg[k].cpu().numpy()
    # frames 1.. start from the previous frame's dipoles: fewer CG iterations than from zero
    assert ev.last_iters[0] == cold_iters[0]
    assert sum(ev.last_iters[1:]) < sum(cold_iters[1:]), (ev.last_iters, cold_iters)
    for k in want:
        got = acc[k].cpu().numpy()
        assert np.abs(got - want[k]).max() <= 1e-7 * np.abs(want[k]).max(), k
    # two frames against the float64 oracle
    for f in (0, 7):
        sf = dict(s, pos=P[f])
        o = oracle_reference(sf, oracle_pairs(sf), tol=1e-10)
        assert abs(E[f] - o["E"]) <= 1e-9 * abs(o["E"])


def test_weighted_loss_per_type_gradient_vs_finite_differences():
    """d/d(pol of oxygen) of sum_f w_f E_f: the accumulated per-atom adjoints summed over the
    oxygens against central differences of the loss (FP64, dipoles re-solved per frame)."""
    s = water_box(64, 12.4, seed=72, lmax=2, pol=True, rc=6.0)
    P, B = _frames(s, 5, seed=5)
    w = np.array([1.0, -0.5, 2.0, 0.25, 1.0])
    eng = make_engine(s, precision="fp64", cg_tol=1e-12)
    E, acc = TrajectoryEvaluator(eng, P, B).evaluate(weights=w)
    g = float(acc["pol"].cpu().numpy()[s["types"] == 0].sum())
    h = 1e-5

    def loss(pol_O):
        e2 = make_engine(s, precision="fp64", cg_tol=1e-12)
        pol = np.where(s["types"] == 0, pol_O, 0.5)
        e2.set_params(s["Q_local"], pol, s["thole"])
        Ef, _ = TrajectoryEvaluator(e2, P, B).evaluate(param_grads=False)
        return float(np.dot(w, Ef))

    fd = (loss(1.0 + h) - loss(1.0 - h)) / (2 * h)
    assert abs(g - fd) <= 1e-6 * abs(fd)
