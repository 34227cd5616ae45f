"""The oracle's exact second-order reference (implicit differentiation of the converged dipoles
through double autograd) against central finite differences of the oracle itself: the
derivatives of a force loss L = <w, dE/dpos> with respect to parameters and positions, the dipoles
re-solved at every displaced point."""
import numpy as np

from dmff_b200.synthetic import water_box
from tests.helpers import oracle_force_loss_grads, oracle_pairs, oracle_reference


def test_oracle_force_loss_gradients_match_finite_differences():
    s = water_box(27, 9.3, seed=24, lmax=2, pol=True, rc=4.6)
    pr = oracle_pairs(s)
    w = np.random.default_rng(5).normal(size=(s["n_atoms"], 3))
    ex = oracle_force_loss_grads(s, pr, w)

    def loss(sd):
        return float(np.sum(w * -oracle_reference(sd, pr, tol=1e-12)["F"]))

    h = 1e-5
    for key, ek, idx in [("pol", "pol", (0,)), ("Q_local", "Q", (1, 4)), ("pos", "pos", (5, 1))]:
        sp = dict(s, **{key: s[key].copy()})
        sm = dict(s, **{key: s[key].copy()})
        sp[key][idx] += h
        sm[key][idx] -= h
        fd = (loss(sp) - loss(sm)) / (2 * h)
        assert abs(fd - ex[ek][idx]) <= 1e-6 * abs(fd), (key, fd, ex[ek][idx])
