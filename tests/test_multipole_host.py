"""Multipole conversions and frame rotations (``dmff_b200.admp.multipole``, the names of
dmff/admp/multipole.py) against the oracle's restatement of the reference on random frames."""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.admp import multipole as M


def _frames(n, seed):
    q, _ = np.linalg.qr(np.random.default_rng(seed).standard_normal((n, 3, 3)))
    return torch.tensor(q)


def test_conversions_match_oracle_and_invert():
    rng = np.random.default_rng(1)
    T = torch.tensor(rng.standard_normal((40, 10)))
    for lmax, nc in ((0, 1), (1, 4), (2, 10)):
        Q = M.convert_cart2harm(T[:, :nc], lmax)
        assert Q.shape == (40, (lmax + 1) ** 2)
        assert torch.equal(Q, R.convert_cart2harm(T[:, :nc], lmax))
        assert torch.equal(M.convert_harm2cart(Q, lmax), R.convert_harm2cart(Q, lmax))
    # harm -> cart -> harm is the identity (traceless quadrupoles)
    Q = torch.tensor(rng.standard_normal((40, 9)))
    assert (M.convert_cart2harm(M.convert_harm2cart(Q, 2), 2) - Q).abs().max() < 1e-14
    with pytest.raises(ValueError):
        M.convert_cart2harm(T, 3)


@pytest.mark.parametrize("lmax", [0, 1, 2])
def test_rotations_match_oracle(lmax):
    F = _frames(64, lmax)
    Q = torch.tensor(np.random.default_rng(7).standard_normal((64, (lmax + 1) ** 2)))
    for name in ("rot_global2local", "rot_local2global"):
        got, want = getattr(M, name)(Q, F, lmax), getattr(R, name)(Q, F, lmax)
        # the reference's closed-form l=2 matrix carries its truncated sqrt(3) (1.73205080757)
        assert (got - want).abs().max() <= 1e-10 * max(1.0, want.abs().max().item())
    back = M.rot_local2global(M.rot_global2local(Q, F, lmax), F, lmax)
    assert (back - Q).abs().max() < 1e-13
    if lmax >= 1:
        U = Q[:, 1:4]
        assert torch.equal(M.rot_ind_global2local(U, F), R.rot_ind_global2local(U, F))


def test_rotation_keeps_quadrupole_invariants():
    """|Q_l2| (the Frobenius norm of the traceless tensor) does not depend on the frame."""
    F = _frames(16, 3)
    Q = torch.tensor(np.random.default_rng(4).standard_normal((16, 9)))
    Ql = M.rot_global2local(Q, F)
    tg = M.convert_harm2cart(Q, 2)[:, 4:10]
    tl = M.convert_harm2cart(Ql, 2)[:, 4:10]
    norm = lambda t: (t[:, :3] ** 2).sum(1) + 2 * (t[:, 3:] ** 2).sum(1)
    assert torch.allclose(norm(tg), norm(tl), rtol=1e-12, atol=0)
    with pytest.raises(NotImplementedError):
        M.rot_global2local(torch.zeros((1, 16)), F[:1], 3)
