"""Local frames, pair frames and global multipoles on the host (``dmff_b200.admp.spatial``,
``ADMPPmeForce.Q_local_to_global``) against the oracle's restatement of dmff/admp/spatial.py
and pme.py:183-196, over all six axis rules."""
import numpy as np
import torch

import oracle.admp_ref as R
from dmff_b200.admp.pme import ADMPPmeForce
from dmff_b200.admp.spatial import build_quasi_internal, generate_construct_local_frames, pbc_shift


def _sites(seed, n=120):
    """Random sites in a sheared box (some far outside it), each with an axis rule and distinct
    z / x / y atoms; indices a rule does not use are -1."""
    rng = np.random.default_rng(seed)
    box = np.array([[14.0, 0, 0], [2.0, 13.0, 0], [-1.5, 1.0, 15.0]])
    pos = rng.uniform(0, 1, (n, 3)) @ box + rng.integers(-2, 3, (n, 3)) @ box
    types = np.arange(n) % 6
    ind = np.full((n, 3), -1)
    for i in range(n):
        others = rng.choice(np.delete(np.arange(n), i), 3, replace=False)
        t = types[i]
        if t != 5:
            ind[i, 0] = others[0]
        if t in (0, 1, 2, 3):
            ind[i, 1] = others[1]
        if t in (2, 3):
            ind[i, 2] = others[2]
    return pos, box, types, ind


def test_local_frames_all_axis_rules_match_oracle():
    for seed in range(3):
        pos, box, types, ind = _sites(seed)
        got = generate_construct_local_frames(types, ind)(torch.tensor(pos), torch.tensor(box))
        want = R.construct_local_frames(pos, box, types, ind)
        assert (got - want).abs().max() < 1e-13
        eye = torch.eye(3, dtype=torch.float64)
        assert (got @ got.transpose(1, 2) - eye).abs().max() < 1e-13  # orthonormal rows
        assert (torch.linalg.det(got) - 1).abs().max() < 1e-13  # right-handed


def test_pbc_shift_and_pair_frames_match_oracle():
    pos, box, _, _ = _sites(5)
    b = torch.tensor(box)
    d = torch.tensor(pos[1:] - pos[:-1])
    assert (pbc_shift(d, b, torch.linalg.inv(b)) - R.pbc_shift(d, b, torch.linalg.inv(b))).abs().max() < 1e-12
    r1, r2 = torch.tensor(pos[:-1]), torch.tensor(pos[1:])
    r2[:5, 1:] = r1[:5, 1:]  # pairs along x: the frame seeds x from e_y
    dr = r1 - r2
    nd = torch.linalg.norm(dr, dim=1)
    assert (build_quasi_internal(r1, r2, dr, nd) - R.build_quasi_internal(r1, r2, dr, nd)).abs().max() < 1e-14


def test_global_multipoles_match_oracle():
    pos, box, types, ind = _sites(9, n=60)
    n_types = 7
    mt = np.random.default_rng(1).integers(0, n_types, len(pos))
    Q_local = torch.tensor(np.random.default_rng(2).standard_normal((n_types, 9)))
    for lmax in (0, 1, 2):
        f = ADMPPmeForce(box, mt, types, ind, 6.0, 5e-4, lmax)
        got = f.Q_local_to_global(torch.tensor(pos), torch.tensor(box), Q_local)
        Qm = Q_local[torch.as_tensor(mt)][:, : (lmax + 1) ** 2]
        if lmax > 0:
            Qm = R.rot_local2global(Qm, R.construct_local_frames(pos, box, types, ind), lmax)
        want = R.convert_harm2cart(Qm, lmax)
        assert got.shape == (len(pos), [1, 4, 10][lmax])
        assert (got - want).abs().max() < 1e-10
    assert f.construct_local_frames is not None
