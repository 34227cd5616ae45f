"""``dmff_b200.admp.pairwise`` (dmff/admp/pairwise.py): the generic pair-sum calculator with the
Tang–Toennies kernels, against the oracle's restatement on a water box; padding rows, the
nbond column and autograd through the per-atom parameters."""
import numpy as np
import torch

import oracle.admp_ref as R
from dmff_b200.admp.pairwise import (TT_damping_qq_c6_kernel, TT_damping_qq_kernel, distribute_matrix,
                                     distribute_scalar, generate_pairwise_interaction)
from dmff_b200.synthetic import pairs_nbond, water_box


def _setup():
    s = water_box(64, 12.4, seed=6, lmax=0, pol=False, rc=5.0)
    pairs = R.brute_force_pairs(s["pos"], s["box"], 5.0)
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    n = s["n_atoms"]
    pad = np.full((25, 3), n)
    pad[:, 2] = 0
    rng = np.random.default_rng(3)
    prm = [torch.tensor(rng.uniform(lo, hi, n), requires_grad=True)
           for lo, hi in ((50.0, 90.0), (3.5, 4.5), (-0.8, 0.4), (0.5, 1.5))]  # A, B, Q, C6
    ms = torch.tensor([0.0, 0.0, 0.5, 1.0, 1.0, 1.0], dtype=torch.float64)
    return s, np.concatenate([pairs, pad]), prm, ms


def test_tt_qq_c6_pair_sum_matches_oracle():
    s, pairs, prm, ms = _setup()
    pos, box = torch.tensor(s["pos"]), torch.tensor(s["box"])
    # a wrapped kernel takes the elementwise torch path (the built-in itself runs on the GPU engine)
    E = generate_pairwise_interaction(lambda *a: TT_damping_qq_c6_kernel(*a), {})(pos, box, pairs, ms, *prm)
    Eo = R.pairwise_energy(R.TT_damping_qq_c6_kernel, pos, box, pairs, ms, *prm)
    assert abs(E.item() - Eo.item()) <= 1e-12 * abs(Eo.item())
    g = torch.autograd.grad(E, prm)
    go = torch.autograd.grad(Eo, prm)
    for a, b in zip(g, go):
        assert (a - b).abs().max() <= 1e-10 * b.abs().max()


def test_tt_qq_kernel_and_distributors():
    s, pairs, prm, ms = _setup()
    pos, box = torch.tensor(s["pos"]), torch.tensor(s["box"])
    b, q = prm[1].detach(), prm[2].detach()
    E = generate_pairwise_interaction(lambda *a: TT_damping_qq_kernel(*a), {})(pos, box, pairs, ms, b, q)
    # the same sum written out: rows i < j, minimum image, m = mScales[nbond - 1]
    real = pairs[pairs[:, 0] < pairs[:, 1]]
    i, j = torch.as_tensor(real[:, 0]), torch.as_tensor(real[:, 1])
    d = R.pbc_shift(pos[i] - pos[j], box, torch.linalg.inv(box)).norm(dim=1)
    bb = torch.sqrt(b[i] * b[j])
    want = (-1389.35455846 * torch.exp(-bb * d) * (1 + bb * d) * q[i] * q[j] / d
            * ms[torch.as_tensor(real[:, 2]) - 1]).sum()
    assert abs(E.item() - want.item()) <= 1e-12 * abs(want.item())
    x = torch.arange(10.0)
    assert torch.equal(distribute_scalar(x, torch.tensor([3, 1])), torch.tensor([3.0, 1.0]))
    assert distribute_matrix(x.reshape(2, 5), 1, 2).item() == 7.0
