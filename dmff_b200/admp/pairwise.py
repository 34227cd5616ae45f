"""Generic pairwise interactions with the names of dmff/admp/pairwise.py.

``generate_pairwise_interaction(kernel, static_args)`` returns
``pair_int(positions, box, pairs, mScales, *atomic_params)``: the sum over pair rows of
``kernel(r, m, p1_i, p1_j, p2_i, p2_j, ...) * [i < j]`` (pairwise.py:47-95).  ``r`` is the
minimum-image distance and ``m = mScales[nbond - 1]``, nbond read from the rows' last column.
``kernel`` is any elementwise torch function of those tensors.  It runs vectorised over all rows
on the rows' device, so user kernels run on the GPU when given CUDA tensors, and autograd
differentiates them.  The Tang–Toennies kernels of the reference (pairwise.py:100-128) are
provided as such functions.  ``ADMPDispForce``'s generator does not use this path: it evaluates
the same short-range term fused with the dispersion pair pass in CUDA.
"""
import torch

from ..utils import pair_buffer_scales, regularize_pairs
from .spatial import pbc_shift

DIELECTRIC = 1389.35455846


def distribute_scalar(params, index):
    """params[index] (pairwise.py:22-41)."""
    return params[index]


distribute_v3 = distribute_multipoles = distribute_dispcoeff = distribute_scalar


def distribute_matrix(multipoles, index1, index2):
    """multipoles[index1, index2] (pairwise.py:44-45)."""
    return multipoles[index1, index2]


def generate_pairwise_interaction(pair_int_kernel, static_args):
    """The pair-sum calculator for ``pair_int_kernel`` (pairwise.py:47-95); ``static_args`` is
    kept for the reference's signature."""

    def pair_int(positions, box, pairs, mScales, *atomic_params):
        pos = torch.as_tensor(positions, dtype=torch.float64)
        dev = pos.device
        rows = (pairs if torch.is_tensor(pairs) else torch.as_tensor(pairs)).to(dev).long()
        ij = regularize_pairs(rows[:, :2])
        buf = pair_buffer_scales(rows[:, :2]).to(torch.float64)
        m = torch.as_tensor(mScales, dtype=torch.float64).to(dev)[rows[:, -1] - 1] * buf
        b = torch.as_tensor(box, dtype=torch.float64).to(dev)
        dr = pbc_shift(pos[ij[:, 0]] - pos[ij[:, 1]], b, torch.linalg.inv(b))
        r = torch.linalg.norm(dr, dim=1)
        per_pair = []
        for p in atomic_params:
            p = torch.as_tensor(p).to(dev)
            per_pair += [p[ij[:, 0]], p[ij[:, 1]]]
        return torch.sum(pair_int_kernel(r, m, *per_pair) * buf)

    return pair_int


def TT_damping_qq_c6_kernel(dr, m, ai, aj, bi, bj, qi, qj, ci, cj):
    """Tang–Toennies short range with charge penetration and damped C6 (pairwise.py:100-117):
    2625.5 A e^{-br} - 2625.5 e^{-br} (1 + br) q / r + f_6(br) c / dr^6, with
    A = sqrt(a_i a_j), b = sqrt(b_i b_j), q = q_i q_j, c = c_i c_j, r = dr in bohr and
    f_6 the sixth-order damping sum; times m."""
    a = torch.sqrt(ai * aj)
    b = torch.sqrt(bi * bj)
    r = dr * 1.889726878
    br = b * r
    e = torch.exp(-br)
    f6 = 1 + br + br ** 2 / 2 + br ** 3 / 6 + br ** 4 / 24 + br ** 5 / 120 + br ** 6 / 720
    return (2625.5 * a * e - 2625.5 * e * (1 + br) * qi * qj / r + e * f6 * ci * cj / dr ** 6) * m


def TT_damping_qq_kernel(dr, m, bi, bj, qi, qj):
    """Charge-penetration term only (pairwise.py:121-128): -DIELECTRIC e^{-br} (1 + br) q / dr,
    b = sqrt(b_i b_j), r = dr; times m."""
    b = torch.sqrt(bi * bj)
    br = b * dr
    return -DIELECTRIC * torch.exp(-br) * (1 + br) * qi * qj / dr * m
