"""Multipole representations and frame rotations with the names of dmff/admp/multipole.py.

The harmonic layout per site is (Q00; Q10, Q11c, Q11s; Q20, Q21c, Q21s, Q22c, Q22s), the
Cartesian one (c; dx, dy, dz; qxx, qyy, qzz, qxy, qxz, qyz) (multipole.py:11-31, 36-112).  The
conversion tables are the reference's, with its truncated sqrt(3), because they define the
representation that parameter files and results are written in.

The rotations (multipole.py:117-236) act on frames ``localframes`` [n, 3, 3] whose rows are the
local axes in global coordinates.  The dipole block is R permuted to the (z, x, y) order.  The
quadrupole block is derived here rather than tabulated: the harmonic components are mapped to
the traceless Cartesian tensor, rotated as R T R^T and mapped back.  This equals the reference's
closed-form 5 x 5 matrix up to the rounding of its truncated sqrt(3).

These are host utilities for preparing parameters and reading results, in torch on the input's
device.  The energy kernels rotate multipoles themselves.  Inputs are [n, ...] batches, as
the reference's vmapped functions take them.
"""
import numpy as np
import torch

rt3 = 1.73205080757  # multipole.py:13
inv_rt3 = 1.0 / rt3

C1_h2c = torch.tensor([[0, 1, 0], [0, 0, 1], [1, 0, 0]], dtype=torch.float64)
C1_c2h = C1_h2c.T.contiguous()
C2_c2h = torch.tensor([[0, 0, 1, 0, 0, 0],
                       [0, 0, 0, 0, 2 * inv_rt3, 0],
                       [0, 0, 0, 0, 0, 2 * inv_rt3],
                       [inv_rt3, -inv_rt3, 0, 0, 0, 0],
                       [0, 0, 0, 2 * inv_rt3, 0, 0]], dtype=torch.float64)
C2_h2c = torch.tensor([[-0.5, 0, 0, rt3 / 2, 0],
                       [-0.5, 0, 0, -rt3 / 2, 0],
                       [1, 0, 0, 0, 0],
                       [0, 0, 0, 0, rt3 / 2],
                       [0, rt3 / 2, 0, 0, 0],
                       [0, 0, rt3 / 2, 0, 0]], dtype=torch.float64)

_ZXY = [2, 0, 1]


def _f64(x, like=None):
    if torch.is_tensor(x):
        return x.to(torch.float64)
    dev = like.device if torch.is_tensor(like) else None
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev)


def _check_lmax(lmax, exc=ValueError):
    if lmax > 2:
        raise exc("l > 2 (beyond quadrupole) not supported")


def convert_cart2harm(Theta, lmax):
    """Cartesian [n, 1 | 4 | 10] -> harmonic [n, (lmax+1)^2] (multipole.py:36-72)."""
    _check_lmax(lmax)
    T = _f64(Theta)
    out = [T[:, 0:1]]
    if lmax >= 1:
        out.append(T[:, 1:4] @ C1_c2h.to(T.device).T)
    if lmax >= 2:
        out.append(T[:, 4:10] @ C2_c2h.to(T.device).T)
    return torch.cat(out, dim=1)


def convert_harm2cart(Q, lmax):
    """Harmonic [n, (lmax+1)^2] -> Cartesian [n, 1 | 4 | 10] (multipole.py:77-112)."""
    _check_lmax(lmax)
    Q = _f64(Q)
    out = [Q[:, 0:1]]
    if lmax >= 1:
        out.append(Q[:, 1:4] @ C1_h2c.to(Q.device).T)
    if lmax >= 2:
        out.append(Q[:, 4:9] @ C2_h2c.to(Q.device).T)
    return torch.cat(out, dim=1)


def _sym(v6):
    """(xx, yy, zz, xy, xz, yz) -> symmetric 3 x 3."""
    xx, yy, zz, xy, xz, yz = v6.unbind(-1)
    return torch.stack([torch.stack([xx, xy, xz], -1), torch.stack([xy, yy, yz], -1),
                        torch.stack([xz, yz, zz], -1)], -2)


def _vec6(m):
    return torch.stack([m[..., 0, 0], m[..., 1, 1], m[..., 2, 2], m[..., 0, 1], m[..., 0, 2], m[..., 1, 2]], -1)


def rot_ind_global2local(U_g, localframes):
    """Dipoles only, harmonic (z, x, y) order: U_l = R_zxy U_g (multipole.py:117-124)."""
    U = _f64(U_g)
    R = _f64(localframes, U)
    return torch.einsum("nij,nj->ni", R[:, _ZXY][:, :, _ZXY], U)


def rot_global2local(Q_gh, localframes, lmax=2):
    """Harmonic moments from the global frame to each site's local frame (multipole.py:129-214)."""
    _check_lmax(lmax, NotImplementedError)
    Q = _f64(Q_gh)
    R = _f64(localframes, Q)
    out = [Q[:, 0:1]]
    if lmax >= 1:
        out.append(torch.einsum("nij,nj->ni", R[:, _ZXY][:, :, _ZXY], Q[:, 1:4]))
    if lmax >= 2:
        T = _sym(Q[:, 4:9] @ C2_h2c.to(Q.device).T)
        T_l = R @ T @ R.transpose(-2, -1)
        out.append(_vec6(T_l) @ C2_c2h.to(Q.device).T)
    return torch.cat(out, dim=1)


def rot_local2global(Q_lh, localframes, lmax=2):
    """Inverse of ``rot_global2local``: the same rotation with the transposed frames
    (multipole.py:218-236)."""
    return rot_global2local(Q_lh, _f64(localframes, Q_lh).transpose(-2, -1), lmax)
