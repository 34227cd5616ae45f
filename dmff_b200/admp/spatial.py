"""Geometry helpers with the names of dmff/admp/spatial.py: minimum-image shifts, local frames and
the quasi-internal pair frame, as host utilities in torch on the input's device.

The engine builds the same local frames per step on the GPU (``k_prepare``); these functions
serve callers that want the frames or the global multipoles on the host, e.g. to fit or
inspect parameters.  Frames are [n, 3, 3] with rows (x, y, z) (spatial.py:44-156).  The axis
rules, by ``axis_types`` code:

  0 ZThenX     z toward the z atom, x toward the x atom, orthogonalised;
  1 Bisector   z along the bisector of the z and x directions;
  2 ZBisect    x along the bisector of the x and y directions;
  3 ThreeFold  z along the sum of the z, x and y directions;
  4 ZOnly      z toward the z atom, x seeded from the lab x or y axis, whichever is farther from z;
  5 NoAxisType the lab frame.
"""
import numpy as np
import torch

ZThenX, Bisector, ZBisect, ThreeFold, Zonly, NoAxisType = range(6)


def _f64(x, like=None):
    if torch.is_tensor(x):
        return x.to(torch.float64)
    dev = like.device if torch.is_tensor(like) else None
    return torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev)


def pbc_shift(drvecs, box, box_inv):
    """Minimum-image vectors (spatial.py:14-32): ds = dr box^-1, ds -= floor(ds + 1/2), ds box."""
    ds = _f64(drvecs) @ _f64(box_inv, drvecs)
    return (ds - torch.floor(ds + 0.5)) @ _f64(box, drvecs)


v_pbc_shift = pbc_shift


def normalize(matrix, axis=1, ord=2):
    """Unit vectors along ``axis`` (spatial.py:37-41)."""
    m = _f64(matrix)
    return m / torch.linalg.norm(m, ord=ord, dim=axis, keepdim=True)


def generate_construct_local_frames(axis_types, axis_indices):
    """``construct_local_frames(positions, box) -> [n, 3, 3]`` for fixed axis rules
    (spatial.py:44-156).  ``axis_indices`` [n, 3] holds the z, x, y atoms; entries a rule does
    not use may be -1."""
    types = np.asarray(axis_types, dtype=np.int64)
    ind = np.asarray(axis_indices, dtype=np.int64).reshape(-1, 3)

    def construct_local_frames(positions, box):
        pos = _f64(positions)
        box_ = _f64(box, pos)
        inv = torch.linalg.inv(box_)
        n = pos.shape[0]
        dev = pos.device
        rule = lambda *codes: torch.as_tensor(np.isin(types, codes), device=dev)[:, None]
        lab = torch.eye(3, dtype=torch.float64, device=dev)

        def toward(col, used):
            # unit minimum-image vector to the atom in column ``col``; rows that do not use it
            # point along the lab x axis so that nothing divides by zero
            j = torch.as_tensor(np.where(np.isin(types, used) & (ind[:, col] >= 0), ind[:, col], 0), device=dev)
            d = pbc_shift(pos[j] - pos, box_, inv)
            return normalize(torch.where(rule(*used), d, lab[0].expand(n, 3)))

        z = toward(0, (ZThenX, Bisector, ZBisect, ThreeFold, Zonly))
        # ZOnly: lab x, or lab y when z is closer to x than to the y-z plane (round(|z_x|) = 1)
        near_x = torch.round(torch.abs(z[:, 0]))[:, None]
        x_zonly = (1.0 - near_x) * lab[0] + near_x * lab[1]
        x = torch.where(rule(Zonly), x_zonly, toward(1, (ZThenX, Bisector, ZBisect, ThreeFold)))
        if (types == Bisector).any():
            z = torch.where(rule(Bisector), normalize(z + x), z)
        if np.isin(types, (ZBisect, ThreeFold)).any():
            y = toward(2, (ZBisect, ThreeFold))
            x = torch.where(rule(ZBisect), normalize(x + y), x)
            z = torch.where(rule(ThreeFold), normalize(z + x + y), z)
        x = normalize(x - z * torch.sum(x * z, dim=1, keepdim=True))
        y = torch.linalg.cross(z, x, dim=1)
        frames = torch.stack((x, y, z), dim=1)
        return torch.where(rule(NoAxisType)[:, :, None], lab.expand(n, 3, 3), frames)

    return construct_local_frames


def build_quasi_internal(r1, r2, dr, norm_dr):
    """Pair frames (spatial.py:160-187): z = dr / |dr|; x from z + e_x (z + e_y when r1 and r2
    share their y and z), orthogonalised; y = z x x."""
    r1, r2, dr = _f64(r1), _f64(r2), _f64(dr)
    z = dr / _f64(norm_dr, dr).reshape(-1, 1)
    lab = torch.eye(3, dtype=torch.float64, device=dr.device)
    off_axis = ((r1[:, 1] != r2[:, 1]) | (r1[:, 2] != r2[:, 2]))[:, None]
    x = z + torch.where(off_axis, lab[0], lab[1])
    x = normalize(x - z * torch.sum(z * x, dim=1, keepdim=True))
    return torch.stack([x, torch.linalg.cross(z, x, dim=1), z], dim=1)
