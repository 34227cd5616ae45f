"""GPU neighbour lists with the reference's interfaces (dmff/common/nblist.py).

``NeighborList(box, rcut, cov_map)`` (nblist.py:12-73); ``allocate(coords)`` returns (i, j, nbond)
rows for all i < j with minimum-image distance < rcut, padded with (N, N, 0) rows up to a capacity
fixed at 1.3x the first count (nblist.py:37-50); ``update`` rebuilds.  The build is the engine's
cell-list kernel; rows are a CUDA int32 tensor sorted by i.

``NoCutoffNeighborList(cov_map)`` (nblist.py:76-123): every i < j row.
``NoPeriodicNeighborList(rcut, cov_map)`` (nblist.py:126-157): i < j with plain (no image)
distance < rcut, built by the same cell-list kernel inside a cubic box whose edge is a power of two
at least twice the coordinate extent plus rcut.  In that box no pair takes an image shift, and the
kernel's FP64 test (d scaled by 1/L, then by L) returns d bit for bit.  So the rows are exactly
those of the plain-distance test |r_i - r_j| < rcut.
"""
import math

import numpy as np
import torch

from ..engine import AdmpEngine


class NeighborList:
    def __init__(self, box, rcut, cov_map, padding=True):
        self.box = np.asarray(box.detach().cpu() if torch.is_tensor(box) else box, dtype=np.float64)
        self.rcut = float(rcut)
        self.cov_map = cov_map
        self.padding = padding
        self.capacity_multiplier = None
        self._engine = None
        self._pairs = None
        self._positions = None

    def _eng(self, n):
        if self._engine is None or self._engine.n != n:
            rows = self.cov_map.pairs() if hasattr(self.cov_map, "pairs") else _dense_rows(self.cov_map)
            self._engine = AdmpEngine(n, 0, False, False, self.rcut, 0.0, (0, 0, 0), None, None, rows,
                                      [0, 0, 1, 1, 1, 1], precision="fp64")
        return self._engine

    def allocate(self, coords, box=None):
        pos = _host_f64(coords)
        self._positions = coords
        n = pos.shape[0]
        eng = self._eng(n)
        b = self.box if box is None else np.asarray(box, dtype=np.float64)
        rows = eng.build_neighbors(pos.to(eng.device).contiguous(), b, self.rcut)
        self._pairs = _padded(self, rows, n)
        return self._pairs

    def update(self, positions, box=None):
        self.allocate(positions, box)

    @property
    def pairs(self):
        return self._pairs

    @property
    def scaled_pairs(self):
        return self._pairs

    @property
    def positions(self):
        return self._positions


def _host_f64(coords):
    return torch.as_tensor(np.asarray(coords.detach().cpu() if torch.is_tensor(coords) else coords),
                           dtype=torch.float64)


def _padded(nl, rows, n):
    """Capacity and padding of nblist.py:37-50: the capacity is fixed at 1.3x the first count and
    grows to any larger count; short lists are filled with (N, N, 0) rows."""
    count = rows.shape[0]
    if nl.capacity_multiplier is None:
        nl.capacity_multiplier = int(count * 1.3)
    if not nl.padding:
        return rows
    nl.capacity_multiplier = max(nl.capacity_multiplier, count)
    pad = nl.capacity_multiplier - count
    if pad > 0:
        padding = torch.full((pad, 3), n, dtype=torch.int32, device=rows.device)
        padding[:, 2] = 0
        rows = torch.cat([rows, padding], dim=0)
    return rows


def _nbond_lookup(cov_map, n, i, j):
    """nbond of rows (i, j): the dense matrix entry (nblist.py:82-85), or the sparse rows of a
    ``CovalentMap``; 0 for pairs that are not bonded."""
    dev = i.device
    if hasattr(cov_map, "pairs"):
        # sparse rows: sorted keys i * n + j of both orientations, looked up by binary search
        r = np.asarray(cov_map.pairs(), dtype=np.int64).reshape(-1, 3)
        if r.shape[0] == 0:
            return torch.zeros(i.shape, dtype=torch.int32, device=dev)
        keys = np.concatenate([r[:, 0] * n + r[:, 1], r[:, 1] * n + r[:, 0]])
        vals = np.concatenate([r[:, 2], r[:, 2]])
        order = np.argsort(keys)
        keys = torch.as_tensor(keys[order], device=dev)
        vals = torch.as_tensor(vals[order], device=dev).to(torch.int32)
        q = i.to(torch.int64) * n + j.to(torch.int64)
        at = torch.searchsorted(keys, q).clamp(max=keys.shape[0] - 1)
        return torch.where(keys[at] == q, vals[at], torch.zeros((), dtype=torch.int32, device=dev))
    else:
        m = cov_map.detach().cpu() if torch.is_tensor(cov_map) else cov_map
        dense = torch.as_tensor(np.asarray(m), device=dev).to(torch.int32)
    return dense[i, j]


class NoCutoffNeighborList:
    """Every i < j row, in (i, j) order, with its nbond (nblist.py:76-123).  The rows are index
    arithmetic made on ``device`` (default: the current CUDA device)."""

    def __init__(self, cov_map, padding=True, device=None):
        self.capacity_multiplier = None
        self.padding = padding
        self.cov_map = cov_map
        self.device = device
        self._pairs = None
        self._positions = None

    def allocate(self, coords, box=None):
        self._positions = coords
        n = int(coords.shape[0])
        dev = torch.device(self.device) if self.device is not None else torch.device("cuda", torch.cuda.current_device())
        ij = torch.triu_indices(n, n, 1, device=dev)
        nbond = _nbond_lookup(self.cov_map, n, ij[0], ij[1])
        rows = torch.stack([ij[0].to(torch.int32), ij[1].to(torch.int32), nbond], dim=1).contiguous()
        self._pairs = _padded(self, rows, n)
        return self._pairs

    def update(self, positions, box=None):
        self.allocate(positions)

    @property
    def pairs(self):
        return self._pairs

    @property
    def scaled_pairs(self):
        return self._pairs

    @property
    def positions(self):
        return self._positions


class NoPeriodicNeighborList(NeighborList):
    """i < j rows with plain distance < rcut (nblist.py:126-157), from the engine's cell-list kernel
    inside an image-free power-of-two box."""

    def __init__(self, rcut, cov_map, padding=True):
        super().__init__(np.eye(3), rcut, cov_map, padding)

    @staticmethod
    def open_box(pos, rcut):
        """Cubic box, edge a power of two >= 2 (extent + rcut): no pair is within rcut of an image,
        and d / L, L * (d / L) are exact."""
        ext = float((pos.max(dim=0).values - pos.min(dim=0).values).max()) if pos.shape[0] else 0.0
        edge = 2.0 ** math.ceil(math.log2(2.0 * (ext + rcut)))
        return np.eye(3) * edge

    def allocate(self, coords, box=None):
        pos = _host_f64(coords)
        if not torch.isfinite(pos).all():
            raise ValueError("coordinates must be finite")
        return super().allocate(coords, self.open_box(pos, self.rcut))

    def update(self, positions, box=None):
        self.allocate(positions)


def _dense_rows(cov):
    m = np.asarray(cov)
    i, j = np.nonzero(np.triu(m, 1))
    return np.stack([i, j, m[i, j]], axis=1).astype(np.int32)


NeighborListFreud = NeighborList
