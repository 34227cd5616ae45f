"""GPU neighbour list with the reference's NeighborList interface (dmff/common/nblist.py:12-73).

``NeighborList(box, rcut, cov_map)``; ``allocate(coords)`` returns (i, j, nbond) rows for all
i < j with minimum-image distance < rcut, padded with (N, N, 0) rows up to a capacity fixed at
1.3x the first count (nblist.py:37-50); ``update`` rebuilds.  The build is the engine's cell-list
kernel; rows are a CUDA int32 tensor sorted by i.
"""
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
        pos = torch.as_tensor(np.asarray(coords.detach().cpu() if torch.is_tensor(coords) else coords),
                              dtype=torch.float64)
        self._positions = coords
        n = pos.shape[0]
        eng = self._eng(n)
        b = self.box if box is None else np.asarray(box, dtype=np.float64)
        rows = eng.build_neighbors(pos.to(eng.device).contiguous(), b, self.rcut)
        count = rows.shape[0]
        if self.capacity_multiplier is None:
            self.capacity_multiplier = int(count * 1.3)
        if not self.padding:
            self._pairs = rows
            return self._pairs
        self.capacity_multiplier = max(self.capacity_multiplier, count)
        pad = self.capacity_multiplier - count
        if pad > 0:
            padding = torch.full((pad, 3), n, dtype=torch.int32, device=rows.device)
            padding[:, 2] = 0
            rows = torch.cat([rows, padding], dim=0)
        self._pairs = rows
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


def _dense_rows(cov):
    m = np.asarray(cov)
    i, j = np.nonzero(np.triu(m, 1))
    return np.stack([i, j, m[i, j]], axis=1).astype(np.int32)


NeighborListFreud = NeighborList
