"""Non-periodic neighbour lists on the GPU (dmff/common/nblist.py:76-157) against the plain
float64 distance test: the row set is bit-exact, nbond comes from the covalent map, and padding
follows the capacity rule."""
import numpy as np
import pytest
import torch

from dmff_b200.api.topology import CovalentMap
from dmff_b200.common.nblist import NoCutoffNeighborList, NoPeriodicNeighborList

pytestmark = pytest.mark.gpu


def _cluster(seed, n_mol=150, spread=14.0):
    """Rigid waters scattered in a sphere (Angstrom), with their intramolecular covalent rows."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((n_mol, 3))
    c *= spread * rng.uniform(0, 1, (n_mol, 1)) ** (1 / 3) / np.linalg.norm(c, axis=1, keepdims=True)
    h = np.array([[0.0, 0.0, 0.0], [0.9572, 0.0, 0.0], [-0.24, 0.9266, 0.0]])
    pos = (c[:, None, :] + h[None]).reshape(-1, 3) - 40.0  # far from the origin on purpose
    rows = []
    for m in range(n_mol):
        o = 3 * m
        rows += [(o, o + 1, 1), (o, o + 2, 1), (o + 1, o + 2, 2)]
    return pos, CovalentMap(len(pos), np.array(rows))


def _plain(pos, rc, cov):
    i, j = np.triu_indices(len(pos), 1)
    keep = np.linalg.norm(pos[i] - pos[j], axis=1) < rc
    i, j = i[keep], j[keep]
    return set(zip(i.tolist(), j.tolist(), cov.lookup(i, j).tolist()))


@pytest.mark.parametrize("rc", [4.0, 7.5])
def test_no_periodic_list_matches_plain_distance(rc):
    pos, cov = _cluster(21)
    nl = NoPeriodicNeighborList(rc, cov)
    pairs = nl.allocate(pos)
    assert pairs.is_cuda and pairs.dtype == torch.int32
    p = pairs.cpu().numpy()
    real = p[p[:, 0] < len(pos)]
    want = _plain(pos, rc, cov)
    assert len(real) == len(want)
    assert set(map(tuple, real.tolist())) == want
    assert p.shape[0] == int(len(want) * 1.3)
    # move the molecules: update rebuilds at the same capacity
    pos2 = pos + np.random.default_rng(2).normal(0, 0.3, pos.shape)
    nl.update(pos2)
    p2 = nl.pairs.cpu().numpy()
    assert set(map(tuple, p2[p2[:, 0] < len(pos)].tolist())) == _plain(pos2, rc, cov)


def test_no_cutoff_list_every_pair():
    pos, cov = _cluster(22, n_mol=40)
    n = len(pos)
    nl = NoCutoffNeighborList(cov, padding=False)
    p = nl.allocate(pos)
    assert p.is_cuda
    p = p.cpu().numpy()
    assert p.shape == (n * (n - 1) // 2, 3)
    i, j = np.triu_indices(n, 1)
    assert np.array_equal(p[:, 0], i) and np.array_equal(p[:, 1], j)
    assert np.array_equal(p[:, 2], cov.lookup(i, j))
