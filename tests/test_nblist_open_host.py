"""Host side of the non-periodic neighbour lists (dmff/common/nblist.py:76-157): the image-free box
(checked by replaying the build kernel's FP64 distance arithmetic in numpy against the plain
distance), the nbond lookup, padding, and the every-pair list made on the CPU device."""
import numpy as np
import torch

from dmff_b200.api.topology import CovalentMap, covalent_rows
from dmff_b200.common.nblist import NoCutoffNeighborList, NoPeriodicNeighborList, _nbond_lookup, _padded


def _kernel_within(pi, pj, L, rc):
    """The build kernel's exact test, op by op in float64 (every product and sum rounded
    separately, x then y then z) for the diagonal box L * I: s = d * (1/L) (+0 +0),
    s -= floor(s + 0.5), e = s * L (+0 +0), sqrt((e0^2 + e1^2) + e2^2) < rc."""
    d = pj - pi
    hinv = 1.0 / L
    s = (d * hinv + 0.0) + 0.0
    s = s - np.floor(s + 0.5)
    e = (s * L + 0.0) + 0.0
    r2 = (e[:, 0] * e[:, 0] + e[:, 1] * e[:, 1]) + e[:, 2] * e[:, 2]
    return np.sqrt(r2) < rc


def _plain_within(pi, pj, rc):
    """nblist.py:143-144: np.linalg.norm(coords[i] - coords[j]) < rcut."""
    return np.linalg.norm(pi - pj, axis=1) < rc


def test_open_box_reproduces_plain_distance_test_bit_for_bit():
    rng = np.random.default_rng(11)
    rc = 0.8
    for scale, shift in ((3.0, 0.0), (40.0, -17.3), (0.5, 123.456)):
        pos = rng.uniform(-scale, scale, (400, 3)) + shift
        # pairs placed on, and one ulp either side of, the cutoff
        u = rng.standard_normal((60, 3))
        u /= np.linalg.norm(u, axis=1, keepdims=True)
        for k, r in enumerate((rc, np.nextafter(rc, 0), np.nextafter(rc, 2))):
            pos[k * 20:(k + 1) * 20] = pos[200 + k * 20:200 + (k + 1) * 20] + r * u[k * 20:(k + 1) * 20]
        box = NoPeriodicNeighborList.open_box(torch.tensor(pos), rc)
        L = box[0, 0]
        assert L == 2.0 ** np.round(np.log2(L)) and L >= 2 * (np.ptp(pos, axis=0).max() + rc)
        i, j = np.triu_indices(len(pos), 1)
        got = _kernel_within(pos[i], pos[j], L, rc)
        want = _plain_within(pos[i], pos[j], rc)
        assert np.array_equal(got, want)
        assert want.sum() > 0


def test_nbond_lookup_dense_and_sparse():
    rows = np.array([[0, 1, 1], [1, 2, 1], [0, 2, 2], [2, 3, 1], [1, 3, 2], [0, 3, 3]])
    cov = CovalentMap(5, rows)
    dense = np.zeros((5, 5), dtype=np.int64)
    for a, b, d in rows:
        dense[a, b] = dense[b, a] = d
    i, j = torch.triu_indices(5, 5, 1)
    want = dense[i.numpy(), j.numpy()]
    assert np.array_equal(_nbond_lookup(cov, 5, i, j).numpy(), want)
    assert np.array_equal(_nbond_lookup(dense, 5, i, j).numpy(), want)
    assert np.array_equal(_nbond_lookup(torch.tensor(dense), 5, i, j).numpy(), want)


def test_no_cutoff_list_rows_and_padding():
    n = 7
    dense = np.zeros((n, n), dtype=np.int64)
    dense[0, 1] = dense[1, 0] = 1
    dense[5, 6] = dense[6, 5] = 2
    nl = NoCutoffNeighborList(dense, device="cpu")
    pairs = nl.allocate(np.zeros((n, 3))).numpy()
    m = n * (n - 1) // 2
    want = [(a, b, dense[a, b]) for a in range(n) for b in range(a + 1, n)]  # permutations order, i < j
    assert pairs.shape == (int(m * 1.3), 3)
    assert [tuple(r) for r in pairs[:m]] == want
    assert (pairs[m:, :2] == n).all() and (pairs[m:, 2] == 0).all()
    nl.update(np.zeros((n, 3)))
    assert nl.pairs.shape[0] == int(m * 1.3) and nl.scaled_pairs is nl.pairs
    assert NoCutoffNeighborList(dense, padding=False, device="cpu").allocate(np.zeros((n, 3))).shape == (m, 3)


def test_padding_capacity_grows_and_stays():
    class NL:
        capacity_multiplier = None
        padding = True
    nl = NL()
    r = torch.zeros((10, 3), dtype=torch.int32)
    assert _padded(nl, r, 4).shape[0] == 13
    assert _padded(nl, torch.zeros((20, 3), dtype=torch.int32), 4).shape[0] == 20
    assert _padded(nl, r, 4).shape[0] == 20


def test_sparse_nbond_lookup_matches_dense_on_a_random_graph():
    rng = np.random.default_rng(17)
    n = 300
    bonds = [(k, int(rng.integers(0, k))) for k in range(1, n)]  # a random tree
    cov = CovalentMap(n, covalent_rows(n, bonds, 3))  # each pair once, distances 1..3
    dense = np.zeros((n, n), dtype=np.int64)
    for a, b, d in cov.pairs():
        dense[a, b] = dense[b, a] = d
    i, j = torch.triu_indices(n, n, 1)
    assert np.array_equal(_nbond_lookup(cov, n, i, j).numpy(), dense[i.numpy(), j.numpy()])
