"""dmffb_build_neighbors_noalloc: the neighbour build for callers that cannot allocate device
memory (an MD platform or framework that owns the device heap).  Its scratch is a fixed array
inside the library; the test checks its rows against dmffb_build_neighbors on two calls in a
row and that the calls leave the device's free memory unchanged.  Kept in a file collected last.
"""
import ctypes

import numpy as np
import pytest
import torch

from dmff_b200 import _lib
from dmff_b200.synthetic import water_box

pytestmark = pytest.mark.gpu


def _cov_csr(sysd, dev):
    rows = sysd["cov_rows"]
    n = sysd["n_atoms"]
    order = np.lexsort((rows[:, 1], rows[:, 0]))
    rows = rows[order]
    ptr = np.zeros(n + 1, dtype=np.int32)
    np.add.at(ptr, rows[:, 0] + 1, 1)
    ptr = np.cumsum(ptr).astype(np.int32)
    to = lambda a: torch.tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)
    return to(ptr), to(rows[:, 1]), to(rows[:, 2])


def _noalloc(lib, pos, n, box, rc, cov, out):
    """Call the entry point through the C ABI; cov None passes three NULL pointers (no covalent
    map), out None a NULL pair buffer."""
    npairs = ctypes.c_int64(0)
    b = np.ascontiguousarray(box, dtype=np.float64).reshape(9)
    cp = [ctypes.c_void_p(None)] * 3 if cov is None else [ctypes.c_void_p(c.data_ptr()) for c in cov]
    st = lib.dmffb_build_neighbors_noalloc(
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.c_void_p(pos.data_ptr()), n,
        b.ctypes.data_as(ctypes.c_void_p), rc, cp[0], cp[1], cp[2],
        ctypes.c_void_p(None if out is None else out.data_ptr()), 0 if out is None else out.shape[0],
        ctypes.byref(npairs))
    return st, npairs.value


def _rows(a):
    return set(map(tuple, np.asarray(a, dtype=np.int64).tolist()))


def _check_against_oracle(lib, s, rc, with_cov=True):
    """One call on system s, compared as a set with the float64 brute-force pair oracle (nbond from
    the covalent rows, or 0 everywhere without a map)."""
    import oracle.admp_ref as R
    from dmff_b200.synthetic import pairs_nbond
    dev = torch.device("cuda", 0)
    want = R.brute_force_pairs(s["pos"], s["box"], rc)
    if with_cov:
        want[:, 2] = pairs_nbond(want, s["cov_rows"], s["n_atoms"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    out = torch.empty((len(want) + 16, 3), dtype=torch.int32, device=dev)
    st, npairs = _noalloc(lib, pos, s["n_atoms"], s["box"], rc, _cov_csr(s, dev) if with_cov else None, out)
    assert st == _lib.DMFFB_OK
    got = out[:npairs].cpu().numpy()
    assert npairs == len(want) > 0
    assert np.all(got[:, 0] < got[:, 1]) and np.all(np.diff(got[:, 0]) >= 0)
    assert _rows(got) == _rows(want)
    return want


def test_noalloc_neighbors_match_allocating_entry_on_two_calls():
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    s = water_box(1000, 31.0, seed=7, lmax=2, pol=False, rc=8.0)
    rng = np.random.default_rng(1)
    positions = [s["pos"], s["pos"] + rng.normal(0.0, 0.05, size=s["pos"].shape)]
    from tests.helpers import make_engine
    eng = make_engine(s, precision="fp64")  # reference entry point: dmffb_build_neighbors
    cov = _cov_csr(s, dev)
    out = torch.empty((400_000, 3), dtype=torch.int32, device=dev)
    pos0 = torch.tensor(positions[0], dtype=torch.float64, device=dev)
    st, _ = _noalloc(lib, pos0, s["n_atoms"], s["box"], 8.0, cov, out)  # first call: per-device set-up
    assert st == _lib.DMFFB_OK
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(dev)[0]
    for p in positions:  # two calls in a row, each checked against the allocating entry point
        pos = torch.tensor(p, dtype=torch.float64, device=dev)
        st, npairs = _noalloc(lib, pos, s["n_atoms"], s["box"], 8.0, cov, out)
        assert st == _lib.DMFFB_OK
        got = out[:npairs].cpu().numpy()
        want = eng.build_neighbors(pos, s["box"], 8.0).cpu().numpy()
        assert npairs == len(want) > 100_000
        assert np.all(got[:, 0] < got[:, 1]) and np.all(np.diff(got[:, 0]) >= 0)
        assert set(map(tuple, got.tolist())) == set(map(tuple, want.tolist()))
        del pos
    torch.cuda.synchronize()
    # the no-alloc calls themselves create no device allocation (the allocating entry point's
    # buffers were already sized by the first comparison; torch tensors above are freed to its cache)
    pos = torch.tensor(positions[1], dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    free_mid = torch.cuda.mem_get_info(dev)[0]
    st, _ = _noalloc(lib, pos, s["n_atoms"], s["box"], 8.0, cov, out)
    torch.cuda.synchronize()
    assert st == _lib.DMFFB_OK
    assert torch.cuda.mem_get_info(dev)[0] == free_mid
    assert free_before > 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    n = _lib.NOALLOC_MAX_ATOMS + 1
    pos = torch.zeros((1, 3), dtype=torch.float64, device=dev)  # never read: the size check comes first
    cov = [torch.zeros(1, dtype=torch.int32, device=dev)] * 3
    out = torch.empty((1, 3), dtype=torch.int32, device=dev)
    st, _ = _noalloc(lib, pos, n, np.eye(3) * 10.0, 4.0, cov, out)
    assert st == _lib.DMFFB_SCRATCH_TOO_SMALL


def test_noalloc_without_covalent_map():
    """NULL covalent map: every row's nbond is 0 (the zeroed empty-row region of the scratch)."""
    s = water_box(300, 21.0, seed=41, lmax=2, pol=False, rc=6.0)
    want = _check_against_oracle(_lib.load(), s, 6.0, with_cov=False)
    assert np.all(want[:, 2] == 0)


def test_noalloc_small_box_every_pair_path():
    """A box narrower than three cut-offs along an axis: no cell grid, the all-pairs kernel runs."""
    s = water_box(27, 9.3, seed=42, lmax=2, pol=False, rc=4.5)
    want = _check_against_oracle(_lib.load(), s, 4.5)
    assert np.any(want[:, 2] > 0)


def test_noalloc_triclinic_box():
    """A sheared (reduced) box, wide enough for three sheared cells per axis."""
    s = water_box(512, 24.8, seed=43, lmax=2, pol=False, rc=6.0)
    L = s["box"][0, 0]
    box = np.array([[L, 0.0, 0.0], [0.2 * L, L, 0.0], [-0.15 * L, 0.1 * L, L]])
    mol = s["pos"].reshape(-1, 3, 3)
    o = mol[:, 0, :]
    s = dict(s, pos=(mol - o[:, None, :] + ((o / L) @ box)[:, None, :]).reshape(-1, 3), box=box)
    _check_against_oracle(_lib.load(), s, 6.0)


def test_noalloc_coarsened_cell_grid():
    """A large sparse box with a short cut-off asks for 64^3 cells, more than the scratch holds:
    the grid is coarsened to at most DMFFB_NOALLOC_MAX_CELLS cells (each stays at least rc wide)."""
    rng = np.random.default_rng(44)
    n = 4000
    s = dict(n_atoms=n, pos=rng.uniform(0.0, 200.0, size=(n, 3)), box=np.eye(3) * 200.0,
             cov_rows=np.zeros((0, 3), dtype=np.int32))
    assert (200.0 // 3.0) ** 3 > 32768
    _check_against_oracle(_lib.load(), s, 3.0, with_cov=False)


def test_noalloc_reports_overflow_with_the_needed_count():
    """Capacity below the pair count (and a NULL pair buffer): DMFFB_NEIGHBOR_OVERFLOW with the
    exact count in *npairs_out, nothing written."""
    import oracle.admp_ref as R
    lib = _lib.load()
    dev = torch.device("cuda", 0)
    s = water_box(125, 15.5, seed=45, lmax=2, pol=False, rc=5.0)
    need = len(R.brute_force_pairs(s["pos"], s["box"], 5.0))
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    cov = _cov_csr(s, dev)
    out = torch.full((need // 2, 3), -7, dtype=torch.int32, device=dev)
    st, npairs = _noalloc(lib, pos, s["n_atoms"], s["box"], 5.0, cov, out)
    assert st == _lib.DMFFB_NEIGHBOR_OVERFLOW and npairs == need
    assert bool((out == -7).all())
    st, npairs = _noalloc(lib, pos, s["n_atoms"], s["box"], 5.0, cov, None)
    assert st == _lib.DMFFB_NEIGHBOR_OVERFLOW and npairs == need
