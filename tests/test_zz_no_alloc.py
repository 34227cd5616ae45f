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
    npairs = ctypes.c_int64(0)
    b = np.ascontiguousarray(box, dtype=np.float64).reshape(9)
    st = lib.dmffb_build_neighbors_noalloc(
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream), ctypes.c_void_p(pos.data_ptr()), n,
        b.ctypes.data_as(ctypes.c_void_p), rc, ctypes.c_void_p(cov[0].data_ptr()), ctypes.c_void_p(cov[1].data_ptr()),
        ctypes.c_void_p(cov[2].data_ptr()), ctypes.c_void_p(out.data_ptr()), out.shape[0], ctypes.byref(npairs))
    return st, npairs.value


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
