"""Host side of the serving loop: a request's arrays and the C request record that points at them,
and the stream statistics (throughput, p50 / p99 latency, failures) computed from finished
records.  No GPU: the records are filled by hand."""
import ctypes

import numpy as np

from dmff_b200 import _lib as L
from dmff_b200.serving import ServingRequest, stream_stats
from dmff_b200.synthetic import water_box


def _sys(n_mol, lmax=2, seed=0):
    return water_box(n_mol, 3.1 * n_mol ** (1 / 3) + 2.0, seed=seed, lmax=lmax, pol=True, rc=5.0)


def test_request_record_points_at_its_arrays():
    s = _sys(27, lmax=1)
    s = dict(s, Q_local=np.asarray(s["Q_local"])[:, :4])  # lmax 1: four harmonic components
    r = ServingRequest(s, t_arrival=1.25)
    c, n = r.c, s["n_atoms"]
    assert c.n_atoms == n and c.t_arrival == 1.25 and c.rc == 5.0
    pos = np.ctypeslib.as_array(ctypes.cast(c.pos, ctypes.POINTER(ctypes.c_double)), shape=(n, 3))
    assert np.array_equal(pos, s["pos"])
    assert list(c.box) == list(np.asarray(s["box"], dtype=np.float64).reshape(9))
    # lmax 1 multipoles are zero-padded to the 9 harmonic components the engine reads
    Q = np.ctypeslib.as_array(ctypes.cast(c.Q_local, ctypes.POINTER(ctypes.c_double)), shape=(n, 9))
    assert np.array_equal(Q[:, :4], s["Q_local"]) and not Q[:, 4:].any()
    assert c.n_cov == len(s["cov_rows"]) and [c.K[k] for k in range(3)] == list(s["K"])
    fo = np.ctypeslib.as_array(ctypes.cast(c.forces_out, ctypes.POINTER(ctypes.c_double)), shape=(n, 3))
    fo[0, 0] = 7.0  # the engine writes forces here; the request exposes the same memory
    assert r.forces[0, 0] == 7.0


def test_stream_stats_from_finished_records():
    reqs = [ServingRequest(_sys(8, seed=k), t_arrival=0.1 * k) for k in range(10)]
    for k, r in enumerate(reqs):
        r.c.t_done = r.c.t_arrival + 0.002 * (k + 1)
        r.c.status = L.DMFFB_OK
    reqs[3].c.status = L.DMFFB_NOT_CONVERGED
    reqs[4].c.status = L.DMFFB_BAD_ARG
    st = stream_stats(reqs)
    lat = np.array([0.002 * (k + 1) for k in range(10)])
    wall = (0.9 + 0.02) - 0.0
    assert st["requests"] == 10 and st["atoms"] == sum(r.n_atoms for r in reqs)
    assert abs(st["wall_s"] - wall) < 1e-12
    assert abs(st["atom_evals_per_s"] - st["atoms"] / wall) < 1e-6
    assert abs(st["p50_ms"] - np.percentile(lat, 50) * 1e3) < 1e-9
    assert abs(st["p99_ms"] - np.percentile(lat, 99) * 1e3) < 1e-9
    assert st["failed"] == 1 and st["not_converged"] == 1
