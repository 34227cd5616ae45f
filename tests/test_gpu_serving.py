"""Serving (continuous batching) on the GPU: every result is the same alone and in the mix, the
FP32 batched path matches the FP64 one-at-a-time path and the float64 oracle, and admission by
device footprint bounds what runs concurrently."""
import numpy as np
import pytest
import torch

from dmff_b200 import _lib as L
from dmff_b200.serving import AdmpServer, ServingRequest
from dmff_b200.synthetic import serving_system
from helpers import oracle_pairs, oracle_reference, rel_force_rms

pytestmark = pytest.mark.gpu

SIZES = [30, 45, 64, 90, 120, 150, 200, 260, 330, 400, 700]


@pytest.fixture(scope="module")
def systems():
    return [serving_system(n, k) for k, n in enumerate(SIZES)]


def _run(server, systems, arrivals=None):
    if arrivals is None:
        arrivals = np.zeros(len(systems))
    reqs, stats = server.run_stream(systems, arrivals)
    assert stats["failed"] == 0 and stats["not_converged"] == 0, [(r.n_atoms, r.status, r.c.n_iter) for r in reqs]
    return reqs, stats


@pytest.fixture(scope="module")
def alone(systems):
    srv = AdmpServer(n_slots=1, capacity_atoms=3 * max(SIZES), precision="fp32")
    out = _run(srv, systems)[0]
    srv.close()
    return out


def test_results_same_alone_and_in_the_mix(systems, alone):
    srv = AdmpServer(n_slots=6, capacity_atoms=3 * max(SIZES), precision="fp32")
    mix, stats = _run(srv, systems)
    srv.close()
    slots = {r.c.slot for r in mix}
    assert len(slots) > 1  # the mix really ran on several slots
    # requests overlapped in time on the device
    iv = sorted((r.c.t_start, r.c.t_done) for r in mix)
    assert any(iv[k + 1][0] < iv[k][1] for k in range(len(iv) - 1))
    # same within the stated FP32 tolerances (energy 1e-5 relative, forces 1e-4 relative RMS):
    # FP32 atomics make two runs sum in different orders and take different paths to the 1e-6
    # relative dipole residual, which moves energies at the 1e-6 and forces at the 1e-5 level
    for a, b in zip(alone, mix):
        assert abs(a.energy - b.energy) <= 1e-5 * abs(a.energy)
        assert rel_force_rms(b.forces, a.forces) < 1e-4
        assert np.abs(a.box_grad - b.box_grad).max() <= 1e-4 * np.abs(a.box_grad).max()


def test_fp32_batched_matches_fp64_plain_and_oracle(systems, alone):
    srv = AdmpServer(n_slots=1, capacity_atoms=3 * max(SIZES), precision="fp64", cg_tol=1e-8, use_graphs=False)
    plain = _run(srv, systems)[0]
    srv.close()
    for a, p in zip(alone, plain):
        assert abs(a.energy - p.energy) <= 1e-5 * abs(p.energy)
        assert rel_force_rms(a.forces, p.forces) < 1e-4
    # the smallest box (rc' < 8 A) against the float64 oracle
    s = systems[0]
    ref = oracle_reference(s, oracle_pairs(s), tol=1e-10)
    assert abs(plain[0].energy - ref["E"]) <= 1e-7 * abs(ref["E"])
    assert rel_force_rms(plain[0].forces, ref["F"]) < 1e-6
    assert abs(alone[0].energy - ref["E"]) <= 1e-5 * abs(ref["E"])
    assert rel_force_rms(alone[0].forces, ref["F"]) < 1e-4


def test_admission_by_footprint_serialises_when_budget_is_small(systems):
    fp = min(L.load().dmffb_request_footprint(s["n_atoms"], s["rc"], (ctypes_i3(s["K"])),
                                              float(np.linalg.det(s["box"])), 1) for s in systems)
    srv = AdmpServer(n_slots=4, capacity_atoms=3 * max(SIZES), precision="fp32", hbm_budget_bytes=fp)
    reqs, _ = _run(srv, systems)
    srv.close()
    iv = sorted((r.c.t_start, r.c.t_done) for r in reqs)
    assert all(iv[k + 1][0] >= iv[k][1] for k in range(len(iv) - 1))  # one in flight at a time


def ctypes_i3(K):
    import ctypes
    return (ctypes.c_int32 * 3)(*[int(k) for k in K])


def test_request_over_capacity_is_refused(systems):
    srv = AdmpServer(n_slots=1, capacity_atoms=100, precision="fp32")
    with pytest.raises(L.EngineError):
        srv.submit(ServingRequest(systems[-1]))
    srv.close()


def test_arrival_times_are_respected(systems):
    srv = AdmpServer(n_slots=4, capacity_atoms=3 * max(SIZES), precision="fp32")
    arr = np.arange(len(systems)) * 0.01
    reqs, stats = _run(srv, systems, arr)
    srv.close()
    for r in reqs:
        assert r.c.t_start >= r.c.t_arrival - 1e-6
    assert stats["p99_ms"] >= stats["p50_ms"] > 0


LARGE = [1000, 2500, 5000, 10000, 100, 150]


def test_large_requests_same_alone_and_in_the_mix_and_fp64():
    """The serving stream's upper end (up to 10000 waters / 30000 atoms, 66.9 A boxes) mixed with
    small boxes: each result is the same alone and in the mix within the FP32 tolerances, and the
    FP32 server matches the FP64 one-at-a-time path."""
    systems = [serving_system(n, 100 + k) for k, n in enumerate(LARGE)]
    cap = 3 * max(LARGE)
    srv = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp32")
    alone = _run(srv, systems)[0]
    srv.close()
    srv = AdmpServer(n_slots=4, capacity_atoms=cap, precision="fp32")
    mix = _run(srv, systems)[0]
    srv.close()
    assert len({r.c.slot for r in mix}) > 1
    srv = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp64", cg_tol=1e-8, use_graphs=False)
    plain = _run(srv, systems)[0]
    srv.close()
    for a, b, p in zip(alone, mix, plain):
        assert abs(a.energy - b.energy) <= 1e-5 * abs(a.energy)
        assert rel_force_rms(b.forces, a.forces) < 1e-4
        assert abs(a.energy - p.energy) <= 1e-5 * abs(p.energy)
        assert rel_force_rms(a.forces, p.forces) < 1e-4


def test_many_mesh_shapes_in_flight():
    """48 requests alternating small and large meshes (17^3 .. 49^3) on 12 slots: engines of
    different meshes launch the persistent solve and the FFT kernels side by side, every request
    succeeds and matches its result alone."""
    sizes = [100, 1500, 150, 1200, 200, 2300, 300, 900, 120, 3900, 450, 700] * 4
    syss = [serving_system(n, 300 + k) for k, n in enumerate(sizes)]
    cap = 3 * max(sizes)
    one = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp32")
    ref, _ = _run(one, syss)
    one.close()
    srv = AdmpServer(n_slots=12, capacity_atoms=cap, precision="fp32")
    reqs, stats = _run(srv, syss)
    srv.close()
    for a, b in zip(reqs, ref):
        assert abs(a.energy - b.energy) <= 2e-6 * abs(b.energy)
        assert rel_force_rms(a.forces, b.forces) < 2e-5
