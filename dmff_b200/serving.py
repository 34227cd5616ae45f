"""Continuous-batching serving of independent ADMP evaluations (energy + forces + virial).

``AdmpServer`` wraps the native server of libdmffb200.so (``dmffb_server_*``): a pool of engine
slots with one host worker thread each, created at the largest request size and re-pointed at
every request.  Requests queue in arrival order and are admitted when their arrival time has
passed, a slot is idle and the summed device footprint of the requests in flight stays within
the HBM budget; admitted requests run concurrently on their slots' CUDA streams.  Inputs and
outputs are host arrays; positions, grids, pair lists and induced dipoles stay on the device
for the whole evaluation.

``run_stream`` submits a list of systems with arrival times and returns per-request latency
(completion - arrival) and the aggregate throughput in atom-evals/s (atoms of all completed
evaluations / time from the first arrival to the last completion).
"""
import ctypes

import numpy as np
import torch

from . import _lib as L

_PREC = {"fp32": L.DMFFB_FP32, "fp64": L.DMFFB_FP64}
_SOLVERS = {"cg": L.DMFFB_SOLVER_CG, "reference": L.DMFFB_SOLVER_REFERENCE}


def _c(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


class ServingRequest:
    """One evaluation: holds the host arrays alive and exposes the results once ``done``."""

    def __init__(self, sysd, t_arrival=0.0):
        n = int(sysd["n_atoms"])
        self.n_atoms = n
        self._arrays = dict(
            pos=_c(sysd["pos"], np.float64).reshape(n, 3), axis_types=_c(sysd["axis_types"], np.int32),
            axis_indices=_c(sysd["axis_indices"], np.int32).reshape(n, 3),
            cov_rows=_c(sysd["cov_rows"], np.int32).reshape(-1, 3), Q_local=np.zeros((n, 9)),
            pol=_c(sysd["pol"], np.float64) if sysd.get("pol") is not None else None,
            thole=_c(sysd["thole"], np.float64) if sysd.get("thole") is not None else None,
            forces=np.zeros((n, 3)))
        Q = np.asarray(sysd["Q_local"], dtype=np.float64)
        self._arrays["Q_local"][:, : Q.shape[1]] = Q
        a = self._arrays
        r = L.Request()
        r.n_atoms = n
        r.pos = a["pos"].ctypes.data
        for k, v in enumerate(np.asarray(sysd["box"], dtype=np.float64).reshape(9)):
            r.box[k] = v
        r.axis_types = a["axis_types"].ctypes.data
        r.axis_indices = a["axis_indices"].ctypes.data
        r.n_cov = a["cov_rows"].shape[0]
        r.cov_rows = a["cov_rows"].ctypes.data
        r.Q_local = a["Q_local"].ctypes.data
        r.pol = a["pol"].ctypes.data if a["pol"] is not None else None
        r.thole = a["thole"].ctypes.data if a["thole"] is not None else None
        r.rc = float(sysd["rc"])
        r.kappa = float(sysd["kappa"])
        for k in range(3):
            r.K[k] = int(sysd["K"][k])
        r.t_arrival = float(t_arrival)
        r.forces_out = a["forces"].ctypes.data
        self.c = r

    @property
    def done(self):
        return bool(self.c.done)

    @property
    def energy(self):
        return self.c.energy

    @property
    def forces(self):
        return self._arrays["forces"]

    @property
    def box_grad(self):
        return np.array(self.c.box_grad).reshape(3, 3)

    @property
    def latency(self):
        return self.c.t_done - self.c.t_arrival

    @property
    def status(self):
        return self.c.status


class AdmpServer:
    def __init__(self, n_slots=8, capacity_atoms=30000, lmax=2, lpol=True, precision="fp32", hbm_budget_bytes=0,
                 mscales=(0, 0, 1, 1, 1, 1), pscales=(0, 0, 1, 1, 1, 1), dscales=(1, 1, 1, 1, 1, 1), solver="cg",
                 cg_tol=1e-6, max_iter=200, use_graphs=True, device=None):
        self.lib = L.load()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        d = L.ServerDesc()
        d.n_slots = int(n_slots)
        d.capacity_atoms = int(capacity_atoms)
        d.hbm_budget_bytes = int(hbm_budget_bytes)
        d.lmax, d.lpol, d.precision = int(lmax), int(bool(lpol)), _PREC[precision]
        for k in range(6):
            d.mscales[k], d.pscales[k], d.dscales[k] = float(mscales[k]), float(pscales[k]), float(dscales[k])
        d.solver = _SOLVERS[solver]
        d.cg_tol = float(cg_tol)
        d.max_iter = int(max_iter)
        d.use_graphs = int(bool(use_graphs))
        self.capacity = int(capacity_atoms)
        self.n_slots = int(n_slots)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = self.lib.dmffb_server_create(ctypes.byref(d), ctypes.byref(h))
        if st != L.DMFFB_OK:
            raise L.EngineError(st, "dmffb_server_create failed")
        self.h = h
        self._live = []

    def clock(self):
        return self.lib.dmffb_server_clock(self.h)

    def submit(self, req):
        st = self.lib.dmffb_server_submit(self.h, ctypes.byref(req.c))
        if st != L.DMFFB_OK:
            raise L.EngineError(st, "dmffb_server_submit failed")
        self._live.append(req)

    def wait(self, timeout=600.0):
        st = self.lib.dmffb_server_wait(self.h, float(timeout))
        if st != L.DMFFB_OK:
            raise TimeoutError("serving requests did not complete in time")
        self._live = [r for r in self._live if not r.done]

    def prewarm(self, reqs):
        arr = (L.Request * len(reqs))(*[r.c for r in reqs])
        st = self.lib.dmffb_server_prewarm(self.h, arr, len(reqs))
        if st not in (L.DMFFB_OK, L.DMFFB_NOT_CONVERGED):
            raise L.EngineError(st, "dmffb_server_prewarm failed")

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.dmffb_server_destroy(self.h)
            self.h = None

    __del__ = close

    def run_stream(self, systems, arrivals, timeout=1800.0):
        """Submit ``systems`` (dicts as built by ``synthetic.serving_system``) with ``arrivals``
        (seconds from now, non-decreasing); returns (requests, stats)."""
        # the requests (host arrays, C structs) are built before the clock starts, so that the
        # arrival times are not already past when they are submitted
        reqs = [ServingRequest(s) for s in systems]
        t0 = self.clock() + 0.05  # a short head start so that submission runs ahead of arrivals
        for r, a in zip(reqs, arrivals):
            r.c.t_arrival = t0 + float(a)
            self.submit(r)
        self.wait(timeout)
        return reqs, stream_stats(reqs)


def stream_stats(reqs):
    lat = np.array([r.latency for r in reqs])
    atoms = sum(r.n_atoms for r in reqs)
    t_first = min(r.c.t_arrival for r in reqs)
    t_last = max(r.c.t_done for r in reqs)
    bad = [r.status for r in reqs if r.status not in (L.DMFFB_OK, L.DMFFB_NOT_CONVERGED)]
    codes = {}
    for c in bad:
        codes[str(int(c))] = codes.get(str(int(c)), 0) + 1
    return {"requests": len(reqs), "atoms": int(atoms), "wall_s": t_last - t_first,
            "atom_evals_per_s": atoms / (t_last - t_first), "p50_ms": float(np.percentile(lat, 50) * 1e3),
            "p99_ms": float(np.percentile(lat, 99) * 1e3), "max_ms": float(lat.max() * 1e3), "failed": len(bad),
            "failed_status": codes,
            "not_converged": sum(1 for r in reqs if r.status == L.DMFFB_NOT_CONVERGED)}


# ----------------------------------------------------------------------------------- replicas
def assign_requests(atoms, n_ranks):
    """Rank of every request for an ``n_ranks``-replica deployment: in arrival order, each request
    goes to the rank with the fewest atoms assigned so far (ties to the lower rank).  Deterministic,
    so every rank computes the same assignment from the same stream without communicating."""
    load = [0] * n_ranks
    out = []
    for a in atoms:
        r = min(range(n_ranks), key=lambda k: (load[k], k))
        out.append(r)
        load[r] += int(a)
    return out


def serve_replicated(systems, arrivals, run_local, group=None, timeout_s=600.0):
    """Serve one request stream on all ranks of a process group, one replica (server) per rank.

    ``run_local(systems, arrivals) -> list of per-request dicts`` runs this rank's share (its own
    GPU and server; no device data crosses ranks: the path has no exchange step).  Per-request
    records (``index``, ``n_atoms``, ``latency`` or ``error``) are gathered on every rank over
    ``group`` (a gloo group: objects, not device tensors).  Requests whose rank raised are
    re-assigned over the ranks that did not and run in a second round.  Returns (records sorted by
    request index, summary dict)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    owner = assign_requests([s["n_atoms"] for s in systems], world)
    mine = [k for k in range(len(systems)) if owner[k] == rank]

    def run(indices):
        try:
            recs = run_local([systems[k] for k in indices], [arrivals[k] for k in indices])
            for k, r in zip(indices, recs):
                r["index"] = k
            return {"rank": rank, "ok": True, "records": recs}
        except Exception as e:  # a failed replica reports instead of leaving the group
            return {"rank": rank, "ok": False, "error": f"{type(e).__name__}: {e}", "indices": list(indices)}

    def gather(obj):
        got = [None] * world
        dist.all_gather_object(got, obj, group=group)
        return got

    first = gather(run(mine))
    records = [r for g in first if g["ok"] for r in g["records"]]
    failed_ranks = [g["rank"] for g in first if not g["ok"]]
    retry = sorted(k for g in first if not g["ok"] for k in g["indices"])
    alive = [r for r in range(world) if r not in failed_ranks]
    redistributed = 0
    if retry and alive:
        sub = assign_requests([systems[k]["n_atoms"] for k in retry], len(alive))
        mine2 = [k for k, a in zip(retry, sub) if alive[a] == rank]
        second = gather(run(mine2) if rank in alive else {"rank": rank, "ok": True, "records": []})
        for g in second:
            if g["ok"]:
                records += g["records"]
        redistributed = len(retry)
    records.sort(key=lambda r: r["index"])
    done = {r["index"] for r in records}
    summary = {"ranks": world, "requests": len(systems), "completed": len(done),
               "failed_ranks": failed_ranks, "redistributed": redistributed,
               "errors": [g["error"] for g in first if not g["ok"]],
               "atoms": int(sum(r["n_atoms"] for r in records))}
    return records, summary


def server_run_local(**server_kw):
    """``run_local`` for ``serve_replicated``: this rank's share on an ``AdmpServer`` on its GPU
    (keyword arguments as ``AdmpServer``; capacity defaults to the share's largest request)."""
    def run_local(systems, arrivals):
        if not systems:
            return []
        kw = dict(server_kw)
        kw.setdefault("capacity_atoms", max(s["n_atoms"] for s in systems))
        srv = AdmpServer(**kw)
        try:
            reqs, _ = srv.run_stream(systems, arrivals)
        finally:
            srv.close()
        return [{"n_atoms": r.n_atoms, "latency": r.latency, "energy": r.energy, "status": r.status,
                 "box_grad": r.box_grad.tolist()} for r in reqs]
    return run_local
