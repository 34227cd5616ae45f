"""Benchmark of the ADMP polarizable PME energy/force/virial step on B200.

Workload (default): 4096 rigid waters (12288 atoms) in a 49.7 A box, lmax=2 multipoles with
local frames, isotropic polarizabilities (O 1.0, H 0.5 A^3), Thole 0.33, rc = 8 A,
ethresh = 5e-4 (kappa 0.3285/A, 50^3 mesh); seeded synthetic coordinates and parameters.
One step = cell-list neighbour rebuild + induced-dipole CG solve (from U = 0) + energy,
forces and box gradient, FP32 pair / mesh arithmetic with FP64 accumulation.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0).  Multi-GPU runs (torchrun) evaluate one independent replica
per GPU (the path has no data exchange); value = all atom-evaluations / max-over-ranks time.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-evals/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c1")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--serving-requests", type=int, default=300,
                   help="requests of the serving stream measured beside the step (0: skip)")
    p.add_argument("--serving-rates", default="100,500,2000", help="Poisson arrival rates (req/s)")
    p.add_argument("--serving-slots", type=int, default=12)
    p.add_argument("--serving-budget-gb", type=float, default=2.0)
    return p.parse_args()


def workload_config(name, s, K):
    return {"workload": {"c1": "polarizable ADMP water box, 4096 waters / 12288 atoms, 49.7 A, rc 8 A",
                         "c0": "ADMP water box, 216 waters / 648 atoms, 18.6 A, rc 6 A, no polarization",
                         "c2": "polarizable ADMP water box, 2048 waters / 6144 atoms, 40 A, rc 8 A"}[name],
            "n_atoms": int(s["n_atoms"]), "lmax": int(s["lmax"]), "polarizable": bool(s["lpol"]),
            "rc_A": s["rc"], "ethresh": s["ethresh"], "pme_mesh": list(s["K"]),
            "cg_tol_rel": 1e-6, "l2": "flushed between timed steps (256 MiB write)",
            "step": "cell-list rebuild + CG dipole solve from U=0 + energy/forces/box gradient"}


# ---------------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) >= 9 for k in range(4) if r[5 + k].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


# ---------------------------------------------------------------------------------- roofline
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


# DRAM bytes per launch from one ncu capture of this workload (profiles/kernels_admp_pol_12288.md:
# dram__bytes_read.sum + dram__bytes_write.sum, 12288-atom polarizable step)
NCU_DRAM_BYTES = {"pair_matvec": 33.11e6, "spread": 2.77e6, "neighbors": 0.5 * (0.52e6 + 2.79e6)}


def roofline(stats, s, npairs, peaks, peak_src):
    """Roofline of the CG matvec (k_matvec_apply: the kernel with the largest share of the step in
    the ncu launch list, profiles/launches_admp_pol_12288.md), plus every kernel class's achieved
    rate against its bound.  Algorithmic work per launch (fixed convention): matvec 12 B per CSR
    entry (2 entries per pair: packed j + two FP32 coefficients); pair FULL polarizable 1900
    flop/pair, FIELD 600 flop/pair; spread N(12 + 4(l+1)^2) + 4K^3 B; gather 4K^3 + N(12 + 4(l+1)^2
    + 24) B; convolution 16 K^3 B; neighbour build 12N + 12 Np B."""
    n = s["n_atoms"]
    K3 = float(np.prod(s["K"]))
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12  # TFLOP/s, nominal at max clock
    models = {"pair_matvec": ("hbm", 12.0 * 2 * npairs), "pair_full": ("fp32", 1900.0 * npairs),
              "pair_field": ("fp32", 600.0 * npairs), "spread": ("hbm", n * (12 + 4 * 9) + 4 * K3),
              "gather_full": ("hbm", 4 * K3 + n * (12 + 4 * 9 + 24)), "gather_field": ("hbm", 4 * K3 + n * (12 + 16 + 24)),
              "conv": ("hbm", 16 * K3), "neighbors": ("hbm", 12 * n + 12 * npairs)}
    out = {}
    for cls, (bound, work) in models.items():
        ms, launches = stats.get(cls, (0.0, 0))
        if launches == 0:
            continue
        per = ms / 1e3 / launches
        if bound == "fp32":
            ach = work / per / 1e12
            out[cls] = {"bound": "fp32", "achieved": ach, "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak,
                        "avg_launch_us": per * 1e6, "launches": launches}
        else:
            ach = work / per / 1e9
            out[cls] = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": ach / peaks["hbm_gbs"], "avg_launch_us": per * 1e6, "launches": launches}
    main = dict(out["pair_matvec"], kernel="k_matvec_apply (CG matvec)", traffic=NCU_DRAM_BYTES["pair_matvec"],
                peak_source=f"hbm_gbs ({peak_src})",
                traffic_source="ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, this workload")
    main["by_class"] = {k: {"frac": round(v["frac"], 4), "achieved": round(v["achieved"], 2), "unit": v["unit"],
                            "avg_launch_us": round(v["avg_launch_us"], 2)} for k, v in out.items()}
    return main


# ---------------------------------------------------------------------------------- CPU side
def cpu_reference_timing(s, n_ref_iter, want_ef=True):
    """Float64 CPU restatement of the reference path (the oracle) on all host threads: one dE/dU
    pass (the unit of the dipole solve) and one energy+forces pass of the same workload."""
    import torch
    import oracle.admp_ref as R
    from dmff_b200.synthetic import pairs_nbond
    torch.set_num_threads(os.cpu_count())
    pr = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pr[:, 2] = pairs_nbond(pr, s["cov_rows"], s["n_atoms"])
    f = R.ADMPPmeForce(s["box"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], s["lmax"], s["lpol"],
                       kappa=s["kappa"], K=s["K"])
    Ql = torch.tensor(s["Q_local"])
    rest = (torch.tensor(s["pol"]), torch.tensor(s["thole"]), torch.tensor(s["mscales"]),
            torch.tensor(s["pscales"]), torch.tensor(s["dscales"]))
    pos = torch.tensor(s["pos"])
    box = torch.tensor(s["box"])
    U0 = torch.zeros((s["n_atoms"], 3), dtype=torch.float64)
    t0 = time.perf_counter()
    f.grad_U(pos, box, pr, Ql, U0, *rest)
    t_g = time.perf_counter() - t0
    t_ef = None
    if want_ef:
        p = pos.clone().requires_grad_(True)
        b = box.clone().requires_grad_(True)
        t0 = time.perf_counter()
        E = f.energy_fn(p, b, pr, Ql, U0, *rest)
        torch.autograd.grad(E, (p, b))
        t_ef = time.perf_counter() - t0
    return t_g, t_ef, torch.get_num_threads()


def run_reference(args, s, rank):
    """--impl reference: the reference's own CPU path (float64 oracle restatement; the JAX
    reference cannot be installed here) on the host cores, same workload/metric/unit."""
    if rank != 0:
        return
    n_ref_iter = 30  # the reference's MAX_N_POL (dmff/admp/settings.py:3)
    warm = min(args.warmup, 1)
    steps = min(args.steps, 3)
    t_ef = None
    for _ in range(max(warm, 1)):
        _, t_ef, cores = cpu_reference_timing(s, n_ref_iter, want_ef=True)
    tg = []
    for _ in range(steps):
        g, _, cores = cpu_reference_timing(s, n_ref_iter, want_ef=False)
        tg.append(g)
    t_eval = t_ef + n_ref_iter * statistics.median(tg)
    value = s["n_atoms"] / t_eval
    sample = (f"per step: one dE/dU pass of the {s['n_atoms']}-atom box (median of {steps}); one energy+forces "
              f"pass timed in warm-up ({t_ef:.2f} s); evaluation = E+F + {n_ref_iter} dE/dU passes "
              f"(the reference's MAX_N_POL)")
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": args.gpus,
           "steps": steps, "warmup": warm, "ms_per_step": t_eval * 1e3, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(args.workload, s, s["K"]),
           "cpu_baseline": {"value": value, "unit": "atom-evals/s", "cores": cores, "kind": "port", "sample": sample},
           "e2e": {"value": value, "unit": "atom-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------------- serving
def make_serving_systems(n_req, seed=3):
    """The serving stream's boxes (sizes log-uniform in [100, 10000] waters, seed 3), built in a
    spawn process pool (started before this process touches CUDA)."""
    import multiprocessing as mp
    from dmff_b200.synthetic import serving_sizes, serving_system
    sizes = serving_sizes(2000, seed=seed)[:n_req]
    with mp.get_context("spawn").Pool(max(1, min(os.cpu_count() or 1, 32))) as pool:
        return pool.starmap_async(serving_system, [(int(n), k) for k, n in enumerate(sizes)]).get(timeout=900)


def bench_serving(args, systems, dev):
    """Continuous-batching FP32 server vs the plain FP64 path (one request at a time, no graphs)
    on the same requests; latency = completion - arrival."""
    from dmff_b200.serving import AdmpServer, ServingRequest
    from dmff_b200.synthetic import serving_arrivals
    cap = max(s["n_atoms"] for s in systems)
    by_k = {}
    for s in systems:
        by_k.setdefault(tuple(s["K"]), s)
    warm = sorted(by_k.values(), key=lambda s: -s["n_atoms"])  # largest first: buffers grow once
    out = {"requests": len(systems), "atoms": int(sum(s["n_atoms"] for s in systems)),
           "sizes": "log-uniform 100-10000 waters (seed 3), 0.0334 molecules/A^3, rc 8 A (rc' = L/2 when L < 16 A)",
           "slots": args.serving_slots, "hbm_budget_GB": args.serving_budget_gb,
           "cg_tol_rel": 1e-6, "step": "polarizable ADMP energy + forces + virial, host buffers in and out"}
    srv = AdmpServer(n_slots=args.serving_slots, capacity_atoms=cap, precision="fp32",
                     hbm_budget_bytes=int(args.serving_budget_gb * (1 << 30)), device=dev)
    srv.prewarm([ServingRequest(s) for s in warm])

    def median_run(server, syss, repeats=3):
        # a stream lasts a fraction of a second: report the median of a few runs (and all rates)
        runs = [server.run_stream(syss, np.zeros(len(syss))) for _ in range(repeats)]
        runs.sort(key=lambda r: r[1]["atom_evals_per_s"])
        reqs_m, st_m = runs[len(runs) // 2]
        return reqs_m, dict(st_m, runs_atom_evals_per_s=[round(r[1]["atom_evals_per_s"]) for r in runs])

    reqs, st = median_run(srv, systems)
    out["offline_fp32"] = st
    fp32 = reqs
    for rate in [float(x) for x in args.serving_rates.split(",") if x]:
        _, st = srv.run_stream(systems, serving_arrivals(len(systems), rate, seed=33))
        out[f"poisson_{int(rate)}_per_s"] = st
    srv.close()
    # plain path: FP64, one slot, graphs off, every 5th request back to back
    sub = systems[::5]
    plain = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp64", use_graphs=False, cg_tol=1e-6, device=dev)
    # the same warm-up as the server: one request per mesh shape, so that neither timed run
    # includes cuFFT plan creation
    plain.prewarm([ServingRequest(s) for s in warm])
    preqs, pst = median_run(plain, sub)
    plain.close()
    out["plain_fp64"] = dict(pst, sample="every 5th request of the stream, one at a time")
    out["speedup_vs_plain"] = out["offline_fp32"]["atom_evals_per_s"] / pst["atom_evals_per_s"]
    # the same plain path with the reference's own dipole iteration (fixed-point steps, POL_CONV 1.0,
    # MAX_N_POL 30, pme.py:342-423) in place of CG: the reference's algorithm run on this GPU
    plain_r = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp64", use_graphs=False, solver="reference",
                         cg_tol=1.0, max_iter=30, device=dev)
    plain_r.prewarm([ServingRequest(s) for s in warm])
    _, rst = median_run(plain_r, sub)
    plain_r.close()
    out["plain_fp64_reference_solver"] = dict(rst, sample="every 5th request of the stream, one at a time",
                                              solver="fixed-point dipole iteration, POL_CONV 1.0, MAX_N_POL 30")
    out["speedup_vs_plain_reference_solver"] = out["offline_fp32"]["atom_evals_per_s"] / rst["atom_evals_per_s"]
    errs_e, errs_f = [], []
    for k, p in enumerate(preqs):
        q = fp32[5 * k]
        errs_e.append(abs(q.energy - p.energy) / abs(p.energy))
        errs_f.append(float(np.sqrt(np.mean((q.forces - p.forces) ** 2)) / np.sqrt(np.mean(p.forces ** 2))))
    out["fp32_vs_fp64"] = {"max_rel_energy": float(max(errs_e)), "max_rel_force_rms": float(max(errs_f))}
    return out


# ---------------------------------------------------------------------------------- classical
def run_classical(args, rank, world, local):
    """--workload c4: large classical system (200 chains x 50 beads + 30000 waters, 70 A box,
    ~100k atoms): LJ + Coulomb PME (rc 10 A, ethresh 1e-5, 154^3 mesh) + harmonic bonds / angles
    + 3-term torsions.  One step = cell-list rebuild + energy / forces / box gradient, FP32 pair
    and mesh arithmetic with FP64 accumulation.  --impl reference: the float64 oracle on a bounded
    sample of pair rows (extrapolated per pair) plus the bonded terms and reciprocal part."""
    import torch
    from dmff_b200.synthetic import polymer_water_box
    s = polymer_water_box(200, 50, 30000, 70.0, seed=4, rc=10.0, ethresh=1e-5)
    cfg = {"workload": "classical polymer + water, 200 x 50 beads + 30000 waters / 100000 atoms, 70 A, rc 10 A",
           "n_atoms": int(s["n_atoms"]), "pme_mesh": list(s["K"]), "ethresh": s["ethresh"],
           "terms": "LJ (LB) + Coulomb PME + harmonic bonds/angles + periodic torsions",
           "l2": "inputs larger than L2 (pair list ~0.7 GB)", "step": "cell-list rebuild + energy/forces/box gradient"}
    if args.impl == "reference":
        if rank != 0:
            return
        out = classical_cpu_reference(s, cfg, args)
        print(json.dumps(out), flush=True)
        return
    from dmff_b200.engine import ClassicalEngine
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    eng = ClassicalEngine(s["n_atoms"], n_types=len(s["sigma"]), coulomb="pme", pbc=True, rc=s["rc"], kappa=s["kappa"],
                          K=s["K"], cov_rows=s["cov_rows"], mscales_coul=s["mscales_coul"], mscales_lj=s["mscales_lj"],
                          precision="fp32", device=dev)
    eng.set_params(s["charges"], s["types"], s["sigma_tt"], s["eps_tt"])
    eng.set_terms("bond", s["bonds"], s["bond_prm"])
    eng.set_terms("angle", s["angles"], s["angle_prm"])
    eng.set_terms("torsion", s["torsions"], s["torsion_prm"])
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        eng.rebuild_internal_pairs(pos, s["box"])
        return eng.compute(pos, s["box"])

    for _ in range(args.warmup):
        res, F = step()
    torch.cuda.synchronize()
    l0 = eng.counters()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            evs[k][0].record(stream)
            res, F = step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total = sum(step_ms)
    l1 = eng.counters()
    if world > 1:
        t = torch.tensor([total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    value = world * args.steps * s["n_atoms"] / (total / 1e3)
    # e2e: pinned host positions in, forces and energy out, through the public engine API
    pos_h = torch.tensor(s["pos"], dtype=torch.float64).pin_memory()
    F_h = torch.empty((s["n_atoms"], 3), dtype=torch.float64).pin_memory()
    e2e = []
    for k in range(args.steps + args.warmup):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        pos.copy_(pos_h, non_blocking=True)
        r, Fd = step()
        F_h.copy_(Fd, non_blocking=True)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    e2e_value = world * args.steps * s["n_atoms"] / sum(e2e)
    eng.set_profiling(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    stats = eng.kernel_stats()
    eng.set_profiling(False)
    peaks, src = measured_peaks()
    ms, nl = stats["pair_full"]
    per = ms / 1e3 / max(nl, 1)
    fp32_peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) * 1e6 / 1e12
    # pair launches: one FP32 launch over all rows and one FP64 launch over the scaled rows, plus
    # the three bonded launches share the class; work per step = 120 flop per pair row
    flops_step = 120.0 * res.n_pairs
    ach = flops_step / (ms / 1e3 / args.steps) / 1e12
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "fp32 pairs/mesh, fp64 accumulation", "data": "synthetic",
               "config": dict(cfg, parallelism=f"replicas x{world}"),
               "e2e": {"value": e2e_value, "unit": "atom-evals/s", "h2d_bytes_per_step": 24 * s["n_atoms"],
                       "d2h_bytes_per_step": 24 * s["n_atoms"], "path": "ClassicalEngine.compute, pinned host copies"},
               "roofline": {"kernel": "k_nb_pair (LJ + erfc Coulomb) + bonded terms", "bound": "fp32", "achieved": ach,
                            "peak": fp32_peak, "unit": "TFLOP/s", "frac": ach / fp32_peak, "traffic": None,
                            "avg_launch_us": per * 1e6, "peak_source": "nominal FP32 CUDA-core peak at max SM clock"},
               "clocks": clk.summary(), "gpu_launches": int(l1["launches"] - l0["launches"]),
               "library_launches": {"cufft_execs": int(l1["fft_execs"] - l0["fft_execs"])},
               "result": {"energy_kJmol": res.energy, "e_coul": res.e_coul_real + res.e_coul_recip + res.e_coul_self,
                          "e_lj": res.e_lj, "e_bonded": res.e_bond + res.e_angle + res.e_torsion,
                          "n_pairs": int(res.n_pairs)},
               "kernel_ms_per_step": {k: v[0] / args.steps for k, v in stats.items() if v[1]}}
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def classical_cpu_reference(s, cfg, args):
    """Float64 oracle (dmff/classical/*.py restated) on the host cores: LJ + real-space Coulomb on
    a bounded sample of 2 M pair rows (scaled to the full pair count), the reciprocal part on the
    full 154^3 mesh once, and all bonded terms."""
    import torch
    import oracle.admp_ref as R
    from dmff_b200.synthetic import pairs_nbond
    torch.set_num_threads(os.cpu_count())
    pos = torch.tensor(s["pos"])
    box = torch.tensor(s["box"])
    # full pair count from the cell-list estimate over a sample of atoms
    rng = np.random.default_rng(0)
    n = s["n_atoms"]
    samp = rng.choice(n, 200, replace=False)
    d = s["pos"][None, :, :] - s["pos"][samp][:, None, :]
    d -= s["box"][0, 0] * np.round(d / s["box"][0, 0])
    npairs = int(round((np.sqrt((d * d).sum(-1)) < s["rc"]).sum(1).mean() - 1) * n / 2)
    m = 2_000_000
    i = rng.integers(0, n, size=m)
    j = (i + rng.integers(1, n, size=m)) % n
    lo, hi = np.minimum(i, j), np.maximum(i, j)
    pr = np.stack([lo, hi, np.zeros(m, dtype=np.int64)], 1)
    pr[:, 2] = pairs_nbond(pr, s["cov_rows"], n)
    t0 = time.perf_counter()
    q = torch.tensor(s["charges"])
    R.lj_energy(pos, box, pr, torch.tensor(s["epsilon"]), torch.tensor(s["sigma"]), s["types"], s["mscales_lj"])
    R.pme_real(pos, box, pr, q.reshape(-1, 1), None, None, None, s["mscales_coul"], None, None, s["kappa"], 0, False)
    t_pairs = (time.perf_counter() - t0) * npairs / m
    t0 = time.perf_counter()
    recip = R.generate_pme_recip(R.Ck_1, s["kappa"], False, 6, *s["K"], 0)
    recip(pos, box, q.reshape(-1, 1))
    t_recip = time.perf_counter() - t0
    b, a, t = (torch.as_tensor(s[k]).long() for k in ("bonds", "angles", "torsions"))
    t0 = time.perf_counter()
    bp, ap, tp = (torch.tensor(s[k]) for k in ("bond_prm", "angle_prm", "torsion_prm"))
    R.bond_energy(pos, b[:, 0], b[:, 1], bp[:, 0], bp[:, 1])
    R.angle_energy(pos, a[:, 0], a[:, 1], a[:, 2], ap[:, 0], ap[:, 1])
    R.torsion_energy(pos, t[:, 0], t[:, 1], t[:, 2], t[:, 3], tp[:, 0], tp[:, 1], tp[:, 2])
    t_bonded = time.perf_counter() - t0
    t_eval = t_pairs + t_recip + t_bonded  # energies only: forces by autograd would add ~2x
    value = n / t_eval
    sample = (f"LJ + real-space Coulomb energies of {m} sampled pair rows scaled to the estimated {npairs} "
              f"pairs ({t_pairs:.1f} s), reciprocal energy on the {s['K'][0]}^3 mesh ({t_recip:.1f} s), all "
              f"bonded terms ({t_bonded:.2f} s); energies only (no forces), a lower bound on the reference's time")
    return {"impl": "reference", "metric": METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": args.gpus,
            "steps": 1, "warmup": 0, "ms_per_step": t_eval * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "atom-evals/s", "cores": torch.get_num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "atom-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------------- GPU side
def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "c4":
        run_classical(args, rank, world, local)
        return
    from dmff_b200.synthetic import workload
    s = workload(args.workload)
    if args.impl == "reference":
        run_reference(args, s, rank)
        return
    serving_systems = None
    if args.serving_requests > 0 and world == 1:
        serving_systems = make_serving_systems(args.serving_requests)
    import torch
    import torch.distributed as dist
    from dmff_b200.engine import AdmpEngine
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    eng = AdmpEngine(s["n_atoms"], s["lmax"], s["lpol"], True, s["rc"], s["kappa"], s["K"], s["axis_types"],
                     s["axis_indices"], s["cov_rows"], s["mscales"], s["pscales"], s["dscales"], precision="fp32",
                     solver="cg", cg_tol=1e-6, max_iter=1000, device=dev)
    eng.set_params(s["Q_local"], s.get("pol"), s.get("thole"))
    eng.set_zero_guess(True)  # every step solves from U = 0 (the reference's U_init = None)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    box = s["box"]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        eng.rebuild_internal_pairs(pos, box)
        return eng.compute(pos, box)

    for _ in range(args.warmup):
        res, F, U = step()
    torch.cuda.synchronize()
    launches0 = eng.counters()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    iters = []
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            res, F, U = step()
            evs[k][1].record(stream)
            iters.append(res.n_iter)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = sum(step_ms)
    launches1 = eng.counters()
    if world > 1:
        t = torch.tensor([total_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps * s["n_atoms"] / (total_ms / 1e3)

    # e2e through the host-buffer C-ABI entry (pinned positions in, forces + dipoles out to pinned
    # caller-owned arrays)
    pos_h = torch.tensor(s["pos"], dtype=torch.float64).pin_memory().numpy()
    F_out = torch.zeros((s["n_atoms"], 3), dtype=torch.float64).pin_memory().numpy()
    U_out = torch.zeros((s["n_atoms"], 3), dtype=torch.float64).pin_memory().numpy()
    e2e_ms = []
    for k in range(args.warmup):
        eng.compute_host(pos_h, box, forces_out=F_out, U_out=U_out)
    for k in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r_h, F_h, U_h = eng.compute_host(pos_h, box, forces_out=F_out, U_out=U_out)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * args.steps * s["n_atoms"] / (e2e_total / 1e3)

    # per-kernel device times over K instrumented steps (events around every launch)
    eng.set_profiling(True)
    for k in range(args.steps):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    stats = eng.kernel_stats()
    eng.set_profiling(False)
    peaks, src = measured_peaks()
    roof = roofline(stats, s, int(res.n_pairs), peaks, src)

    out = None
    if rank == 0:
        n_iter = int(statistics.median(iters))
        out = {"metric": METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "fp32 pairs/mesh, fp64 accumulation",
               "data": "synthetic", "config": dict(workload_config(args.workload, s, s["K"]),
                                                   parallelism=f"replicas x{world}"),
               "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                              "e2e_p50": float(np.percentile(e2e_ms, 50)), "e2e_p99": float(np.percentile(e2e_ms, 99))},
               "e2e": {"value": e2e_value, "unit": "atom-evals/s", "h2d_bytes_per_step": 3 * 8 * s["n_atoms"],
                       "d2h_bytes_per_step": 2 * 3 * 8 * s["n_atoms"],
                       "path": "dmffb_admp_compute_host (C ABI, host buffers)"},
               "roofline": roof, "clocks": clk.summary(),
               "gpu_launches": int(launches1["launches"] - launches0["launches"]),
               "library_launches": {"cufft_execs": int(launches1["fft_execs"] - launches0["fft_execs"])},
               "result": {"energy_kJmol": res.energy, "cg_iters": n_iter, "converged": int(res.converged),
                          "n_pairs": int(res.n_pairs)},
               "kernel_ms_per_step": {k: v[0] / args.steps for k, v in stats.items() if v[1]}}
        if world == 1 and not args.no_cpu_baseline:
            t_g, t_ef, cores = cpu_reference_timing(s, n_iter)
            t_eval = t_ef + n_iter * t_g
            out["cpu_baseline"] = {
                "value": s["n_atoms"] / t_eval, "unit": "atom-evals/s", "cores": cores, "kind": "port",
                "sample": (f"one dE/dU pass ({t_g:.2f} s) and one energy+forces pass ({t_ef:.2f} s) of the same "
                           f"box with the float64 oracle; evaluation = E+F + {n_iter} dE/dU passes (the GPU's CG "
                           f"iteration count)")}
        if serving_systems is not None:
            out["serving"] = bench_serving(args, serving_systems, dev)
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
