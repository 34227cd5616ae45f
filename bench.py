"""Benchmark of the ADMP polarizable PME energy/force/virial step on B200.

Workload (default, the headline line): 4096 rigid waters (12288 atoms) in a 49.7 A box, lmax=2
multipoles with local frames, isotropic polarizabilities (O 1.0, H 0.5 A^3), Thole 0.33, rc = 8 A,
ethresh = 5e-4 (kappa 0.3285/A, 50^3 mesh); seeded synthetic coordinates and parameters.
One step = cell-list neighbour rebuild + induced-dipole CG solve (from U = 0) + energy,
forces and box gradient, FP32 pair / mesh arithmetic with FP64 accumulation.

The same line carries two more measurements of this path at N = 1:
  "c4": the 100 000-atom classical polymer + water box (LJ + Coulomb PME + bonded, rc 10 A);
  "c3": the serving stream (2000 polarizable water boxes of 100-10000 molecules, Poisson
        arrivals at 50 ... 2000 requests/s) on the batched FP32 server and on the plain FP64 path.

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
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atom-evals/s"
L2_FLUSH_BYTES = 256 << 20
POL_CONV, MAX_N_POL = 1.0, 30  # the reference's dipole iteration limits (dmff/admp/settings.py:2-3)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="c1", choices=["c0", "c1", "c2", "c4"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-c4", action="store_true", help="skip the classical 100k-atom sub-measurement")
    p.add_argument("--serving-requests", type=int, default=2000,
                   help="requests of the serving stream measured beside the step (0: skip)")
    p.add_argument("--serving-rates", default="50,100,200,500,1000,2000", help="Poisson arrival rates (req/s)")
    p.add_argument("--serving-slots", type=int, default=8)
    p.add_argument("--serving-budget-gb", type=float, default=8.0)
    p.add_argument("--cg", default="auto", choices=["auto", "persistent", "per-pass"],
                   help="dipole solve: persistent CG kernel, graph-replayed per-pass solve, or the "
                        "engine's size rule (persistent up to 4096 atoms)")
    p.add_argument("--size-sweep", action="store_true",
                   help="per-request latency of single serving boxes (150-9000 waters) with the per-pass and "
                        "the persistent dipole solve, one JSON line, then exit")
    p.add_argument("--fused-fft", action="store_true",
                   help="dipole-solve convolution through the engine's FFT kernels instead of cuFFT")
    return p.parse_args()


def workload_config(name, s, world=1):
    """config of the JSON line; the same keys on both arms."""
    return {"workload": {"c1": "polarizable ADMP water box, 4096 waters / 12288 atoms, 49.7 A, rc 8 A",
                         "c0": "ADMP water box, 216 waters / 648 atoms, 18.6 A, rc 6 A, no polarization",
                         "c2": "polarizable ADMP water box, 2048 waters / 6144 atoms, 40 A, rc 8 A"}[name],
            "n_atoms": int(s["n_atoms"]), "lmax": int(s["lmax"]), "polarizable": bool(s["lpol"]),
            "rc_A": s["rc"], "ethresh": s["ethresh"], "pme_mesh": [int(k) for k in s["K"]],
            "cg_tol_rel": 1e-6, "l2": "flushed between timed steps (256 MiB write)",
            "step": "cell-list rebuild + dipole solve from U=0 + energy/forces/box gradient",
            "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock, power and clock-event reasons sampled while the timed region runs: one
    ``nvidia-smi --query-gpu ... -lms 20`` process (read-only queries, a sample every 20 ms) from
    entry to exit, its CSV parsed afterwards."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    PERIOD_MS = 20

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []  # (sm_mhz, max_mhz, [reason names])
        self._p = None

    def __enter__(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                        "--format=csv,noheader,nounits", "-lms", str(self.PERIOD_MS)],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        time.sleep(2 * self.PERIOD_MS / 1000.0)  # at least one sample after the timed region
        self._p.terminate()
        try:
            out, _ = self._p.communicate(timeout=10)
        except Exception:
            self._p.kill()
            out, _ = self._p.communicate()
        for line in out.strip().splitlines():
            r = [x.strip() for x in line.split(",")]
            if len(r) >= 9 and r[1].replace(".", "").isdigit():
                self.rows.append((float(r[1]), float(r[2]),
                                  [n for k, n in enumerate(self.NAMES) if r[5 + k] == "Active"]))

    def summary(self):
        sm = [r[0] for r in self.rows]
        mx = [r[1] for r in self.rows]
        reasons = sorted({n for r in self.rows for n in r[2]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm), "source": f"nvidia-smi -lms {self.PERIOD_MS}"}


# ---------------------------------------------------------------------------------- roofline
def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "sm_max_mhz": 1965.0}, "fallback"


def measure_fp32_peak(dev):
    """FP32 CUDA-core throughput measured in this run: cuBLAS SGEMM 8192^3 with TF32 off (FFMA
    only), best of 5 (TFLOP/s).  The pair kernels are FP32 CUDA-core code, so this is their bound."""
    import torch
    prev = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    try:
        n = 8192
        a = torch.randn((n, n), device=dev, dtype=torch.float32)
        b = torch.randn((n, n), device=dev, dtype=torch.float32)
        c = a @ b
        best = 1e30
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            torch.matmul(a, b, out=c)
            e1.record()
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        del a, b, c
        return 2.0 * n ** 3 / best / 1e12
    finally:
        torch.backends.cuda.matmul.allow_tf32 = prev


def class_rooflines(stats, steps, work, fp32_peak, hbm_peak):
    """Per kernel class: launches per step, device time per step and per launch (CUDA events around
    every launch of that class, summed over ``steps`` instrumented steps), and the achieved rate of
    its algorithmic work per launch against its bound.  ``work[cls] = (bound, units per launch)``
    with bound 'fp32' (flop) or 'hbm' (bytes)."""
    out = {}
    total = sum(v[0] for v in stats.values())
    for cls, (ms, launches) in stats.items():
        if launches == 0:
            continue
        per = ms / 1e3 / launches
        row = {"ms_per_step": round(ms / steps, 4), "launches_per_step": launches / steps,
               "avg_launch_us": round(per * 1e6, 2), "share": round(ms / total, 4) if total else None}
        if cls in work and work[cls][1] > 0:
            bound, units = work[cls]
            if bound == "fp32":
                ach = units / per / 1e12
                row.update(bound="fp32", achieved=round(ach, 3), unit="TFLOP/s", frac=round(ach / fp32_peak, 4))
            elif bound == "fp64":
                ach = units / per / 1e12
                row.update(bound="fp64 (rows with a topological scale)", achieved=round(ach, 3), unit="TFLOP/s")
            else:
                ach = units / per / 1e9
                row.update(bound="hbm", achieved=round(ach, 1), unit="GB/s", frac=round(ach / hbm_peak, 4))
        out[cls] = row
    return out


def cg_solve_bytes(s, n_pairs, iters):
    """Algorithmic bytes of one persistent CG solve (k_cg_solve) of ``iters`` iterations, per
    iteration: the matvec's 12 B per CSR entry (24 B per pair), the dipole spread and field gather
    (N(12 + 16) + 4K^3 and 4K^3 + N(12 + 16 + 24)), the three FFT passes (mesh read, spectrum
    written, spectrum read and written by the column pass, spectrum read, mesh written: 24 K^3 in
    FP32 complex half-spectrum units counted as 4 B per real mesh point), and the CG vectors (the
    direction update reads z, p and writes p; the update reads p, Ap, fmv, r, x, pol and writes x,
    r, z: 24 + 80 B per atom component)."""
    n = s["n_atoms"]
    K3 = float(np.prod(s["K"]))
    per_iter = 24.0 * n_pairs + n * (12 + 16) + 4 * K3 + 4 * K3 + n * (12 + 16 + 24) + 24 * K3 + 3 * n * (24 + 80)
    return iters * per_iter


def admp_work(s, n_pairs, n_scaled, iters=0):
    """Algorithmic work per launch of each class for a polarizable ADMP step (fixed convention:
    FMA = 2 flop, exp / erf / erfc / sqrt / div = 1 flop): pair FULL polarizable 1900 flop/pair,
    FIELD 600 flop/pair, the CG matvec 12 B per CSR entry (two entries per pair: packed j + two
    FP32 coefficients), its coefficient set-up 200 flop/pair, dipole spread N(12 + 4*4) + 4K^3 B,
    field gather 4K^3 + N(12 + 4*4 + 24) B, convolution 16 K^3 B, neighbour build 12N + 12Np B per
    step (its launches share it).  Pair classes count the rows they run over: the FP32 launches
    take the unscaled rows, the FP64 launches the n_scaled rows with a topological scale."""
    n = s["n_atoms"]
    K3 = float(np.prod(s["K"]))
    un = n_pairs - n_scaled
    return {"pair_full": ("fp32", 1900.0 * un), "pair_field": ("fp32", 600.0 * un),
            "pair_full_scaled": ("fp64", 1900.0 * n_scaled), "pair_field_scaled": ("fp64", 600.0 * n_scaled),
            "pair_matvec": ("hbm", 12.0 * 2 * n_pairs), "matvec_coef": ("fp32", 200.0 * n_pairs),
            "spread": ("hbm", n * (12 + 4 * 4) + 4 * K3), "gather_field": ("hbm", 4 * K3 + n * (12 + 16 + 24)),
            "conv": ("hbm", 16 * K3), "cg_persistent": ("hbm", cg_solve_bytes(s, n_pairs, iters))}


def headline_roofline(classes, per_launch_bytes, traffic, peak, peak_src, kernel, cls):
    """The roofline object of the line: the dominant kernel's achieved rate of algorithmic bytes
    per launch (live CUDA events over the instrumented steps) against the measured HBM peak."""
    row = classes[cls]
    ach = per_launch_bytes / (row["avg_launch_us"] * 1e-6) / 1e9
    return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "unit": "GB/s", "frac": round(ach / peak, 4),
            "traffic": traffic, "kernel": kernel, "kernel_class": cls, "avg_launch_us": row["avg_launch_us"],
            "share_of_step": row["share"], "peak_source": f"hbm_gbs ({peak_src})"}


# ---------------------------------------------------------------------------------- CPU side
def cpu_sample_system():
    """The bounded CPU sample of the c1 workload: 512 waters (1536 atoms) in a 24.85 A box, the same
    density, seed, force field, rc 8 A and ethresh (so the same kappa and mesh spacing, 25^3)."""
    from dmff_b200.synthetic import water_box
    return water_box(512, 49.7 / 2, seed=1, lmax=2, pol=True, rc=8.0)


def cpu_reference_evaluation(s, f, pr, tensors):
    """One complete evaluation by the reference's own algorithm, restated in float64 (the oracle):
    the fixed-point dipole iteration to POL_CONV (max |dE/dU| < 1 over sites with pol > 0.001,
    at most MAX_N_POL steps, dmff/admp/pme.py:373-401) from U = 0, then energy + forces + box
    gradient by autograd (jax.value_and_grad over positions and box, pme.py:339).  Returns
    (seconds, iterations)."""
    import torch
    Ql, pol, th, ms, ps, ds = tensors
    t0 = time.perf_counter()
    pos = torch.tensor(s["pos"])
    box = torch.tensor(s["box"])
    U, _, n_it = f.optimize_Uind(pos, box, pr, Ql, pol, th, ms, ps, ds, steps_pol=None, maxiter=MAX_N_POL,
                                 thresh=POL_CONV)
    p = pos.clone().requires_grad_(True)
    b = box.clone().requires_grad_(True)
    E = f.energy_fn(p, b, pr, Ql, U.detach(), pol, th, ms, ps, ds)
    torch.autograd.grad(E, (p, b))
    return time.perf_counter() - t0, int(n_it)


def cpu_reference_runner():
    """Set-up of the CPU sample (untimed: pair list and parameters); returns a callable that runs
    one timed evaluation, and the thread count used."""
    import torch
    import oracle.admp_ref as R
    from dmff_b200.synthetic import pairs_nbond
    torch.set_num_threads(os.cpu_count())
    s = cpu_sample_system()
    pr = R.brute_force_pairs(s["pos"], s["box"], s["rc"])
    pr[:, 2] = pairs_nbond(pr, s["cov_rows"], s["n_atoms"])
    f = R.ADMPPmeForce(s["box"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], s["lmax"], s["lpol"],
                       kappa=s["kappa"], K=s["K"])
    tensors = (torch.tensor(s["Q_local"]), torch.tensor(s["pol"]), torch.tensor(s["thole"]),
               torch.tensor(s["mscales"]), torch.tensor(s["pscales"]), torch.tensor(s["dscales"]))
    return s, (lambda: cpu_reference_evaluation(s, f, pr, tensors)), torch.get_num_threads()


def cpu_sample_text(s, iters, secs):
    return (f"complete evaluations of a {s['n_atoms']}-atom sample of the workload ({s['n_atoms'] // 3} waters, "
            f"24.85 A, same density / rc / ethresh, {s['K'][0]}^3 mesh) by the float64 restatement of the "
            f"reference: fixed-point dipole iteration to POL_CONV 1.0 (max {MAX_N_POL} steps; took "
            f"{statistics.median(iters):.0f}) + energy/forces/box gradient by autograd; median "
            f"{statistics.median(secs):.2f} s per evaluation")


def run_reference(args, s_full, rank):
    """--impl reference: the reference's own CPU algorithm for the path (float64 restatement; JAX
    is not installed) on all host cores, on a bounded sample of the workload; every step is one
    complete, timed evaluation."""
    if rank != 0:
        return
    s, run, cores = cpu_reference_runner()
    for _ in range(args.warmup):
        run()
    secs, iters = [], []
    for _ in range(args.steps):
        t, it = run()
        secs.append(t)
        iters.append(it)
    total = sum(secs)
    value = args.steps * s["n_atoms"] / total
    out = {"impl": "reference", "metric": METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": workload_config(args.workload, s_full, args.gpus),
           "cpu_baseline": {"value": value, "unit": "atom-evals/s", "cores": cores, "kind": "port",
                            "sample": cpu_sample_text(s, iters, secs)},
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
        return pool.starmap_async(serving_system, [(int(n), k) for k, n in enumerate(sizes)]).get(timeout=1800)


def serving_ideal_seconds(systems, iters, peaks, fp32_peak):
    """Ideal time t* of a set of polarizable evaluations (fixed convention): FP32 pair flops at the
    FP32 peak plus the memory-bound stages' bytes at the HBM peak.  Per request: pairs Np from the
    molecule density (0.1002 atoms/A^3 within rc), flops 1900 Np (FULL) + 600 Np (FIELD) + 200 Np
    (matvec set-up), bytes 12N + 12Np (neighbours) + per CG iteration 24 Np (matvec) + dipole spread
    N*28 + 4K^3 + gather 4K^3 + N*52 + convolution 16 K^3, cuFFT counted as 2 x 2.5 K^3 log2 K^3
    flops per iteration."""
    flops = 0.0
    byts = 0.0
    for s, it in zip(systems, iters):
        n = s["n_atoms"]
        npairs = n * 0.5 * (4.0 / 3.0) * math.pi * s["rc"] ** 3 * 0.1002
        K3 = float(np.prod(s["K"]))
        flops += (1900 + 600 + 200) * npairs + it * 2 * 2.5 * K3 * math.log2(K3)
        byts += 12 * n + 12 * npairs + it * (24 * npairs + 28 * n + 8 * K3 + 52 * n + 16 * K3)
    return flops / (fp32_peak * 1e12) + byts / (peaks["hbm_gbs"] * 1e9)


def serving_ceiling(systems, fp32_seq, plain, offline_wall_s, large_server_s):
    """Where the plain path's time goes and what cross-request batching could at most gain: per
    size bucket (waters) the requests, their share of the atoms, and the per-request service times
    of the FP32 engine and of the plain FP64 path, each run one request at a time; then bounds on
    the whole-stream speed-up over the plain path when every request below the largest bucket is
    free (perfect batching of the small, launch-bound boxes): with the largest bucket run one
    request at a time, and with it run through the server (``large_server_s``, its requests alone,
    concurrently); and with every request at the largest bucket's server rate."""
    edges = [100, 300, 1000, 3000, 10001]
    waters = np.array([s["n_atoms"] // 3 for s in systems])
    atoms = np.array([s["n_atoms"] for s in systems], dtype=np.float64)
    t32 = np.array([r.c.t_done - r.c.t_start for r in fp32_seq])
    t64 = np.array([r.c.t_done - r.c.t_start for r in plain])
    buckets = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        m = (waters >= lo) & (waters < hi)
        if not m.any():
            continue
        buckets.append({"waters": f"{lo}-{hi - 1}", "requests": int(m.sum()),
                        "atom_share": round(float(atoms[m].sum() / atoms.sum()), 4),
                        "fp32_ms_median": round(float(np.median(t32[m])) * 1e3, 3),
                        "fp64_plain_ms_median": round(float(np.median(t64[m])) * 1e3, 3),
                        "fp32_s": round(float(t32[m].sum()), 4), "fp64_plain_s": round(float(t64[m].sum()), 4),
                        "fp32_atom_evals_per_s": float(atoms[m].sum() / t32[m].sum()),
                        "fp64_plain_atom_evals_per_s": float(atoms[m].sum() / t64[m].sum())})
    top = buckets[-1]
    T64 = float(t64.sum())
    big = waters >= edges[-2]
    rate_big_server = float(atoms[big].sum()) / large_server_s
    return {"buckets": buckets, "plain_fp64_service_s": round(T64, 4),
            "fp32_sequential_service_s": round(float(t32.sum()), 4), "offline_fp32_wall_s": round(offline_wall_s, 4),
            "largest_bucket_server_s": round(large_server_s, 4),
            "largest_bucket_server_atom_evals_per_s": rate_big_server,
            "bound_small_free_largest_one_at_a_time": round(T64 / top["fp32_s"], 3),
            "bound_small_free_largest_through_server": round(T64 / large_server_s, 3),
            "bound_all_at_largest_bucket_server_rate": round(T64 / (float(atoms.sum()) / rate_big_server), 3),
            "measured_offline_speedup": round(T64 / offline_wall_s, 3)}


def bench_serving(args, systems, dev, peaks, fp32_peak):
    """The serving stream: continuous-batching FP32 server (saturation and Poisson arrivals) and the
    plain FP64 path (one request at a time, no graphs) on the same requests; latency = completion -
    arrival."""
    from dmff_b200.serving import AdmpServer, ServingRequest
    from dmff_b200.synthetic import serving_arrivals
    cap = max(s["n_atoms"] for s in systems)
    by_k = {}
    for s in systems:
        by_k.setdefault(tuple(s["K"]), s)
    warm = sorted(by_k.values(), key=lambda s: -s["n_atoms"])  # largest first: buffers grow once
    out = {"requests": len(systems), "atoms": int(sum(s["n_atoms"] for s in systems)),
           "sizes": "log-uniform 100-10000 waters (seed 3), 0.0334 molecules/A^3, rc 8 A (rc' = L/2 when L < 16 A)",
           "small_boxes_rc_reduced": int(sum(1 for s in systems if s["rc"] < 8.0)),
           "slots": args.serving_slots, "hbm_budget_GB": args.serving_budget_gb,
           "slots_budget_choice": "best of a sweep of 8-32 slots x 2 / 8 GB on this stream (8 slots, 8 GB)",
           "cg_tol_rel": 1e-6, "step": "polarizable ADMP energy + forces + virial, host buffers in and out"}
    import torch
    torch.cuda.synchronize(dev)
    free0 = torch.cuda.mem_get_info(dev)[0]
    srv = AdmpServer(n_slots=args.serving_slots, capacity_atoms=cap, precision="fp32",
                     hbm_budget_bytes=int(args.serving_budget_gb * (1 << 30)), device=dev)
    srv.prewarm([ServingRequest(s) for s in warm])
    torch.cuda.synchronize(dev)
    # device memory the slots really hold once every mesh shape has run on each (engines at the
    # largest request, grown pair and mesh buffers, cached cuFFT plans)
    used = free0 - torch.cuda.mem_get_info(dev)[0]
    out["server_device_bytes"] = {"all_slots": int(used), "per_slot": int(used // args.serving_slots),
                                  "admission": "analytical per-request footprint against the budget "
                                               "(dmffb_request_footprint); it limits how many large "
                                               "requests run at once"}
    reqs, st = srv.run_stream(systems, np.zeros(len(systems)))
    out["offline_fp32"] = st
    fp32 = reqs
    # the largest bucket (3000-10000 waters) alone through the same server: the part of the
    # stream that batching the small requests cannot remove
    big = [s for s in systems if s["n_atoms"] // 3 >= 3000]
    _, bst = srv.run_stream(big, np.zeros(len(big)))
    large_server_s = bst["wall_s"]
    iters = [r.c.n_iter for r in reqs]
    t_ideal = serving_ideal_seconds(systems, iters, peaks, fp32_peak)
    out["roofline"] = {"model": "ideal time t* = FP32 pair flops / measured FP32 peak + stage bytes / measured "
                                "HBM peak, summed over the requests (see serving_ideal_seconds)",
                       "t_ideal_s": round(t_ideal, 4), "t_measured_s": round(st["wall_s"], 4),
                       "frac": round(t_ideal / st["wall_s"], 4)}
    for rate in [float(x) for x in args.serving_rates.split(",") if x]:
        preq, st = srv.run_stream(systems, serving_arrivals(len(systems), rate, seed=33))
        # the five slowest requests: queue wait (arrival to admission) and service time
        worst = sorted(preq, key=lambda r: -r.latency)[:5]
        st["slowest"] = [{"waters": r.n_atoms // 3, "wait_ms": round((r.c.t_start - r.c.t_arrival) * 1e3, 2),
                          "service_ms": round((r.c.t_done - r.c.t_start) * 1e3, 2)} for r in worst]
        out[f"poisson_{int(rate)}_per_s"] = st
    srv.close()
    # plain path: FP64, one slot, graphs off, every request back to back
    plain = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp64", use_graphs=False, cg_tol=1e-6, device=dev)
    # the same warm-up as the server: one request per mesh shape, so that neither timed run
    # includes cuFFT plan creation
    plain.prewarm([ServingRequest(s) for s in warm])
    preqs, pst = plain.run_stream(systems, np.zeros(len(systems)))
    plain.close()
    out["plain_fp64"] = dict(pst, sample="every request of the stream, one at a time")
    out["speedup_vs_plain"] = out["offline_fp32"]["atom_evals_per_s"] / pst["atom_evals_per_s"]
    # the same plain path with the reference's own dipole iteration (fixed-point steps, POL_CONV 1.0,
    # MAX_N_POL 30, pme.py:342-423) in place of CG: the reference's algorithm run on this GPU
    plain_r = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp64", use_graphs=False, solver="reference",
                         cg_tol=POL_CONV, max_iter=MAX_N_POL, device=dev)
    plain_r.prewarm([ServingRequest(s) for s in warm])
    _, rst = plain_r.run_stream(systems, np.zeros(len(systems)))
    plain_r.close()
    out["plain_fp64_reference_solver"] = dict(rst, sample="every request of the stream, one at a time",
                                              solver="fixed-point dipole iteration, POL_CONV 1.0, MAX_N_POL 30")
    out["speedup_vs_plain_reference_solver"] = out["offline_fp32"]["atom_evals_per_s"] / rst["atom_evals_per_s"]
    # the same FP32 engine one request at a time (graphs on): per-request service times for the
    # ceiling breakdown
    seq = AdmpServer(n_slots=1, capacity_atoms=cap, precision="fp32", device=dev)
    seq.prewarm([ServingRequest(s) for s in warm])
    sreqs, sst = seq.run_stream(systems, np.zeros(len(systems)))
    seq.close()
    out["sequential_fp32"] = dict(sst, sample="every request of the stream, one at a time, graphs on")
    out["ceiling"] = serving_ceiling(systems, sreqs, preqs, out["offline_fp32"]["wall_s"], large_server_s)
    errs_e, errs_f = [], []
    for q, p in zip(fp32, preqs):
        errs_e.append(abs(q.energy - p.energy) / abs(p.energy))
        errs_f.append(float(np.sqrt(np.mean((q.forces - p.forces) ** 2)) / np.sqrt(np.mean(p.forces ** 2))))
    out["fp32_vs_fp64"] = {"max_rel_energy": float(max(errs_e)), "max_rel_force_rms": float(max(errs_f))}
    return out


# ---------------------------------------------------------------------------------- classical
def c4_system():
    from dmff_b200.synthetic import polymer_water_box
    return polymer_water_box(200, 50, 30000, 70.0, seed=4, rc=10.0, ethresh=1e-5)


C4_CFG = {"workload": "classical polymer + water, 200 x 50 beads + 30000 waters / 100000 atoms, 70 A, rc 10 A",
          "terms": "LJ (LB) + Coulomb PME + harmonic bonds/angles + periodic torsions",
          "l2": "flushed between timed steps (256 MiB write)",
          "step": "cell binning + all pairs within rc from the cell grid + PME + bonded: energy/forces/box gradient"}


def measure_c4(args, dev, peaks, fp32_peak, world=1, dist=None):
    """The 100k-atom classical step (200 chains x 50 beads + 30000 waters, 70 A box): LJ + Coulomb
    PME (rc 10 A, ethresh 1e-5, 154^3 mesh) + harmonic bonds / angles + 3-term torsions.  One step
    = cell-list rebuild + energy / forces / box gradient, FP32 pair and mesh arithmetic with FP64
    accumulation.  Returns the measurement dict (value = atom-evals/s over all ranks)."""
    import torch
    from dmff_b200.engine import ClassicalEngine
    s = c4_system()
    eng = ClassicalEngine(s["n_atoms"], n_types=len(s["sigma"]), coulomb="pme", pbc=True, rc=s["rc"], kappa=s["kappa"],
                          K=s["K"], cov_rows=s["cov_rows"], mscales_coul=s["mscales_coul"], mscales_lj=s["mscales_lj"],
                          precision="fp32", device=dev)
    eng.set_params(s["charges"], s["types"], s["sigma_tt"], s["eps_tt"])
    eng.set_terms("bond", s["bonds"], s["bond_prm"])
    eng.set_terms("angle", s["angles"], s["angle_prm"])
    eng.set_terms("torsion", s["torsions"], s["torsion_prm"])
    # every step evaluates the pairs within rc of its own positions straight from the cell grid
    # (the same pair set as a list rebuild + a compute on the list, without writing the list)
    eng.set_cell_pass(True)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def step():
        return eng.compute(pos, s["box"])

    for _ in range(args.warmup):
        res, F = step()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    l0 = eng.counters()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev.index or 0) as clk:
        for k in range(args.steps):
            flush.zero_()
            evs[k][0].record(stream)
            res, F = step()
            evs[k][1].record(stream)
        torch.cuda.synchronize()
    total = sum(a.elapsed_time(b) for a, b in evs)
    l1 = eng.counters()
    if dist is not None:
        t = torch.tensor([total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    value = world * args.steps * s["n_atoms"] / (total / 1e3)
    # e2e: pinned host positions in, forces out, through the public engine API
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
    e2e_total = sum(e2e)
    if dist is not None:
        t = torch.tensor([e2e_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * args.steps * s["n_atoms"] / e2e_total
    # per-class device times over instrumented steps
    eng.set_profiling(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    stats = eng.kernel_stats()
    eng.set_profiling(False)
    n_pairs = int(res.n_pairs)
    n = s["n_atoms"]
    K3 = float(np.prod(s["K"]))
    # the cell pass (class pair_full) tests every candidate of the 5^3 half-cell stencil and
    # evaluates each pair within rc from both of its atoms: 120 flop per pair row, counted once
    # (the list convention); binning (class neighbors) moves 12N B per step
    work = {"pair_full": ("fp32", 120.0 * n_pairs), "spread": ("hbm", n * 16 + 4 * K3),
            "gather_full": ("hbm", 4 * K3 + n * 40), "conv": ("hbm", 16 * K3)}
    nb_launches = stats["neighbors"][1] / args.steps
    if nb_launches:
        work["neighbors"] = ("hbm", 12.0 * n / nb_launches)
    classes = class_rooflines(stats, args.steps, work, fp32_peak, peaks["hbm_gbs"])
    pf = classes.get("pair_full", {})
    return {"metric": METRIC, "value": value, "unit": "atom-evals/s", "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total / args.steps, "config": dict(C4_CFG, n_atoms=int(n), pme_mesh=[int(k) for k in s["K"]],
                                                               ethresh=s["ethresh"], parallelism=f"replicas x{world}"),
            "e2e": {"value": e2e_value, "unit": "atom-evals/s", "h2d_bytes_per_step": 24 * n,
                    "d2h_bytes_per_step": 24 * n, "path": "ClassicalEngine.compute, pinned host copies"},
            "roofline": {"kernel": "k_nb_cells (LJ + erfc Coulomb from the cell grid, no pair list)", "bound": "fp32",
                         "achieved": pf.get("achieved"), "peak": round(fp32_peak, 2), "unit": "TFLOP/s",
                         "frac": pf.get("frac"), "traffic": None, "avg_launch_us": pf.get("avg_launch_us"),
                         "peak_source": "cuBLAS FP32 SGEMM (TF32 off) measured in this run",
                         "work": "120 flop per pair within rc"},
            "by_class": classes, "clocks": clk.summary(), "gpu_launches": int(l1["launches"] - l0["launches"]),
            "library_launches": {"cufft_execs": int(l1["fft_execs"] - l0["fft_execs"])},
            "result": {"energy_kJmol": res.energy, "e_coul": res.e_coul_real + res.e_coul_recip + res.e_coul_self,
                       "e_lj": res.e_lj, "e_bonded": res.e_bond + res.e_angle + res.e_torsion, "n_pairs": n_pairs}}


def run_classical(args, rank, world, local):
    """--workload c4: the classical step alone as the line (the default line carries it as "c4")."""
    import torch
    if args.impl == "reference":
        if rank != 0:
            return
        print(json.dumps(classical_cpu_reference(c4_system(), dict(C4_CFG), args)), flush=True)
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    peaks, src = measured_peaks()
    fp32_peak = measure_fp32_peak(dev)
    m = measure_c4(args, dev, peaks, fp32_peak, world, dist)
    if rank == 0:
        out = dict(m, n_gpus=world, higher_is_better=True, scaling="weak", vs_baseline=None,
                   dtype="fp32 pairs/mesh, fp64 accumulation", data="synthetic")
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
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(cfg, n_atoms=int(n), pme_mesh=[int(k) for k in s["K"]], ethresh=s["ethresh"],
                           parallelism=f"replicas x{args.gpus}"),
            "cpu_baseline": {"value": value, "unit": "atom-evals/s", "cores": torch.get_num_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "atom-evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------------- GPU side
def size_sweep(dev):
    """One engine re-pointed at serving boxes of 150-9000 waters (three boxes per size, four passes
    each, the first dropped): median host time of reconfigure + set_params + compute_host and the
    engine's device time of the dipole solve, per-pass vs persistent CG."""
    import torch
    from dmff_b200.engine import AdmpEngine
    from dmff_b200.synthetic import serving_system
    sizes = [150, 300, 600, 1200, 2500, 5000, 9000]
    systems = {n: [serving_system(n, 100 * n + k) for k in range(3)] for n in sizes}
    s0 = systems[sizes[-1]][0]
    eng = AdmpEngine(3 * max(sizes), 2, True, True, s0["rc"], s0["kappa"], s0["K"], s0["axis_types"],
                     s0["axis_indices"], s0["cov_rows"], s0["mscales"], s0["pscales"], s0["dscales"],
                     precision="fp32", solver="cg", cg_tol=1e-6, max_iter=500, device=dev)
    out = {}
    for mode, name in ((0, "per_pass"), (1, "persistent")):
        eng.set_persistent_cg(mode)
        for n in sizes:
            rows = []
            for rep in range(4):
                for s in systems[n]:
                    t0 = time.perf_counter()
                    eng.reconfigure(s["n_atoms"], s["rc"], s["kappa"], s["K"], s["axis_types"], s["axis_indices"],
                                    s["cov_rows"], s["mscales"], s["pscales"], s["dscales"])
                    eng.set_params(s["Q_local"], s["pol"], s["thole"])
                    eng.set_timing(True)
                    res, _, _ = eng.compute_host(s["pos"], s["box"])
                    t1 = time.perf_counter()
                    solve_ms = eng.timings()[1]
                    eng.set_timing(False)
                    if rep > 0:
                        rows.append((t1 - t0, solve_ms, res.n_iter))
            r = np.median(np.array(rows), axis=0)
            out.setdefault(str(n), {"K": int(systems[n][0]["K"][0])})[name] = {
                "request_ms": round(float(r[0]) * 1e3, 3), "solve_ms": round(float(r[1]), 3), "cg_iters": int(r[2])}
    print(json.dumps({"size_sweep": out, "unit": "ms, median of 9", "waters": sizes}), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "c4":
        run_classical(args, rank, world, local)
        return
    if args.size_sweep:
        import torch
        torch.cuda.set_device(local)
        size_sweep(torch.device("cuda", local))
        return
    from dmff_b200.synthetic import workload
    s = workload(args.workload)
    if args.impl == "reference":
        run_reference(args, s, rank)
        return
    serving_systems = None
    if args.serving_requests > 0 and world == 1 and args.workload == "c1":
        serving_systems = make_serving_systems(args.serving_requests)
    import torch
    import torch.distributed as dist
    from dmff_b200.engine import AdmpEngine
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    peaks, src = measured_peaks()
    fp32_peak = measure_fp32_peak(dev)
    eng = AdmpEngine(s["n_atoms"], s["lmax"], s["lpol"], True, s["rc"], s["kappa"], s["K"], s["axis_types"],
                     s["axis_indices"], s["cov_rows"], s["mscales"], s["pscales"], s["dscales"], precision="fp32",
                     solver="cg", cg_tol=1e-6, max_iter=1000, device=dev)
    eng.set_params(s["Q_local"], s.get("pol"), s.get("thole"))
    eng.set_fused_fft(args.fused_fft)
    eng.set_persistent_cg({"auto": "auto", "persistent": 1, "per-pass": 0}[args.cg])
    if s["lpol"]:
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
    # caller-owned arrays; the call rebuilds the neighbour list for the copied-in positions)
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
        eng.compute_host(pos_h, box, forces_out=F_out, U_out=U_out)
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    e2e_total = sum(e2e_ms)
    if world > 1:
        t = torch.tensor([e2e_total], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * args.steps * s["n_atoms"] / (e2e_total / 1e3)

    # per-kernel-class device times over K instrumented steps (events around every launch)
    eng.set_profiling(True)
    for k in range(args.steps):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    stats = eng.kernel_stats()
    eng.set_profiling(False)
    n_pairs = int(res.n_pairs)
    n_scaled = int((eng.internal_pairs()[:, 2] != 0).sum().item())
    n_iter_med = int(statistics.median(iters)) if s["lpol"] else 0
    classes = class_rooflines(stats, args.steps, admp_work(s, n_pairs, n_scaled, n_iter_med), fp32_peak,
                              peaks["hbm_gbs"])
    if "cg_persistent" in classes:
        # the kernel with the largest share of the step: the persistent CG solve; its passes
        # timed on the device clock inside the kernel (CTA 0, barrier waits included)
        classes["cg_persistent"]["passes_ms_per_step"] = {k: round(v / args.steps, 4)
                                                          for k, v in eng.cg_phase_times().items()}
        roof = headline_roofline(classes, cg_solve_bytes(s, n_pairs, n_iter_med), None, peaks["hbm_gbs"], src,
                                 "k_cg_solve (persistent CG dipole solve)", "cg_persistent")
    else:
        # the per-pass solve: the CG matvec, 12 B per CSR entry
        roof = headline_roofline(classes, 12.0 * 2 * n_pairs, None, peaks["hbm_gbs"], src,
                                 "k_matvec_apply (CG matvec)", "pair_matvec")

    c4 = None
    if world == 1 and not args.no_c4 and args.workload == "c1":
        del flush
        torch.cuda.empty_cache()
        c4 = measure_c4(args, dev, peaks, fp32_peak)

    out = None
    if rank == 0:
        n_iter = int(statistics.median(iters)) if s["lpol"] else 0
        out = {"metric": METRIC, "value": value, "unit": "atom-evals/s", "n_gpus": world, "steps": args.steps,
               "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "fp32 pairs/mesh, fp64 accumulation",
               "data": "synthetic", "config": workload_config(args.workload, s, world),
               "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99)),
                              "e2e_p50": float(np.percentile(e2e_ms, 50)), "e2e_p99": float(np.percentile(e2e_ms, 99))},
               "e2e": {"value": e2e_value, "unit": "atom-evals/s", "h2d_bytes_per_step": 3 * 8 * s["n_atoms"],
                       "d2h_bytes_per_step": 2 * 3 * 8 * s["n_atoms"],
                       "path": "dmffb_admp_compute_host (C ABI, host buffers)"},
               "roofline": roof, "fp32_peak_tflops": round(fp32_peak, 2),
               "fp32_peak_source": "cuBLAS FP32 SGEMM 8192^3 (TF32 off), measured in this run",
               "by_class": classes, "clocks": clk.summary(),
               "gpu_launches": int(launches1["launches"] - launches0["launches"]),
               "library_launches": {"cufft_execs": int(launches1["fft_execs"] - launches0["fft_execs"])},
               "result": {"energy_kJmol": res.energy, "cg_iters": n_iter, "converged": int(res.converged),
                          "n_pairs": n_pairs, "n_pairs_scaled": n_scaled}}
        pcg = eng.persistent_cg_blocks() > 0
        out["config"]["dipole_solve"] = (f"persistent CG kernel k_cg_solve ({eng.persistent_cg_blocks()} co-resident CTAs)"
                                         if pcg else "graph-replayed per-pass CG")
        out["config"]["dipole_convolution"] = ("engine FFT passes inside k_cg_solve" if pcg else
                                               "engine FFT kernels (k_fc_*)" if eng.fused_fft_active()
                                               else "cuFFT R2C + k_conv + cuFFT C2R")
        if world == 1 and not args.no_cpu_baseline:
            cs, run, cores = cpu_reference_runner()
            run()  # warm-up
            secs, its = [], []
            for _ in range(2):
                t, it = run()
                secs.append(t)
                its.append(it)
            out["cpu_baseline"] = {"value": cs["n_atoms"] / statistics.median(secs), "unit": "atom-evals/s",
                                   "cores": cores, "kind": "port", "sample": cpu_sample_text(cs, its, secs)}
        if c4 is not None:
            out["c4"] = c4
        if serving_systems is not None:
            out["c3"] = bench_serving(args, serving_systems, dev, peaks, fp32_peak)
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
