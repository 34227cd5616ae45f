"""GPU parity at the benchmark configurations themselves, against the float64 oracle.

c0 (216 waters, seed 0, 18.6 A, lmax 2, no polarization) and c1 (4096 waters / 12288 atoms,
seed 1, 49.7 A, polarizable, rc 8 A, 50^3 mesh) run exactly as the benchmark builds them; c2 (2048
waters / 6144 atoms, 40 A) runs polarizable ADMP plus dispersion PME with Tang-Toennies damping,
with energies, forces and parameter gradients against the oracle and per-type gradients against
central finite differences.  The neighbour lists the engine builds for itself (the block-per-cell
kernel at c1 density, the warp-per-atom kernel at the density of the 100k-atom classical box) are
compared with the oracle's brute-force set row for row.  Reference semantics:
dmff/admp/pme.py:186-232 (ADMPPmeForce.get_energy), dmff/admp/disp_pme.py:45-130,
dmff/admp/pairwise.py:47-118, dmff/common/nblist.py:27-55.
"""
import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.engine import ClassicalEngine, DispEngine
from dmff_b200.synthetic import disp_params, pairs_nbond, polymer_water_box, workload
from tests.helpers import make_engine, oracle_pairs, oracle_reference, rel_force_rms

pytestmark = pytest.mark.gpu

# FP32 path: the north-star bar (energy 1e-5 relative, forces 1e-4 relative RMS); the FP64
# instantiation of the same kernels is held to the oracle far tighter
TOL = {"fp32": dict(e=1e-5, f=1e-4, b=1e-4, u=1e-4), "fp64": dict(e=1e-10, f=1e-8, b=1e-8, u=1e-8)}


def _sorted_rows(a):
    a = np.asarray(a, dtype=np.int64).reshape(-1, 3)
    return a[np.lexsort((a[:, 1], a[:, 0]))]


def _relmax(got, want):
    got, want = np.asarray(got), np.asarray(want)
    return float(np.abs(got - want).max() / max(np.abs(want).max(), 1e-300))


def _bench_path(eng, s):
    """The benchmark's step: the engine builds its own list, the solve starts from U = 0."""
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    if s["lpol"]:
        eng.set_zero_guess(True)
    eng.rebuild_internal_pairs(pos, s["box"])
    res, F, U = eng.compute(pos, s["box"])
    torch.cuda.synchronize()
    return res, F.cpu().numpy().copy(), None if U is None else U.cpu().numpy().copy()


def _check(res, F, U, ref, prec, n_pairs):
    t = TOL[prec]
    assert res.n_pairs == n_pairs
    assert abs(res.energy - ref["E"]) <= t["e"] * abs(ref["E"]), (res.energy, ref["E"])
    assert rel_force_rms(F, ref["F"]) <= t["f"]
    bg = np.array(res.box_grad).reshape(3, 3)
    assert np.abs(bg - ref["box_grad"]).max() <= t["b"] * np.abs(ref["box_grad"]).max()
    if ref["U"] is not None:
        assert res.converged == 1
        assert _relmax(U, ref["U"]) <= t["u"]


# ------------------------------------------------------------------------------------------- c0
@pytest.fixture(scope="module")
def c0():
    s = workload("c0")
    pr = oracle_pairs(s)
    return s, pr, oracle_reference(s, pr)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_c0_matches_oracle(c0, prec):
    s, pr, ref = c0
    eng = make_engine(s, precision=prec)
    res, F, U = _bench_path(eng, s)
    _check(res, F, U, ref, prec, len(pr))
    assert np.array_equal(_sorted_rows(eng.internal_pairs().cpu().numpy()), _sorted_rows(pr))


# ------------------------------------------------------------------------------------------- c1
@pytest.fixture(scope="module")
def c1():
    s = workload("c1")
    pr = oracle_pairs(s)  # 1.35 M rows, float64 brute force
    # CG in the oracle to an RMS dE/dU of 1e-8 (about 1e-10 of the permanent field's RMS)
    return s, pr, oracle_reference(s, pr, solver="cg", tol=1e-8)


def test_c1_neighbour_list_is_the_oracle_set(c1):
    """The block-per-cell build (half-width cells, candidates staged in shared memory) at c1."""
    s, pr, _ = c1
    eng = make_engine(s, precision="fp32")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.rebuild_internal_pairs(pos, s["box"])
    got = eng.internal_pairs().cpu().numpy()
    assert len(got) == len(pr) > 1_300_000
    assert np.array_equal(_sorted_rows(got), _sorted_rows(pr))
    # the allocating public builder gives the same set
    assert np.array_equal(_sorted_rows(eng.build_neighbors(pos, s["box"], s["rc"]).cpu().numpy()), _sorted_rows(pr))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_c1_matches_oracle(c1, prec):
    """Energy, forces, box gradient and induced dipoles of the benchmark's own step."""
    s, pr, ref = c1
    eng = make_engine(s, precision=prec, cg_tol=1e-11 if prec == "fp64" else 1e-6)
    res, F, U = _bench_path(eng, s)
    _check(res, F, U, ref, prec, len(pr))


# ------------------------------------------------------------------------------------------- c2
@pytest.fixture(scope="module")
def c2():
    s = workload("c2")
    d = disp_params(2048, seed=2)
    pr = oracle_pairs(s)
    ref = oracle_reference(s, pr, solver="cg", tol=1e-8)
    # parameter gradients of the ADMP energy at the converged dipoles (stationary in U)
    f = R.ADMPPmeForce(s["box"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], s["lmax"], s["lpol"],
                       kappa=s["kappa"], K=s["K"])
    Ql = torch.tensor(s["Q_local"], requires_grad=True)
    pol = torch.tensor(s["pol"], requires_grad=True)
    th = torch.tensor(s["thole"], requires_grad=True)
    ms, ps, ds = (torch.tensor(s[k]) for k in ("mscales", "pscales", "dscales"))
    E = f.energy_fn(torch.tensor(s["pos"]), torch.tensor(s["box"]), pr, Ql, torch.tensor(ref["U"]), pol, th, ms, ps, ds)
    ref["gQ"], ref["gpol"], ref["gthole"] = (g.numpy() for g in torch.autograd.grad(E, (Ql, pol, th)))
    # dispersion PME (C6/C8/C10) + Tang-Toennies short range, energies / forces / parameter grads
    pos = torch.tensor(s["pos"], requires_grad=True)
    box = torch.tensor(s["box"], requires_grad=True)
    c = torch.tensor(d["c_list"], requires_grad=True)
    a, b, q = (torch.tensor(d[k], requires_grad=True) for k in ("a", "b", "q"))
    dms = torch.tensor(d["mscales"])
    fd = R.ADMPDispPmeForce(s["box"], s["rc"], s["ethresh"], 10)
    Elr = fd.get_energy(pos, box, pr, c, dms)
    Esr = R.pairwise_energy(R.TT_damping_qq_c6_kernel, pos, box, pr, dms, a, b, q, c[:, 0])
    glr = torch.autograd.grad(Elr, (pos, box, c), retain_graph=True)
    gsr = torch.autograd.grad(Esr, (pos, box, a, b, q, c))
    disp = dict(Elr=Elr.item(), Esr=Esr.item(), Flr=-glr[0].numpy(), Fsr=-gsr[0].numpy(), Blr=glr[1].numpy(),
                Bsr=gsr[1].numpy(), gc=glr[2].numpy(), ga=gsr[2].numpy(), gb=gsr[3].numpy(), gq=gsr[4].numpy(),
                gc6=gsr[5][:, 0].numpy())
    return s, d, pr, ref, disp


@pytest.mark.parametrize("prec,ptol", [("fp64", 1e-7), ("fp32", 2e-4)])
def test_c2_admp_energy_forces_param_grads(c2, prec, ptol):
    s, d, pr, ref, _ = c2
    eng = make_engine(s, precision=prec, cg_tol=1e-11 if prec == "fp64" else 1e-6)
    eng.set_param_grads(True)
    res, F, U = _bench_path(eng, s)
    _check(res, F, U, ref, prec, len(pr))
    pg = eng.param_grads()
    assert _relmax(pg["Q_local"].cpu().numpy(), ref["gQ"]) < ptol
    assert _relmax(pg["pol"].cpu().numpy(), ref["gpol"]) < ptol
    assert _relmax(pg["thole"].cpu().numpy(), ref["gthole"]) < ptol


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_c2_dispersion_and_tt(c2, prec):
    s, d, pr, _, ref = c2
    t = TOL[prec]
    eng = DispEngine(s["n_atoms"], 10, True, s["rc"], s["kappa"], s["K"], s["cov_rows"], d["mscales"], tt=True,
                     precision=prec)
    eng.set_params(d["c_list"], d["a"], d["b"], d["q"])
    eng.set_param_grads(True)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.rebuild_internal_pairs(pos, s["box"])
    res, (Flr, Fsr) = eng.compute(pos, s["box"])
    assert res.n_pairs == len(pr)
    assert abs(res.energy - ref["Elr"]) <= t["e"] * abs(ref["Elr"])
    assert abs(res.e_sr - ref["Esr"]) <= t["e"] * abs(ref["Esr"])
    assert rel_force_rms(Flr.cpu().numpy(), ref["Flr"]) <= t["f"]
    assert rel_force_rms(Fsr.cpu().numpy(), ref["Fsr"]) <= t["f"]
    assert np.abs(np.array(res.box_grad[:]).reshape(3, 3) - ref["Blr"]).max() <= t["b"] * np.abs(ref["Blr"]).max()
    pg = eng.param_grads()
    ptol = 1e-8 if prec == "fp64" else 1e-4
    for key, want in (("c", ref["gc"]), ("a", ref["ga"]), ("b", ref["gb"]), ("q", ref["gq"]), ("c6", ref["gc6"])):
        assert _relmax(pg[key].cpu().numpy(), want) < ptol, key


def test_c2_per_type_gradients_vs_finite_differences(c2):
    """Per-type gradients at the full c2 size through the drop-in autograd path (FP64 engine, CG
    to 1e-12 relative) against central differences h = 1e-5 of the same energy, re-solving the
    dipoles at every displaced parameter."""
    from dmff_b200.admp.pme import ADMPPmeForce
    s = c2[0]
    types = torch.as_tensor(s["types"])
    f = ADMPPmeForce(s["box"], s["types"], s["axis_types"], s["axis_indices"], s["rc"], s["ethresh"], 2, True, True,
                     cov_rows=s["cov_rows"], precision="fp64", cg_tol=1e-12, max_iter=2000)
    pr = c2[2]
    Qt = torch.tensor(s["Q_type"], requires_grad=True)
    pt = torch.tensor([1.0, 0.5], dtype=torch.float64, requires_grad=True)
    tt = torch.tensor([0.33, 0.33], dtype=torch.float64, requires_grad=True)
    ms, ps, ds = (torch.tensor(s[k]) for k in ("mscales", "pscales", "dscales"))
    pos, box = torch.tensor(s["pos"]), torch.tensor(s["box"])

    def energy(Q, p, t):
        return f.get_energy(pos, box, pr, Q[types], p[types], t[types], ms, ps, ds,
                            U_init=torch.zeros((s["n_atoms"], 3)))

    E = energy(Qt, pt, tt)
    gQ, gp, gt = torch.autograd.grad(E, (Qt, pt, tt))
    h = 1e-5
    with torch.no_grad():
        for k, grad, idx in [(0, gQ, (0, 0)), (0, gQ, (0, 1)), (0, gQ, (1, 4)), (1, gp, (0,)), (1, gp, (1,)),
                             (2, gt, (0,))]:
            args = [Qt.detach().clone(), pt.detach().clone(), tt.detach().clone()]
            base = args[k][idx].item()
            args[k][idx] = base + h
            ep = energy(*args).item()
            args[k][idx] = base - h
            em = energy(*args).item()
            fdv = (ep - em) / (2 * h)
            assert abs(fdv - grad[idx].item()) <= 1e-5 * max(abs(fdv), 1.0), (k, idx, fdv, grad[idx].item())


def test_c2_dispersion_per_type_c6_vs_finite_differences(c2):
    """dE_lr/dC6 of the oxygen type (per-atom adjoints through c = sqrt(C6 1e6)) against central
    differences of the FP64 engine energy."""
    s, d = c2[0], c2[1]
    eng = DispEngine(s["n_atoms"], 10, True, s["rc"], s["kappa"], s["K"], s["cov_rows"], d["mscales"], tt=False,
                     precision="fp64")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    C = d["C_type"].copy()
    types = np.tile([0, 1, 1], s["n_atoms"] // 3)

    def energy(Cmat, grads=False):
        eng.set_params(np.sqrt(Cmat[types] * np.array([1e6, 1e8, 1e10])))
        eng.set_param_grads(grads)
        res, _ = eng.compute(pos, s["box"])
        return res.energy, (eng.param_grads()["c"].cpu().numpy() if grads else None)

    E0, gc = energy(C, True)
    c_list = np.sqrt(C[types] * np.array([1e6, 1e8, 1e10]))
    # dE/dC6_O = sum over oxygens of dE/dc * dc/dC6, c = sqrt(1e6 C6)
    want = float(np.sum(gc[types == 0, 0] * 0.5 * 1e6 / c_list[types == 0, 0]))
    h = 1e-5 * C[0, 0]
    Cp, Cm = C.copy(), C.copy()
    Cp[0, 0] += h
    Cm[0, 0] -= h
    fdv = (energy(Cp)[0] - energy(Cm)[0]) / (2 * h)
    assert abs(fdv - want) <= 1e-6 * abs(fdv)


# ------------------------------------------------------------------------------- c4 density
def test_neighbour_list_at_classical_box_density():
    """A 40 A block at the density of the 100k-atom polymer + water box (rc 10 A, ~4 600
    candidates per atom): the engine takes the warp-per-atom build; its rows equal the oracle's
    brute-force set, nbond included."""
    scale = (40.0 / 70.0) ** 3
    s = polymer_water_box(int(round(200 * scale)), 50, int(round(30000 * scale)), 40.0, seed=4, rc=10.0,
                          ethresh=1e-5)
    assert abs(s["n_atoms"] / 40.0 ** 3 - 100000 / 70.0 ** 3) < 0.01 * 100000 / 70.0 ** 3
    want = R.brute_force_pairs(s["pos"], s["box"], 10.0)
    want[:, 2] = pairs_nbond(want, s["cov_rows"], s["n_atoms"])
    eng = ClassicalEngine(s["n_atoms"], n_types=len(s["sigma"]), coulomb="pme", pbc=True, rc=10.0, kappa=s["kappa"],
                          K=s["K"], cov_rows=s["cov_rows"], mscales_coul=s["mscales_coul"],
                          mscales_lj=s["mscales_lj"], precision="fp32")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.rebuild_internal_pairs(pos, s["box"])
    got = eng.internal_pairs().cpu().numpy()
    assert len(got) == len(want) > 10_000_000
    assert np.array_equal(_sorted_rows(got), _sorted_rows(want))
