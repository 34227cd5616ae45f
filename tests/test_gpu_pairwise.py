"""The built-in short-range kernels of dmff/admp/pairwise.py on the GPU engine's pair kernel
(dmffb_pairwise_*), through the drop-in ``generate_pairwise_interaction``: energy, forces, box
gradient and per-atom parameter gradients against the float64 oracle (FP64 and FP32 engines),
second derivatives against the oracle's double autograd, the reference's edge cases (padding rows,
rows with i > j, the nbond column, an empty pair set), the engine's own neighbour list, and the
nine PEG dimer energies of the reference's short-range test (tests/test_admp/test_slater.py)."""
import json
import os

import numpy as np
import pytest
import torch

import oracle.admp_ref as R
from dmff_b200.admp.pairwise import (TT_damping_qq_c6_kernel, TT_damping_qq_kernel, generate_pairwise_interaction,
                                     slater_disp_damping_kernel, slater_sr_kernel)
from dmff_b200.synthetic import pairs_nbond, water_box

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "golden", "data")

# (ours, oracle, per-atom parameter ranges in kernel order, Angstrom units)
KERNELS = {
    "tt_qq": (TT_damping_qq_kernel, R.TT_damping_qq_kernel, [(3.5, 4.5), (-0.8, 0.4)]),
    "slater_disp": (slater_disp_damping_kernel, R.slater_disp_damping_kernel,
                    [(3.5, 4.5), (0.5, 1.5), (1.0, 3.0), (2.0, 6.0)]),
    "slater_sr": (slater_sr_kernel, R.slater_sr_kernel, [(5.0, 15.0), (3.5, 4.5)]),
    "tt_qq_c6": (TT_damping_qq_c6_kernel, R.TT_damping_qq_c6_kernel,
                 [(50.0, 90.0), (3.5, 4.5), (-0.8, 0.4), (0.5, 1.5)]),
}
MS = [0.0, 0.0, 0.5, 1.0, 1.0, 1.0]


def _system(seed=6, n_pad=25):
    s = water_box(64, 12.4, seed=seed, lmax=0, pol=False, rc=5.0)
    pairs = R.brute_force_pairs(s["pos"], s["box"], 5.0)
    pairs[:, 2] = pairs_nbond(pairs, s["cov_rows"], s["n_atoms"])
    n = s["n_atoms"]
    pad = np.full((n_pad, 3), n)
    pad[:, 2] = 0
    return s, np.concatenate([pairs, pad])


def _params(name, n, seed=3):
    rng = np.random.default_rng(seed)
    return [torch.tensor(rng.uniform(lo, hi, n), dtype=torch.float64) for lo, hi in KERNELS[name][2]]


def _eval(fn, pos, box, pairs, prm, ms, create_graph=False):
    pos = pos.clone().requires_grad_(True)
    box = box.clone().requires_grad_(True)
    prm = [p.clone().requires_grad_(True) for p in prm]
    E = fn(pos, box, pairs, ms, *prm)
    g = torch.autograd.grad(E, [pos, box] + prm, create_graph=create_graph)
    return E, g, (pos, box, prm)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", list(KERNELS))
def test_kernel_matches_oracle(name, precision):
    s, pairs = _system()
    ours, ref, _ = KERNELS[name]
    prm = _params(name, s["n_atoms"])
    ms = torch.tensor(MS, dtype=torch.float64)
    pos = torch.tensor(s["pos"], dtype=torch.float64)
    box = torch.tensor(s["box"], dtype=torch.float64)
    E, g, _ = _eval(generate_pairwise_interaction(ours, {}, precision=precision), pos.cuda(), box.cuda(), pairs,
                    [p.cuda() for p in prm], ms)
    Eo, go, _ = _eval(lambda *a: R.pairwise_energy(ref, *a), pos, box, pairs, prm, ms)
    tol_e, tol_g = (1e-11, 1e-9) if precision == "fp64" else (2e-5, 2e-4)
    assert abs(E.item() - Eo.item()) <= tol_e * abs(Eo.item()), (E.item(), Eo.item())
    names = ["positions", "box"] + [f"param{k}" for k in range(len(prm))]
    for nm, a, b in zip(names, g, go):
        a = a.detach().cpu()
        assert (a - b).abs().max() <= tol_g * b.abs().max(), (nm, (a - b).abs().max().item(), b.abs().max().item())


@pytest.mark.parametrize("name", ["tt_qq_c6", "slater_disp"])
def test_second_derivatives_match_oracle(name):
    """d/d(theta) of (F . c): double backward through the engine (central differences of its
    analytic first derivatives) against the oracle's double autograd."""
    s, pairs = _system(seed=8)
    ours, ref, _ = KERNELS[name]
    prm = _params(name, s["n_atoms"], seed=5)
    ms = torch.tensor(MS, dtype=torch.float64)
    pos = torch.tensor(s["pos"], dtype=torch.float64)
    box = torch.tensor(s["box"], dtype=torch.float64)
    c = torch.tensor(np.random.default_rng(2).normal(size=s["pos"].shape))
    _, g, (p_, b_, pr_) = _eval(generate_pairwise_interaction(ours, {}, precision="fp64"), pos.cuda(), box.cuda(),
                                pairs, [p.cuda() for p in prm], ms, create_graph=True)
    h = torch.autograd.grad((g[0] * c.cuda()).sum(), [p_] + pr_)
    _, go, (po, bo, pro) = _eval(lambda *a: R.pairwise_energy(ref, *a), pos, box, pairs, prm, ms, create_graph=True)
    ho = torch.autograd.grad((go[0] * c).sum(), [po] + pro)
    for a, b in zip(h, ho):
        a = a.detach().cpu()
        assert (a - b).abs().max() <= 1e-5 * b.abs().max(), ((a - b).abs().max().item(), b.abs().max().item())


def test_row_conventions_and_empty_pairs():
    """Rows with i > j and padding rows (index n) add nothing; the third column picks mScales;
    an empty pair set gives zero energy and zero gradients."""
    s, pairs = _system()
    n = s["n_atoms"]
    prm = [p.cuda() for p in _params("slater_sr", n)]
    fn = generate_pairwise_interaction(slater_sr_kernel, {}, precision="fp64")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    box = torch.tensor(s["box"], dtype=torch.float64, device="cuda")
    ms = torch.tensor(MS, dtype=torch.float64)
    real = pairs[pairs[:, 0] < n]
    E_ref = fn(pos, box, real, ms, *prm).item()
    flipped = np.concatenate([real, real[:, [1, 0, 2]], np.full((7, 3), n)])
    assert abs(fn(pos, box, flipped, ms, *prm).item() - E_ref) <= 1e-12 * abs(E_ref)
    # the non-bonded rows (nbond 0: the last scale, 1.0) re-labelled nbond 3 (scale 0.5) halve their sum
    far = real[real[:, 2] == 0]
    E_far = fn(pos, box, far, ms, *prm).item()
    half = far.copy()
    half[:, 2] = 3
    assert abs(fn(pos, box, half, ms, *prm).item() - 0.5 * E_far) <= 1e-12 * abs(E_far)
    p0 = pos.clone().requires_grad_(True)
    E0 = fn(p0, box, np.zeros((0, 3), dtype=np.int64), ms, *prm)
    assert E0.item() == 0.0
    (g0,) = torch.autograd.grad(E0, [p0])
    assert float(g0.abs().max()) == 0.0


def test_engine_neighbour_list_matches_given_rows():
    """PairwiseEngine with its own cell list (covalent rows for nbond) against the given rows."""
    from dmff_b200 import _lib as L
    from dmff_b200.engine import PairwiseEngine
    s, pairs = _system()
    n = s["n_atoms"]
    prm = torch.stack(_params("tt_qq_c6", n))
    eng = PairwiseEngine(n, L.DMFFB_SR_TT_QQ_C6, rc=5.0, cov_rows=s["cov_rows"], mscales=MS, precision="fp64")
    eng.set_params(prm)
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    r_list, F_list = eng.compute(pos, s["box"], pairs=torch.tensor(pairs[:, :3], dtype=torch.int32, device="cuda"))
    E_list, F_list = r_list.energy, F_list.clone()
    eng.rebuild_internal_pairs(pos, s["box"])
    r_int, F_int = eng.compute(pos, s["box"])
    assert abs(r_int.energy - E_list) <= 1e-12 * abs(E_list)
    assert (F_int - F_list).abs().max().item() <= 1e-10 * F_list.abs().max().item()


def _peg_case():
    from dmff_b200 import Hamiltonian, NeighborList, PDBFile
    gold = json.load(open(os.path.join(HERE, "golden", "energies.json")))["peg2_slater"]
    pdb = PDBFile(os.path.join(DATA, gold["pdb"]))
    H = Hamiltonian(os.path.join(DATA, gold["xml"]))
    # FP64 and the reference's own dipole iteration (fixed-point steps to POL_CONV), as the values were made
    pots = H.createPotential(pdb.topology, nonbondedCutoff=gold["rc_nm"], nonbondedMethod="CutoffPeriodic",
                             ethresh=gold["ethresh"], precision="fp64", pol_solver="reference")
    cov = pdb.topology.buildCovMat()
    pos = np.asarray(pdb.positions, dtype=np.float64)
    box = np.asarray(pdb.topology.getPeriodicBoxVectors(), dtype=np.float64)
    nbl = NeighborList(box, gold["rc_nm"], cov)
    nbl.allocate(pos)
    pairs = nbl.pairs
    pairs = pairs.cpu().numpy() if torch.is_tensor(pairs) else np.asarray(pairs)
    pairs = pairs[pairs[:, 0] < pairs[:, 1]]
    return gold, H, pots, pos, box, pairs


def test_peg_dimer_short_range_goldens():
    """tests/test_admp/test_slater.py: the nine potentials of peg.xml on the PEG dimer (rc 1.49 nm),
    each to four decimals of the reference's value."""
    gold, H, pots, pos, box, pairs = _peg_case()
    dev = torch.device("cuda")
    for name, want in zip(gold["forces"], gold["values"]):
        pot = pots.dmff_potentials[name]
        E = pot(torch.tensor(pos, device=dev), torch.tensor(box, device=dev), pairs, H.paramset)
        np.testing.assert_almost_equal(float(E), want, decimal=gold["decimal"], err_msg=name)
