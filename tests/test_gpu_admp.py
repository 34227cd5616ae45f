"""GPU parity: the CUDA engine (through the C ABI) against the float64 oracle."""
import numpy as np
import pytest
import torch

from dmff_b200.synthetic import water_box
from tests.helpers import make_engine, oracle_pairs, oracle_reference, rel_force_rms

pytestmark = pytest.mark.gpu

# tolerances of the FP32 path and of the FP64 instantiation
TOL = {"fp32": dict(e=1e-5, f=1e-4, b=1e-4), "fp64": dict(e=1e-10, f=1e-8, b=1e-8)}


def _run(eng, sysd, pairs):
    dev = torch.device("cuda")
    pos = torch.tensor(sysd["pos"], dtype=torch.float64, device=dev)
    pr = torch.tensor(pairs, dtype=torch.int32, device=dev)
    res, F, U = eng.compute(pos, sysd["box"], pairs=pr)
    return res, F.cpu().numpy(), U.cpu().numpy()


# the float64 oracle's energy of the c0_small fixture, reproduced bit for bit on every host it has
# been run on (any thread count); a host whose CPU arithmetic gives another value cannot check the
# FP64 tolerances below, and says so here instead of failing them
C0_SMALL_ORACLE_E = -398.00509400279407


@pytest.fixture(scope="module")
def c0_small():
    s = water_box(64, 12.4, seed=10, lmax=2, pol=False, rc=6.0)
    pr = oracle_pairs(s)
    ref = oracle_reference(s, pr)
    assert abs(ref["E"] - C0_SMALL_ORACLE_E) <= 1e-12 * abs(C0_SMALL_ORACLE_E), (
        f"the float64 oracle is not reproducible on this host: {ref['E']!r} != {C0_SMALL_ORACLE_E!r}")
    return s, pr, ref


@pytest.fixture(scope="module")
def pol_small():
    s = water_box(64, 12.4, seed=11, lmax=2, pol=True, rc=6.0)
    pr = oracle_pairs(s)
    return s, pr, oracle_reference(s, pr, solver="cg", tol=1e-9)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_nonpol_energy_forces_boxgrad(c0_small, prec):
    s, pr, ref = c0_small
    eng = make_engine(s, precision=prec)
    res, F, _ = _run(eng, s, pr)
    t = TOL[prec]
    assert abs(res.energy - ref["E"]) <= t["e"] * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= t["f"]
    bg = np.array(res.box_grad).reshape(3, 3)
    assert np.abs(bg - ref["box_grad"]).max() <= t["b"] * np.abs(ref["box_grad"]).max()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_pol_energy_forces_dipoles(pol_small, prec):
    s, pr, ref = pol_small
    eng = make_engine(s, precision=prec, cg_tol=1e-6 if prec == "fp32" else 1e-11)
    res, F, U = _run(eng, s, pr)
    t = TOL[prec]
    assert res.converged == 1
    assert abs(res.energy - ref["E"]) <= t["e"] * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= t["f"]
    assert np.abs(U - ref["U"]).max() <= (1e-4 if prec == "fp32" else 1e-8) * np.abs(ref["U"]).max()
    bg = np.array(res.box_grad).reshape(3, 3)
    assert np.abs(bg - ref["box_grad"]).max() <= t["b"] * np.abs(ref["box_grad"]).max()


def test_field_entry_point_matches_oracle_grad_U(pol_small):
    """dmffb_admp_field (dE/dU at a given U, the reference's grad_U_fn, pme.py:181) at positions
    other than the engine's last compute: it builds its own CSR and pair tensors."""
    import oracle.admp_ref as R
    s, pr, _ = pol_small
    eng = make_engine(s, precision="fp64", cg_tol=1e-8)
    pos_a = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.U.zero_()
    eng.compute(pos_a, s["box"], pairs=torch.tensor(pr, dtype=torch.int32, device="cuda"))
    rng = np.random.default_rng(9)
    sb = dict(s, pos=s["pos"] + rng.normal(0.0, 0.05, size=s["pos"].shape))
    prb = oracle_pairs(sb)
    U = rng.normal(0.0, 0.02, size=(s["n_atoms"], 3))
    got = eng.field(torch.tensor(sb["pos"], dtype=torch.float64, device="cuda"), sb["box"],
                    torch.tensor(prb, dtype=torch.int32, device="cuda"),
                    torch.tensor(U, dtype=torch.float64, device="cuda")).cpu().numpy()
    f = R.ADMPPmeForce(sb["box"], sb["axis_types"], sb["axis_indices"], sb["rc"], sb["ethresh"], sb["lmax"],
                       sb["lpol"], kappa=sb["kappa"], K=sb["K"])
    want = f.grad_U(torch.tensor(sb["pos"]), torch.tensor(sb["box"]), prb, torch.tensor(sb["Q_local"]),
                    torch.tensor(U), torch.tensor(sb["pol"]), torch.tensor(sb["thole"]), torch.tensor(sb["mscales"]),
                    torch.tensor(sb["pscales"]), torch.tensor(sb["dscales"])).numpy()
    assert rel_force_rms(got, want) <= 1e-9


def test_zero_guess_matches_explicit_zero(pol_small):
    """dmffb_admp_set_zero_guess: the U buffer's content is ignored and the CG set-up skips its
    A U pass; results equal a solve from an explicitly zeroed U and the oracle."""
    s, pr, ref = pol_small
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    prt = torch.tensor(pr, dtype=torch.int32, device="cuda")
    e1 = make_engine(s, precision="fp64", cg_tol=1e-8)
    e1.U.zero_()
    r1, F1, _ = e1.compute(pos, s["box"], pairs=prt)
    F1 = F1.cpu().numpy().copy()
    e2 = make_engine(s, precision="fp64", cg_tol=1e-8)
    e2.set_zero_guess(True)
    e2.U.fill_(123.0)  # ignored on input
    r2, F2, U2 = e2.compute(pos, s["box"], pairs=prt)
    assert r2.n_iter == r1.n_iter
    assert abs(r2.energy - r1.energy) <= 1e-12 * abs(r1.energy)
    assert rel_force_rms(F2.cpu().numpy(), F1) <= 1e-12
    assert abs(r2.energy - ref["E"]) <= 1e-9 * abs(ref["E"])
    assert bool(torch.isfinite(U2).all())


def test_reference_solver_matches_fixed_step_oracle():
    s = water_box(27, 9.3, seed=12, lmax=2, pol=True, rc=4.5)
    pr = oracle_pairs(s)
    ref = oracle_reference(s, pr, solver="reference", steps_pol=5)
    eng = make_engine(s, precision="fp64", solver="reference", steps_pol=5)
    res, F, U = _run(eng, s, pr)
    assert res.n_iter == 5
    assert abs(res.energy - ref["E"]) <= 1e-9 * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= 1e-8


def test_host_buffer_path_matches_device_path(pol_small):
    s, pr, ref = pol_small
    eng = make_engine(s, precision="fp32", cg_tol=1e-6)
    res_d, F_d, U_d = _run(eng, s, pr)
    res_h, F_h, U_h = eng.compute_host(s["pos"], s["box"], pairs=pr)
    assert abs(res_h.energy - res_d.energy) <= 1e-6 * abs(res_d.energy)
    assert rel_force_rms(F_h, F_d) <= 1e-5


def test_host_buffer_path_into_caller_arrays(pol_small):
    """compute_host writes forces and dipoles into caller-owned (here pinned) arrays."""
    s, pr, _ = pol_small
    eng = make_engine(s, precision="fp32", cg_tol=1e-6)
    res_a, F_a, U_a = eng.compute_host(s["pos"], s["box"], pairs=pr)
    F_out = torch.zeros((s["n_atoms"], 3), dtype=torch.float64).pin_memory().numpy()
    U_out = torch.full((s["n_atoms"], 3), 7.0, dtype=torch.float64).pin_memory().numpy()
    res_b, F_b, U_b = eng.compute_host(s["pos"], s["box"], pairs=pr, forces_out=F_out, U_out=U_out)
    assert F_b is F_out and U_b is U_out
    assert abs(res_b.energy - res_a.energy) <= 1e-6 * abs(res_a.energy)
    assert rel_force_rms(F_b, F_a) <= 1e-5
    assert rel_force_rms(U_b, U_a) <= 1e-5
    with pytest.raises(ValueError):
        eng.compute_host(s["pos"], s["box"], pairs=pr, forces_out=np.zeros((s["n_atoms"], 3), np.float32))


@pytest.mark.parametrize("name,L,n,rc", [("tiny", 9.3, 27, 4.5), ("c0", 18.6, 216, 6.0), ("mid", 31.0, 1000, 8.0)])
def test_neighbor_set_bit_exact(name, L, n, rc):
    import oracle.admp_ref as R
    s = water_box(n, L, seed=20, lmax=2, pol=False, rc=rc)
    pr_o = oracle_pairs(s)
    eng = make_engine(s, precision="fp64")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    rows = eng.build_neighbors(pos, s["box"], rc).cpu().numpy()
    assert rows.shape[0] == pr_o.shape[0]
    assert np.all(rows[:, 0] < rows[:, 1])
    assert np.all(np.diff(rows[:, 0]) >= 0)  # sorted by i
    got = set(map(tuple, rows.tolist()))
    want = set(map(tuple, pr_o.tolist()))
    assert got == want


def test_internal_pairs_equal_given_pairs(c0_small):
    s, pr, ref = c0_small
    eng = make_engine(s, precision="fp64")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    res, F, _ = eng.compute(pos, s["box"])  # engine-built cell list
    assert res.n_pairs == len(pr)
    assert abs(res.energy - ref["E"]) <= 1e-10 * abs(ref["E"])
    assert rel_force_rms(F.cpu().numpy(), ref["F"]) <= 1e-8


@pytest.mark.parametrize("pol", [False, True])
def test_internal_pairs_clustered_box(pol):
    """Every molecule of one octant and about 1/8 of the others (4x the mean density in that
    octant, liquid contacts everywhere): the dense octant's candidate lists exceed the neighbour
    count pass's mask stride and the fill pass repeats the distance tests, while the rest use the
    stored masks.  The engine-built list must give the oracle's pair count and the same FP64
    energy and forces as the oracle's rows fed in."""
    full = water_box(1000, 31.0, seed=21, lmax=2, pol=pol, rc=6.0)
    mol = full["pos"].reshape(-1, 3, 3)
    c = mol[:, 0, :] % 31.0
    rng = np.random.default_rng(5)
    keep = np.all(c < 15.5, axis=1) | (rng.random(len(mol)) < 0.125)
    s = water_box(int(keep.sum()), 31.0, seed=21, lmax=2, pol=pol, rc=6.0)
    s["pos"] = mol[keep].reshape(-1, 3).copy()
    pr = oracle_pairs(s)
    eng = make_engine(s, precision="fp64", cg_tol=1e-8)
    p = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    eng.U.zero_()
    res_i, F_i, _ = eng.compute(p, s["box"])  # engine-built cell list
    E_i, F_i = res_i.energy, F_i.cpu().numpy().copy()
    eng.U.zero_()
    res_g, F_g, _ = eng.compute(p, s["box"], pairs=torch.tensor(pr, dtype=torch.int32, device="cuda"))
    assert res_i.n_pairs == len(pr)
    assert abs(E_i - res_g.energy) <= 1e-9 * abs(res_g.energy)
    assert rel_force_rms(F_i, F_g.cpu().numpy()) <= 1e-8


@pytest.mark.parametrize("xml,key,dec", [("admp.xml", "dimer_pol_lmax2_steppol5", 1),
                                         ("admp_mono.xml", "dimer_pol_lmax0_steppol5", 2),
                                         ("admp_nonpol.xml", "dimer_nonpol_lmax2", 2)])
def test_dropin_api_water_dimer_goldens(xml, key, dec):
    """tests/test_admp/test_compute.py:36-145 through Hamiltonian / NeighborList / potential_fn."""
    import json
    import os
    from dmff_b200 import Hamiltonian, NeighborList, PDBFile
    here = os.path.join(os.path.dirname(__file__), "golden")
    gold = json.load(open(os.path.join(here, "energies.json")))[key]["value"]
    H = Hamiltonian(os.path.join(here, "data", xml))
    pdb = PDBFile(os.path.join(here, "data", "water_dimer.pdb"))
    pot = H.createPotential(pdb.topology, nonbondedMethod="CutoffPeriodic", nonbondedCutoff=0.4, ethresh=5e-4,
                            step_pol=5, precision="fp64")
    box = pdb.topology.getPeriodicBoxVectors()
    nbl = NeighborList(box, 0.4, pot.meta["cov_map"])
    nbl.allocate(pdb.positions)
    assert int((nbl.pairs[:, 0] < nbl.pairs[:, 1]).sum()) == 15
    assert nbl.pairs.shape[0] == int(15 * 1.3)
    efunc = pot.getPotentialFunc(names=["ADMPPmeForce"])
    pos = torch.tensor(pdb.positions, requires_grad=True)
    E = efunc(pos, box, nbl.pairs, H.paramset)
    np.testing.assert_almost_equal(E.item(), gold, decimal=dec)
    (g,) = torch.autograd.grad(E, pos)
    assert torch.isfinite(g).all()


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_pair_row_order_and_padding_do_not_matter(pol_small, prec):
    """the reference accepts rows in any order with padding / invalid rows (utils.py:67-85)."""
    s, pr, ref = pol_small
    rng = np.random.default_rng(0)
    n = s["n_atoms"]
    junk = np.array([[n, n, 0], [5, 5, 0], [7, 3, 1], [n, n, 0]] * 50)
    rows = np.concatenate([pr, junk])[rng.permutation(len(pr) + len(junk))]
    eng = make_engine(s, precision=prec, cg_tol=1e-6 if prec == "fp32" else 1e-11)
    res, F, U = _run(eng, s, rows)
    t = TOL[prec]
    assert abs(res.energy - ref["E"]) <= t["e"] * abs(ref["E"])
    assert rel_force_rms(F, ref["F"]) <= t["f"]


def test_full_size_fp32_matches_fp64():
    """size-independent check at the benchmark size (12288 atoms): the FP32 path against the FP64
    instantiation of the same kernels (which matches the oracle on every small case)."""
    from dmff_b200.synthetic import workload
    s = workload("c1")
    dev = torch.device("cuda")
    pos = torch.tensor(s["pos"], dtype=torch.float64, device=dev)
    out = {}
    for prec in ("fp64", "fp32"):
        eng = make_engine(s, precision=prec, cg_tol=1e-8)
        eng.rebuild_internal_pairs(pos, s["box"])
        res, F, U = eng.compute(pos, s["box"])
        out[prec] = (res.energy, F.cpu().numpy().copy(), U.cpu().numpy().copy(), np.array(res.box_grad[:]),
                     res.n_pairs)
    e64, F64, U64, B64, n64 = out["fp64"]
    e32, F32, U32, B32, n32 = out["fp32"]
    assert n32 == n64 > 1_000_000
    assert abs(e32 - e64) <= 1e-6 * abs(e64)
    assert rel_force_rms(F32, F64) <= 1e-5
    assert np.abs(U32 - U64).max() <= 1e-4 * np.abs(U64).max()
    assert np.abs(B32 - B64).max() <= 1e-4 * np.abs(B64).max()
