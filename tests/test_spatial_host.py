"""Local frames, pair frames and global multipoles on the host (``dmff_b200.admp.spatial``,
``ADMPPmeForce.Q_local_to_global``) against the oracle's restatement of dmff/admp/spatial.py
and pme.py:183-196, over all six axis rules."""
import numpy as np
import torch

import oracle.admp_ref as R
from dmff_b200.admp.pme import ADMPPmeForce
from dmff_b200.admp.spatial import build_quasi_internal, generate_construct_local_frames, pbc_shift


def _sites(seed, n=120):
    """Random sites in a sheared box (some far outside it), each with an axis rule and distinct
    z / x / y atoms; indices a rule does not use are -1."""
    rng = np.random.default_rng(seed)
    box = np.array([[14.0, 0, 0], [2.0, 13.0, 0], [-1.5, 1.0, 15.0]])
    pos = rng.uniform(0, 1, (n, 3)) @ box + rng.integers(-2, 3, (n, 3)) @ box
    types = np.arange(n) % 6
    ind = np.full((n, 3), -1)
    for i in range(n):
        others = rng.choice(np.delete(np.arange(n), i), 3, replace=False)
        t = types[i]
        if t != 5:
            ind[i, 0] = others[0]
        if t in (0, 1, 2, 3):
            ind[i, 1] = others[1]
        if t in (2, 3):
            ind[i, 2] = others[2]
    return pos, box, types, ind


def test_local_frames_all_axis_rules_match_oracle():
    for seed in range(3):
        pos, box, types, ind = _sites(seed)
        got = generate_construct_local_frames(types, ind)(torch.tensor(pos), torch.tensor(box))
        want = R.construct_local_frames(pos, box, types, ind)
        assert (got - want).abs().max() < 1e-13
        eye = torch.eye(3, dtype=torch.float64)
        assert (got @ got.transpose(1, 2) - eye).abs().max() < 1e-13  # orthonormal rows
        assert (torch.linalg.det(got) - 1).abs().max() < 1e-13  # right-handed


def test_pbc_shift_and_pair_frames_match_oracle():
    pos, box, _, _ = _sites(5)
    b = torch.tensor(box)
    d = torch.tensor(pos[1:] - pos[:-1])
    assert (pbc_shift(d, b, torch.linalg.inv(b)) - R.pbc_shift(d, b, torch.linalg.inv(b))).abs().max() < 1e-12
    r1, r2 = torch.tensor(pos[:-1]), torch.tensor(pos[1:])
    r2[:5, 1:] = r1[:5, 1:]  # pairs along x: the frame seeds x from e_y
    dr = r1 - r2
    nd = torch.linalg.norm(dr, dim=1)
    assert (build_quasi_internal(r1, r2, dr, nd) - R.build_quasi_internal(r1, r2, dr, nd)).abs().max() < 1e-14


def test_global_multipoles_match_oracle():
    pos, box, types, ind = _sites(9, n=60)
    n_types = 7
    mt = np.random.default_rng(1).integers(0, n_types, len(pos))
    Q_local = torch.tensor(np.random.default_rng(2).standard_normal((n_types, 9)))
    for lmax in (0, 1, 2):
        f = ADMPPmeForce(box, mt, types, ind, 6.0, 5e-4, lmax)
        got = f.Q_local_to_global(torch.tensor(pos), torch.tensor(box), Q_local)
        Qm = Q_local[torch.as_tensor(mt)][:, : (lmax + 1) ** 2]
        if lmax > 0:
            Qm = R.rot_local2global(Qm, R.construct_local_frames(pos, box, types, ind), lmax)
        want = R.convert_harm2cart(Qm, lmax)
        assert got.shape == (len(pos), [1, 4, 10][lmax])
        assert (got - want).abs().max() < 1e-10
    assert f.construct_local_frames is not None


def test_esp_helpers_match_oracle():
    """ADMPPmeForce.generate_esp (pme.py:236-293) and CoulNoCutoffForce.generate_esp
    (inter.py:176-201) on grid points around a small water cluster."""
    from dmff_b200.classical.inter import CoulNoCutoffForce
    from dmff_b200.synthetic import water_box
    s = water_box(8, 6.4, seed=2, lmax=2, pol=True, rc=3.0)
    pos = np.asarray(s["pos"]) / 10.0  # nm, as the reference's ESP fits use
    n = len(pos)
    grids = np.random.default_rng(4).uniform(-0.3, 0.95, (5000, 3))  # > one 4096-point chunk
    mt = np.arange(n)
    Q = torch.tensor(np.asarray(s["Q_local"], dtype=np.float64))
    U = torch.tensor(np.random.default_rng(5).normal(0, 0.01, (n, 3)))
    f = ADMPPmeForce(np.eye(3) * 30, mt, s["axis_types"], s["axis_indices"], 6.0, 5e-4, 2, lpol=True)
    got = f.generate_esp()(torch.tensor(pos), torch.tensor(grids), Q, U)
    big = np.eye(3) * 1000.0
    Qg = R.convert_harm2cart(R.rot_local2global(Q, R.construct_local_frames(pos, big, s["axis_types"],
                                                                            s["axis_indices"]), 2), 2)
    want = R.admp_esp(pos, grids, Qg, U)
    assert got.shape == (5000,)
    assert (got - want).abs().max() <= 1e-10 * want.abs().max()
    f0 = ADMPPmeForce(np.eye(3) * 30, mt, s["axis_types"], s["axis_indices"], 6.0, 5e-4, 2)
    got0 = f0.generate_esp()(torch.tensor(pos), torch.tensor(grids), Q)
    assert (got0 - R.admp_esp(pos, grids, Qg, torch.zeros((n, 3)))).abs().max() <= 1e-10 * want.abs().max()
    q = np.asarray(s["Q_local"])[:, 0]
    top = np.random.default_rng(6).integers(-1, 2, (n, 2)).astype(float)
    nc = CoulNoCutoffForce(q, topology_matrix=top)
    bcc = torch.tensor([0.02, -0.01], dtype=torch.float64)
    got = nc.generate_esp()(torch.tensor(pos), torch.tensor(grids), bcc)
    want = R.coul_nocutoff_esp(pos, grids, torch.tensor(q) + torch.tensor(top) @ bcc)
    assert (got - want).abs().max() <= 1e-12 * want.abs().max()


def test_esp_equals_probe_interaction_energy():
    """The reference's ESP consistency check (tests/test_admp/test_esp.py): E(water + Na+) -
    E(water), both from the float64 oracle without periodic images, equals q_Na times the ESP of
    the water's multipoles at the ion (admp_charge.xml).  The reference asserts 1e-3 relative;
    the two agree to ~1e-14 here, so the bound is 1e-10."""
    import os

    from dmff_b200 import Hamiltonian, PDBFile
    from test_oracle_golden import oracle_from_xml
    data = os.path.join(os.path.dirname(__file__), "golden", "data")
    xml = os.path.join(data, "admp_charge.xml")
    water, probe = PDBFile(os.path.join(data, "water.pdb")), PDBFile(os.path.join(data, "water_ion.pdb"))
    box = np.eye(3) * 100.0
    E_w, _, _ = oracle_from_xml(xml, water.topology, np.asarray(water.positions), box, 10.0, "NoCutoff", 1)
    E_p, _, _ = oracle_from_xml(xml, probe.topology, np.asarray(probe.positions), box, 10.0, "NoCutoff", 1)
    H = Hamiltonian(xml)
    H.createPotential(water.topology, nonbondedMethod="NoCutoff", nonbondedCutoff=10.0, ethresh=5e-4, step_pol=1)
    esp = H.generators["ADMPPmeForce"].pme_force.generate_esp()
    ion = np.asarray(probe.positions)[3:4]
    v = esp(torch.tensor(np.asarray(water.positions)), torch.tensor(ion), H.paramset["ADMPPmeForce"]["Q_local"])
    np.testing.assert_allclose(E_p - E_w, v[0].item() * 1.0, rtol=1e-10)
