"""Host-side logic: XML / topology / generator set-up, the C-ABI library symbols, builders."""
import ctypes
import os
import re
import subprocess

import numpy as np
import torch
import pytest

from dmff_b200 import Hamiltonian, PDBFile
from dmff_b200 import _lib
from dmff_b200.synthetic import water_box, workload, pairs_nbond

HERE = os.path.dirname(__file__)
ROOT = os.path.dirname(HERE)
DATA = os.path.join(HERE, "golden", "data")


def test_header_symbols_exported_by_library():
    """every function include/dmffb200.h declares is exported by libdmffb200.so (no GPU calls)."""
    header = open(os.path.join(ROOT, "include", "dmffb200.h")).read()
    declared = set(re.findall(r"\b(dmffb_\w+)\s*\(", header))
    assert declared, "no declarations found"
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared == set(_lib.EXPORTED)


def test_ctypes_struct_layout_matches_header():
    """every ctypes mirror of a header struct has the C layout: size and the offset of each field,
    printed by a tiny C program compiled here against include/dmffb200.h."""
    lines = []
    for cname, cls in _lib.STRUCTS.items():
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"dmffb200.h\"\nint main(void) {\n" + \
          "\n".join(lines) + "\n  return 0; }\n"
    tmp = os.path.join(os.environ.get("TMPDIR", "/tmp"), "dmffb_layout")
    with open(tmp + ".c", "w") as f:
        f.write(src)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), tmp + ".c", "-o", tmp], check=True)
    vals = [int(x) for x in subprocess.run([tmp], capture_output=True, text=True, check=True).stdout.split()]
    want = []
    for cls in _lib.STRUCTS.values():
        want.append(ctypes.sizeof(cls))
        want += [getattr(cls, fname).offset for fname, _ in cls._fields_]
    assert vals == want


def test_generator_parses_reference_xml_like_reference():
    H = Hamiltonian(os.path.join(DATA, "admp.xml"))
    pdb = PDBFile(os.path.join(DATA, "water_dimer.pdb"))
    pot = H.createPotential(pdb.topology, nonbondedMethod="CutoffPeriodic", nonbondedCutoff=0.4, ethresh=5e-4,
                            step_pol=5)
    g = H.generators["ADMPPmeForce"]
    pf = g.pme_force
    # axis types / indices of tests/test_admp/test_sptial.py:71-142
    assert pf.axis_type.tolist() == [1, 0, 0, 1, 0, 0]
    assert pf.axis_indices.tolist() == [[1, 2, -1], [0, 2, -1], [0, 1, -1], [4, 5, -1], [3, 5, -1], [3, 4, -1]]
    Q = H.paramset["ADMPPmeForce"]["Q_local"].numpy()
    np.testing.assert_allclose(Q[0], [-1.0614, -0.23671684, 0, 0, -0.0714102, 0, 0, 0.01106659, 0], rtol=1e-6)
    np.testing.assert_allclose(H.paramset["ADMPPmeForce"]["pol"].numpy(), [0.88, 0.0])
    assert g.mScales == [0.0, 0.0, 0.0, 1.0, 1.0, 1.0]
    assert pf.kappa == 0.0 and pf.lpme is False
    assert pot.meta["cov_map"][0, 1] == 1 and pot.meta["cov_map"][1, 2] == 2 and pot.meta["cov_map"][0, 3] == 0
    assert "ADMPPmeForce" in pot.dmff_potentials


def test_pme_parameters_follow_reference_formula():
    from dmff_b200.admp.pme import setup_ewald_parameters
    kappa, K1, K2, K3 = setup_ewald_parameters(6.0, 5e-4, np.eye(3) * 18.6)
    assert abs(kappa - 0.43804) < 1e-5 and (K1, K2, K3) == (25, 25, 25)
    kappa, K1, _, _ = setup_ewald_parameters(8.0, 5e-4, np.eye(3) * 49.7)
    assert abs(kappa - 0.32853) < 1e-5 and K1 == 50


def test_covalent_map_matches_dense_reference_semantics():
    from dmff_b200.api.topology import covalent_rows, CovalentMap
    # a 7-atom chain with a branch: shortest paths up to 6 bonds
    bonds = [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (2, 6)]
    cm = CovalentMap(7, covalent_rows(7, bonds))
    d = cm.dense()
    assert d[0, 1] == 1 and d[0, 2] == 2 and d[0, 6] == 3 and d[3, 6] == 2 and d[0, 4] == 4
    assert (d == d.T).all() and (np.diag(d) == 0).all()


def test_water_builder_properties():
    s = water_box(216, 18.6, seed=0)
    assert s["pos"].shape == (648, 3)
    import oracle.admp_ref as R
    pr = R.brute_force_pairs(s["pos"], s["box"], 1.7)
    mol = np.arange(648) // 3
    assert (mol[pr[:, 0]] == mol[pr[:, 1]]).all()  # no intermolecular contact below 1.7 A
    oh = np.linalg.norm(s["pos"][1::3] - s["pos"][0::3], axis=1)
    np.testing.assert_allclose(oh, 0.9572, atol=1e-12)
    assert workload("c1")["K"] == (50, 50, 50)


def test_pairs_nbond_lookup():
    s = water_box(8, 6.2, seed=3)
    pr = np.array([[0, 1, 0], [1, 2, 0], [0, 3, 0], [3, 5, 0]])
    np.testing.assert_array_equal(pairs_nbond(pr, s["cov_rows"], s["n_atoms"]), [1, 2, 0, 1])


def test_build_covalent_map_matches_reference_loop():
    """build_covalent_map (hamiltonian.py:17-35) on chains, rings and branches, against the
    oracle's step-for-step restatement of the reference's loop."""
    from types import SimpleNamespace

    import oracle.admp_ref as R
    from dmff_b200.api.hamiltonian import build_covalent_map
    rng = np.random.default_rng(3)
    graphs = [
        [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 0)],            # six-ring
        [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 6), (6, 7)],    # chain longer than the map
        [(0, 1), (0, 2), (0, 3), (3, 4), (4, 5), (4, 6), (6, 7), (7, 3)],  # branch + four-ring
    ]
    tree = [(k, int(rng.integers(0, k))) for k in range(1, 14)]
    graphs.append(tree + [(2, 9), (5, 12)])  # random tree with two extra ring bonds
    for bonds in graphs:
        n = max(max(b) for b in bonds) + 2  # one isolated atom
        data = SimpleNamespace(atoms=list(range(n)), bonds=[SimpleNamespace(atom1=a, atom2=b) for a, b in bonds])
        for mx in (1, 3, 6):
            got = build_covalent_map(data, mx)
            want = R.build_covalent_map(n, bonds, mx)
            assert np.array_equal(got, want), (bonds, mx)


def test_utils_pair_helpers_match_oracle():
    import oracle.admp_ref as R
    from dmff_b200 import utils as U
    rng = np.random.default_rng(8)
    p = rng.integers(0, 50, (200, 2))
    p[:20] = 50  # (N, N) padding rows
    assert np.array_equal(U.regularize_pairs(p).numpy(), R.regularize_pairs(p).numpy())
    assert np.array_equal(U.pair_buffer_scales(p).numpy(), R.pair_buffer_scales(p).numpy().astype(int))
    assert U.convertStr2Float("1.5") == 1.5 and U.convertStr2Float("OW") == "OW"
    assert U.findItemInList("b", ["a", "b"]) == 1 and U.findItemInList("c", ["a"]) == -1
    d = U.dict_to_jnp({"A": {"k": [1, 2]}, "x": 3.0})
    assert d["A"]["k"].dtype == torch.float64 and float(d["x"]) == 3.0
    assert U.jit_condition(static_argnums=(1,))(len) is len


# every import a caller of the reference's energy/force path makes, as (module, names)
DROP_IN_IMPORTS = [
    ("", ["Hamiltonian", "NeighborList", "NeighborListFreud"]),
    ("api", ["Hamiltonian", "DMFFTopology"]),
    ("api.hamiltonian", ["Hamiltonian", "Potential", "build_covalent_map"]),
    ("admp.pme", ["ADMPPmeForce", "setup_ewald_parameters", "DIELECTRIC"]),
    ("admp.disp_pme", ["ADMPDispPmeForce"]),
    ("admp.settings", ["POL_CONV", "MAX_N_POL"]),
    ("admp.pairwise", ["generate_pairwise_interaction", "TT_damping_qq_c6_kernel", "TT_damping_qq_kernel",
                       "distribute_scalar", "distribute_v3", "distribute_matrix"]),
    ("admp.spatial", ["pbc_shift", "v_pbc_shift", "normalize", "generate_construct_local_frames",
                      "build_quasi_internal"]),
    ("admp.multipole", ["convert_cart2harm", "convert_harm2cart", "rot_global2local", "rot_local2global",
                        "rot_ind_global2local", "C1_h2c", "C2_h2c"]),
    ("classical.inter", ["LennardJonesForce", "LennardJonesLongRangeForce", "CoulNoCutoffForce",
                         "CoulReactionFieldForce", "CoulombPMEForce"]),
    ("classical.intra", ["HarmonicBondJaxForce", "HarmonicAngleJaxForce", "PeriodicTorsionJaxForce"]),
    ("common.nblist", ["NeighborList", "NeighborListFreud", "NoCutoffNeighborList", "NoPeriodicNeighborList"]),
    ("generators", ["ADMPPmeGenerator", "ADMPDispPmeGenerator", "ADMPDispGenerator", "NonbondedGenerator",
                    "CoulombGenerator", "LennardJonesGenerator", "HarmonicBondGenerator", "HarmonicAngleGenerator",
                    "PeriodicTorsionGenerator"]),
    ("utils", ["regularize_pairs", "pair_buffer_scales", "DMFFException"]),
]


@pytest.mark.parametrize("mod,names", DROP_IN_IMPORTS, ids=[m or "dmff" for m, _ in DROP_IN_IMPORTS])
def test_drop_in_import_surface(mod, names):
    import importlib
    m = importlib.import_module("dmff_b200" + ("." + mod if mod else ""))
    for n in names:
        assert getattr(m, n, None) is not None, f"dmff.{mod}.{n}"


@pytest.mark.parametrize("files,n_types,residues,n_bond,n_nb", [
    (["xmlio_test1.xml"], 4, [(4, 3, 2)], 3, 4),
    (["xmlio_test1.xml", "xmlio_test2.xml"], 8, [(4, 3, 2), (5, 4, 2)], 6, 8),
])
def test_xml_reader_counts_like_reference(files, n_types, residues, n_bond, n_nb):
    """tests/test_frontend/test_xmlio.py:7-57: one file, and two files merged, read into atom
    types, residue templates (particles, bonds, externals) and force nodes with their attributes."""
    from dmff_b200.api.xmlio import XMLIO
    io = XMLIO()
    for f in files:
        io.loadXML(os.path.join(DATA, f))
    ret = io.parseXML()
    assert len(ret["AtomTypes"]) == n_types
    assert [(len(r["particles"]), len(r["bonds"]), len(r["externals"])) for r in ret["Residues"]] == residues
    assert len(ret["Forces"]) == 2
    assert len(ret["Forces"]["HarmonicBondForce"]["node"]) == n_bond
    assert {"k", "length", "type1", "type2"} <= set(ret["Forces"]["HarmonicBondForce"]["node"][0]["attrib"])
    assert len(ret["Forces"]["NonbondedForce"]["node"]) == n_nb
    assert {"charge", "epsilon", "sigma", "type"} <= set(ret["Forces"]["NonbondedForce"]["node"][0]["attrib"])
