"""Regenerate the golden fixtures in tests/golden/ from the reference checkout.

Run from the repository root with the path of a reference checkout (the argument, or the
environment variable DMFF_REFERENCE):

    python tests/golden/make_golden.py <path to deepmodeling/DMFF>

It copies the reference's small force-field XML / PDB inputs, converts the 996-water box
to a compact .npz, extracts the reference's golden energies (test files and example
``ref_out`` files), and pulls the numeric known-answer arrays out of the reference's
pytest parametrisations with ``ast`` (no reference code is imported or executed).
The pickled MPID dipoles are read with an unpickler that only admits numpy's array
reconstruction globals.
"""
import ast
import io
import json
import os
import pickle
import re
import shutil
import sys

import numpy as np

REF = None  # the reference checkout, set by main() from argv or DMFF_REFERENCE
HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data")


def _arr_literal(node):
    """Turn jnp.array(X) / np.array(X, dtype=...) calls into their literal first argument."""

    class Strip(ast.NodeTransformer):
        def visit_Call(self, n):
            self.generic_visit(n)
            f = n.func
            name = f.attr if isinstance(f, ast.Attribute) else getattr(f, "id", "")
            if name == "array" and n.args:
                return n.args[0]
            return n

    return ast.literal_eval(Strip().visit(node))


def parametrize_cases(path):
    """{test_name: [case tuples]} for every @pytest.mark.parametrize in a test file."""
    tree = ast.parse(open(path).read())
    out = {}
    for fn in ast.walk(tree):
        if not isinstance(fn, ast.FunctionDef):
            continue
        for dec in fn.decorator_list:
            if isinstance(dec, ast.Call) and getattr(dec.func, "attr", "") == "parametrize":
                names = [s.strip() for s in ast.literal_eval(dec.args[0]).split(",")]
                cases = []
                for elt in dec.args[1].elts:
                    vals = [_arr_literal(v) for v in elt.elts]
                    cases.append(dict(zip(names, vals)))
                out[fn.name] = cases
    return out


class _NumpyOnly(pickle.Unpickler):
    ALLOWED = {("numpy.core.multiarray", "_reconstruct"), ("numpy._core.multiarray", "_reconstruct"),
               ("numpy", "ndarray"), ("numpy", "dtype")}

    def find_class(self, module, name):
        if (module, name) in self.ALLOWED:
            if module.startswith("numpy.core"):
                module = "numpy._core.multiarray"
            return super().find_class(module, name)
        raise pickle.UnpicklingError(f"blocked global {module}.{name}")


def read_pdb_positions(path):
    pos, names, resnames, resids = [], [], [], []
    box = None
    for line in open(path):
        if line.startswith("CRYST1"):
            box = [float(line[6:15]), float(line[15:24]), float(line[24:33])]
        if line.startswith(("ATOM", "HETATM")):
            names.append(line[12:16].strip())
            resnames.append(line[17:20].strip())
            resids.append(int(line[22:26]))
            pos.append([float(line[30:38]), float(line[38:46]), float(line[46:54])])
    return np.array(pos), np.array(box), names, resnames, resids


def main():
    global REF
    REF = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DMFF_REFERENCE")
    if not REF or not os.path.isdir(REF):
        sys.exit("usage: python tests/golden/make_golden.py <path to a deepmodeling/DMFF checkout> "
                 "(or set DMFF_REFERENCE)")
    os.makedirs(DATA, exist_ok=True)
    wf = f"{REF}/examples/water_fullpol"
    copies = {
        f"{REF}/tests/data/water_dimer.pdb": "water_dimer.pdb",
        f"{REF}/tests/data/admp.xml": "admp.xml",
        f"{REF}/tests/data/admp_mono.xml": "admp_mono.xml",
        f"{REF}/tests/data/admp_nonpol.xml": "admp_nonpol.xml",
        # ESP consistency inputs (tests/test_admp/test_esp.py)
        f"{REF}/tests/data/admp_charge.xml": "admp_charge.xml",
        f"{REF}/tests/data/water.pdb": "water.pdb",
        f"{REF}/tests/data/water_ion.pdb": "water_ion.pdb",
        # XML reader inputs (tests/test_frontend/test_xmlio.py)
        f"{REF}/tests/data/test1.xml": "xmlio_test1.xml",
        f"{REF}/tests/data/test2.xml": "xmlio_test2.xml",
        # Slater-ISA / short-range inputs (tests/test_admp/test_slater.py)
        f"{REF}/tests/data/peg.xml": "peg.xml",
        f"{REF}/tests/data/peg2.pdb": "peg2.pdb",
        # charge-equilibration inputs (tests/test_admp/test_qeq.py)
        f"{REF}/tests/data/qeq.xml": "qeq.xml",
        f"{REF}/tests/data/qeq.pdb": "qeq.pdb",
        f"{REF}/tests/data/qeq2.xml": "qeq2.xml",
        f"{REF}/tests/data/qeq2.pdb": "qeq2.pdb",
        f"{wf}/forcefield.xml": "waterbox_forcefield.xml",
        f"{wf}/residues.xml": "waterbox_residues.xml",
        f"{wf}/quadrupole_nonpol/forcefield.xml": "waterbox_quadrupole_nonpol.xml",
        f"{wf}/monopole_polarizable/forcefield.xml": "waterbox_monopole_pol.xml",
    }
    # classical-term inputs (tests/test_classical/*)
    for f in ["bond1.pdb", "bond1.xml", "angle1.pdb", "angle1.xml", "proper1.pdb", "proper1.xml", "proper2.pdb",
              "proper2.xml", "impr1.pdb", "impr1.xml", "wild1.xml", "wild2.xml", "lj2.pdb", "lj2.xml", "lj3.pdb",
              "lj3.xml", "coul2.xml", "coul3.xml", "coul3-res.xml", "methane_water.pdb",
              "methane_water_coul.xml"]:
        copies[f"{REF}/tests/data/{f}"] = f
    for src, dst in copies.items():
        shutil.copy(src, os.path.join(DATA, dst))

    pos, box, names, resnames, resids = read_pdb_positions(f"{wf}/waterbox_31ang.pdb")
    np.savez_compressed(os.path.join(DATA, "waterbox_996.npz"), positions_A=pos, box_A=box,
                        names=np.array(names), resnames=np.array(resnames), resids=np.array(resids))

    # golden energies
    def ref_out_numbers(path):
        return [float(x) for x in re.findall(r"-?\d+\.\d+", open(path).read().split("\n", 5)[0:5].__str__())]

    compute = open(f"{REF}/tests/test_admp/test_compute.py").read()
    dimer = [float(x) for x in re.findall(r"assert_almost_equal\(energy, (-?[\d.]+)", compute)]
    ref_out = open(f"{wf}/ref_out").read().splitlines()
    qnp = open(f"{wf}/quadrupole_nonpol/ref_out").read().splitlines()
    mpol = open(f"{wf}/monopole_polarizable/ref_out").read().splitlines()
    mpid = open(f"{wf}/mpid_ref/results.txt").read().splitlines()
    energies = {
        "dimer_pol_lmax2_steppol5": {"value": dimer[0], "decimal": 1,
                                     "source": "tests/test_admp/test_compute.py:55"},
        "dimer_pol_lmax0_steppol5": {"value": dimer[3], "decimal": 2,
                                     "source": "tests/test_admp/test_compute.py:124"},
        "dimer_nonpol_lmax2": {"value": dimer[4], "decimal": 2,
                               "source": "tests/test_admp/test_compute.py:145"},
        "waterbox996_es_pol": {"value": float(ref_out[1].split()[1]),
                               "source": "examples/water_fullpol/ref_out:2"},
        "waterbox996_disp_damp": {"value": float(ref_out[3].split()[1]),
                                  "source": "examples/water_fullpol/ref_out:4"},
        "waterbox996_quadrupole_nonpol_es": {"value": float(qnp[1].split()[1]),
                                             "source": "examples/water_fullpol/quadrupole_nonpol/ref_out:2"},
        "waterbox996_monopole_pol_es": {"value": float(mpol[1].split()[0]),
                                        "source": "examples/water_fullpol/monopole_polarizable/ref_out:2"},
        "waterbox996_mpid_es_rc8": {"value": float(mpid[1].split()[1]),
                                    "source": "examples/water_fullpol/mpid_ref/results.txt:2"},
    }
    # classical goldens: (pdb, xml, value) parametrisations of the reference's classical tests
    classical = []
    for path, tol in [("tests/test_classical/test_bonded.py", {"decimal": 3}),
                      ("tests/test_classical/test_lj.py", {"decimal": 3}),
                      ("tests/test_classical/test_coul.py", {"decimal": 3})]:
        for test, cases in parametrize_cases(f"{REF}/{path}").items():
            for c in cases:
                entry = {"test": test, "pdb": os.path.basename(c["pdb"]), "xml": os.path.basename(c["prm"]),
                         "value": float(c["value"]), "source": path}
                entry.update({"atol": 1e-2} if test == "test_coul_pme" else tol)
                classical.append(entry)
    energies["classical"] = classical
    # the nine PEG dimer energies of the short-range test, in the order its potentials are called
    slater = parametrize_cases(f"{REF}/tests/test_admp/test_slater.py")["test_admp_slater"][0]
    energies["peg2_slater"] = {
        "pdb": os.path.basename(slater["pdb"]), "xml": os.path.basename(slater["prm"]), "rc_nm": 1.49,
        "ethresh": 1e-4, "decimal": 4, "source": "tests/test_admp/test_slater.py:17-27",
        "forces": ["ADMPPmeForce", "ADMPDispPmeForce", "SlaterExForce", "SlaterSrEsForce", "SlaterSrPolForce",
                   "SlaterSrDispForce", "SlaterDhfForce", "QqTtDampingForce", "SlaterDampingForce"],
        "values": [float(v) for v in slater["values"]]}
    # the two charge-equilibration energies of tests/test_admp/test_qeq.py
    qeq_src = open(f"{REF}/tests/test_admp/test_qeq.py").read()
    qm = re.findall(r"assert_almost_equal\(energy, (-?[\d.]+), decimal=(\d)", qeq_src)
    qv = [float(v) for v, _ in qm]
    qd = [int(d) for _, d in qm]
    energies["qeq"] = {"xml": "qeq.xml", "pdb": "qeq.pdb", "rc_nm": 0.6, "ethresh": 1e-3, "value": qv[0],
                       "decimal": qd[0], "source": "tests/test_admp/test_qeq.py:12-40"}
    energies["qeq2"] = {"xml": "qeq2.xml", "pdb": "qeq2.pdb", "rc_nm": 0.6, "ethresh": 1e-3, "value": qv[1],
                        "decimal": qd[1], "source": "tests/test_admp/test_qeq.py:43-89",
                        "groups": [[0, 144], [144, 147]], "group_vals": [0.0, 0.0], "lagmt0": [1.0, 1.0]}
    with open(os.path.join(HERE, "energies.json"), "w") as f:
        json.dump(energies, f, indent=1)

    # induced dipoles: ref_out lines 5.. hold (MPID, MPID, DMFF) per component, in nm*e
    dip = np.array([[float(v) for v in l.split()] for l in ref_out[4:] if l.strip()])
    with open(f"{wf}/mpid_dip.pickle", "rb") as f:
        mpid_dip = np.asarray(_NumpyOnly(f).load(), dtype=np.float64)
    np.savez_compressed(os.path.join(DATA, "waterbox_996_dipoles.npz"), ref_out_cols=dip,
                        mpid_dip=mpid_dip)

    # known-answer arrays from the reference's parametrised tests
    kats = {}
    for name, path in [("multipole", "tests/test_admp/test_multipole.py"),
                       ("spatial", "tests/test_admp/test_sptial.py"),
                       ("noaxistype", "tests/test_admp/test_noaxistype.py")]:
        cases = parametrize_cases(f"{REF}/{path}")
        kats[name] = {"source": path, "cases": cases}
    kats["utils"] = {"source": "tests/test_utils.py:8-32",
                     "pairs": [[0, 0], [1, 0], [0, 1], [1, 1]],
                     "regularized": [[-1, -2], [0, -2], [0, 1], [0, -1]],
                     "buffer_scales": [0, 0, 1, 0]}
    kats["nblist"] = {"source": "tests/test_common/test_nblist.py:61-68,108-117",
                      "dimer_rc_A": 4.0, "npairs": 15, "capacity": int(15 * 1.3)}
    with open(os.path.join(HERE, "kats.json"), "w") as f:
        json.dump(kats, f)


if __name__ == "__main__":
    main()
