"""Classical generators: XML -> ParamSet + potential_fn on the B200 classical engine.

Mirrors dmff/generators/classical.py: ``HarmonicBondGenerator`` (15-217),
``HarmonicAngleGenerator`` (220-445), ``PeriodicTorsionGenerator`` (448-787, proper and improper
torsions with wildcard matching and the amber improper atom ordering), ``NonbondedGenerator``
(790-1023, LJ + Coulomb with PME / reaction field / no cutoff and the optional LJ dispersion
correction), ``CoulombGenerator`` (1026-1188) and ``LennardJonesGenerator`` (1191-1400, with
NBFix pairs).  Same XML attributes, ParamSet names and masks, same term enumeration order
and the same potential_fn(positions_nm, box_nm, pairs, params, aux=None) call; energies in
kJ/mol.  The engine works in Angstrom: sigma and lengths x10, bond k / 100.
"""
import itertools
import math

import numpy as np
import torch

from ..admp.pme import setup_ewald_parameters
from ..api.hamiltonian import _DMFFGenerators, method_name
from ..api.paramset import ParamSet
from ..classical.forces import ClassicalForce

# standard atomic weights (g/mol) for the improper-torsion atom ordering rule (classical.py:645-652)
_MASS = {"H": 1.008, "He": 4.0026, "Li": 6.94, "Be": 9.0122, "B": 10.81, "C": 12.011, "N": 14.007, "O": 15.999,
         "F": 18.998, "Ne": 20.180, "Na": 22.990, "Mg": 24.305, "Al": 26.982, "Si": 28.085, "P": 30.974,
         "S": 32.06, "Cl": 35.45, "Ar": 39.948, "K": 39.098, "Ca": 40.078, "Mn": 54.938, "Fe": 55.845,
         "Co": 58.933, "Ni": 58.693, "Cu": 63.546, "Zn": 65.38, "Se": 78.971, "Br": 79.904, "Kr": 83.798,
         "Rb": 85.468, "Sr": 87.62, "I": 126.90, "Cs": 132.91, "Ba": 137.33}


def _elem(sym):
    s = str(sym).strip()
    return s[:1].upper() + s[1:].lower()


def _mass(sym):
    return _MASS.get(_elem(sym), 0.0)


def _rc_nm(nonbondedCutoff):
    if hasattr(nonbondedCutoff, "value_in_unit"):
        import openmm.unit as unit
        return nonbondedCutoff.value_in_unit(unit.nanometer)
    return float(nonbondedCutoff)


def _has_aux(kwargs):
    return bool(kwargs.get("has_aux", False))


def _mask(attribs):
    return 0.0 if attribs.get("mask", "").upper() == "TRUE" else 1.0


def _t(x):
    return torch.as_tensor(x, dtype=torch.float64)


# ------------------------------------------------------------------------- bonds
class HarmonicBondGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "HarmonicBondForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        self.key_type = None
        keys, ks, lengths, masks = [], [], [], []
        for node in ffinfo["Forces"][self.name]["node"]:
            at = node["attrib"]
            if self.key_type is None:
                if "type1" in at:
                    self.key_type = "type"
                elif "class1" in at:
                    self.key_type = "class"
                else:
                    raise ValueError("Cannot find key type for HarmonicBondForce.")
            keys.append((at[self.key_type + "1"], at[self.key_type + "2"]))
            ks.append(float(at["k"]))
            lengths.append(float(at["length"]))
            masks.append(_mask(at))
        self.bond_keys = keys
        paramset.addParameter(np.array(lengths), "length", field=self.name, mask=np.array(masks))
        paramset.addParameter(np.array(ks), "k", field=self.name, mask=np.array(masks))

    def getName(self):
        return self.name

    def _find_key_index(self, key):
        for i, k in enumerate(self.bond_keys):
            if (k[0] == key[0] and k[1] == key[1]) or (k[0] == key[1] and k[1] == key[0]):
                return i
        return None

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        idx, prm = [], []
        for bond in topdata.bonds():
            a1, a2 = bond.atom1, bond.atom2
            p = self._find_key_index((a1.meta[self.key_type], a2.meta[self.key_type]))
            if p is None:
                continue
            idx.append((a1.index, a2.index))
            prm.append(p)
        idx = np.asarray(idx, dtype=np.int32).reshape(-1, 2)
        pi = torch.as_tensor(np.asarray(prm, dtype=np.int64))
        self.bond_idx, self.bond_prm_idx = idx, pi
        force = ClassicalForce(topdata.getNumAtoms(), precision=kwargs.get("precision", "fp32"))
        self.force = force
        name, has_aux = self.name, _has_aux(kwargs)

        def potential_fn(positions, box, pairs, params, aux=None):
            p = params[name]
            bprm = torch.stack([_t(p["k"])[pi] / 100.0, _t(p["length"])[pi] * 10.0], dim=1)
            E = force.energy(_t(positions) * 10.0, _t(box) * 10.0, None, bond_idx=idx, bond_prm=bprm)
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


# ------------------------------------------------------------------------- angles
class HarmonicAngleGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "HarmonicAngleForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        self.key_type = None
        keys, ks, th, masks = [], [], [], []
        for node in ffinfo["Forces"][self.name]["node"]:
            at = node["attrib"]
            if self.key_type is None:
                if "type1" in at:
                    self.key_type = "type"
                elif "class1" in at:
                    self.key_type = "class"
                else:
                    raise ValueError("Cannot find key type for HarmonicAngleForce.")
            keys.append((at[self.key_type + "1"], at[self.key_type + "2"], at[self.key_type + "3"]))
            ks.append(float(at["k"]))
            th.append(float(at["angle"]))
            masks.append(_mask(at))
        self.angle_keys = keys
        paramset.addParameter(np.array(th), "angle", field=self.name, mask=np.array(masks))
        paramset.addParameter(np.array(ks), "k", field=self.name, mask=np.array(masks))

    def getName(self):
        return self.name

    def _find_key_index(self, key):
        for i, k in enumerate(self.angle_keys):
            if k[0] == key[0] and k[1] == key[1] and k[2] == key[2]:
                return i
            if k[0] == key[2] and k[1] == key[1] and k[2] == key[0]:
                return i
        return None

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        # angle enumeration of classical.py:380-396: centres in first-seen bond order
        acenters = {}
        for bond in topdata.bonds():
            a1, a2 = bond.atom1, bond.atom2
            acenters.setdefault(a1.index, [a1]).append(a2)
            acenters.setdefault(a2.index, [a2]).append(a1)
        angles = []
        for ic in acenters:
            if len(acenters[ic]) < 3:
                continue
            c, links = acenters[ic][0], acenters[ic][1:]
            for ii in range(len(links)):
                for jj in range(ii + 1, len(links)):
                    angles.append((links[ii], c, links[jj]))
        idx, prm = [], []
        kt = self.key_type
        for a1, a2, a3 in angles:
            p = self._find_key_index((a1.meta[kt], a2.meta[kt], a3.meta[kt]))
            if p is None:
                continue
            idx.append((a1.index, a2.index, a3.index))
            prm.append(p)
        idx = np.asarray(idx, dtype=np.int32).reshape(-1, 3)
        pi = torch.as_tensor(np.asarray(prm, dtype=np.int64))
        self.angle_idx, self.angle_prm_idx = idx, pi
        force = ClassicalForce(topdata.getNumAtoms(), precision=kwargs.get("precision", "fp32"))
        self.force = force
        name, has_aux = self.name, _has_aux(kwargs)

        def potential_fn(positions, box, pairs, params, aux=None):
            p = params[name]
            aprm = torch.stack([_t(p["k"])[pi], _t(p["angle"])[pi]], dim=1)
            E = force.energy(_t(positions) * 10.0, _t(box) * 10.0, None, angle_idx=idx, angle_prm=aprm)
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


# ------------------------------------------------------------------------- torsions
class PeriodicTorsionGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "PeriodicTorsionForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        self.key_type = None
        pk, ik = [], []
        pper, pprm, pmap = [], [], {}
        iper, iprm, imap = [], [], {}
        for node in ffinfo["Forces"][self.name]["node"]:
            at = node["attrib"]
            if "type1" in at:
                self.key_type = "type"
            elif "class1" in at:
                self.key_type = "class"
            key = tuple(at[self.key_type + str(q)] for q in range(1, 5))
            if node["name"] == "Proper":
                pk.append(key)
            elif node["name"] == "Improper":
                ik.append(key)
            m = _mask(at)
            for pkey in at.keys():
                if "periodicity" not in pkey:
                    continue
                order = int(pkey.replace("periodicity", ""))
                per = int(at[pkey])
                phase = float(at["phase" + str(order)])
                k = float(at["k" + str(order)])
                if node["name"] == "Proper":
                    pper.append(per)
                    pprm.append((phase, k, m))
                    pmap.setdefault(len(pk) - 1, []).append(len(pper) - 1)
                elif node["name"] == "Improper":
                    iper.append(per)
                    iprm.append((phase, k, m))
                    imap.setdefault(len(ik) - 1, []).append(len(iper) - 1)
        self.proper_keys, self.proper_periods, self.proper_key_to_prms = pk, np.array(pper), pmap
        self.imp_keys, self.imp_periods, self.imp_key_to_prms = ik, np.array(iper), imap
        pm = np.array([x[2] for x in pprm])
        im = np.array([x[2] for x in iprm])
        paramset.addParameter(np.array([x[0] for x in pprm]), "proper_phase", field=self.name, mask=pm)
        paramset.addParameter(np.array([x[1] for x in pprm]), "proper_k", field=self.name, mask=pm)
        paramset.addParameter(np.array([x[0] for x in iprm]), "improper_phase", field=self.name, mask=im)
        paramset.addParameter(np.array([x[1] for x in iprm]), "improper_k", field=self.name, mask=im)

    def getName(self):
        return self.name

    def _find_proper_key_index(self, key):
        wc = []
        for i, k in enumerate(self.proper_keys):
            for kk in (key, key[::-1]):
                if all(k[q] in ("", kk[q]) for q in range(4)):
                    if "" in k:
                        wc.append(i)
                    else:
                        return i
        return wc[0] if wc else None

    def _find_improper_key_index(self, improper):
        kt = self.key_type
        t = [a.meta[kt] for a in improper]
        wild = lambda tp, tps: tps == "" or tp == tps
        matched = None
        for ndef, tordef in enumerate(self.imp_keys):
            has_wc = "" in tordef
            if matched is not None and has_wc:
                continue
            if t[0] in tordef[0]:  # substring test, as in classical.py:642
                for (t2, t3, t4) in itertools.permutations(((t[1], 1), (t[2], 2), (t[3], 3))):
                    if wild(t2[0], tordef[1]) and wild(t3[0], tordef[2]) and wild(t4[0], tordef[3]):
                        a1, a2 = improper[t2[1]].index, improper[t3[1]].index
                        e1, e2 = _elem(improper[t2[1]].element), _elem(improper[t3[1]].element)
                        m1, m2 = _mass(e1), _mass(e2)
                        if e1 == e2 and a1 > a2:
                            a1, a2 = a2, a1
                        elif e1 != "C" and (e2 == "C" or m1 < m2):
                            a1, a2 = a2, a1
                        matched = (a1, a2, improper[0].index, improper[t4[1]].index, ndef)
                        break
        if matched is None:
            return None, None
        return matched[4], matched[:4]

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        has_aux = _has_aux(kwargs)
        if self.key_type is None:
            def potential_fn_zero(positions, box, pairs, params, aux=None):
                z = torch.zeros((1,), dtype=torch.float64)
                return (z, aux) if has_aux else z
            self._jaxPotential = potential_fn_zero
            return potential_fn_zero
        atoms = list(topdata.atoms())
        acenters = {}
        for bond in topdata.bonds():
            i1, i2 = bond.atom1.index, bond.atom2.index
            acenters.setdefault(i1, []).append(i2)
            acenters.setdefault(i2, []).append(i1)
        propers = []
        for bond in topdata.bonds():
            i1, i2 = bond.atom1.index, bond.atom2.index
            for i3 in [i for i in acenters[i1] if i != i2]:
                for i4 in [i for i in acenters[i2] if i != i1]:
                    if i3 != i4:
                        propers.append((atoms[i3], atoms[i1], atoms[i2], atoms[i4]))
        imprs = []
        for i1 in acenters:
            if len(acenters[i1]) < 3:
                continue
            for item in itertools.combinations(acenters[i1], 3):
                imprs.append((atoms[i1], atoms[item[0]], atoms[item[1]], atoms[item[2]]))
        kt = self.key_type
        idx, per, sel_p, sel_i = [], [], [], []
        for pr in propers:
            pidx = self._find_proper_key_index(tuple(a.meta[kt] for a in pr))
            if pidx is None:
                continue
            for q in self.proper_key_to_prms[pidx]:
                idx.append(tuple(a.index for a in pr))
                per.append(self.proper_periods[q])
                sel_p.append(q)
        n_prop = len(idx)
        for im in imprs:
            iidx, order = self._find_improper_key_index(im)
            if iidx is None:
                continue
            for q in self.imp_key_to_prms[iidx]:
                idx.append(tuple(atoms[o].index for o in order))
                per.append(self.imp_periods[q])
                sel_i.append(q)
        idx = np.asarray(idx, dtype=np.int32).reshape(-1, 4)
        per = torch.as_tensor(np.asarray(per, dtype=np.float64))
        sp = torch.as_tensor(np.asarray(sel_p, dtype=np.int64))
        si = torch.as_tensor(np.asarray(sel_i, dtype=np.int64))
        self.torsion_idx, self.torsion_per, self.sel_proper, self.sel_improper = idx, per, sp, si
        force = ClassicalForce(topdata.getNumAtoms(), precision=kwargs.get("precision", "fp32"))
        self.force = force
        self.n_proper, self.n_improper = n_prop, len(idx) - n_prop
        name = self.name

        def potential_fn(positions, box, pairs, params, aux=None):
            p = params[name]
            k = torch.cat([_t(p["proper_k"])[sp], _t(p["improper_k"])[si]]) if len(si) else _t(p["proper_k"])[sp]
            ph = (torch.cat([_t(p["proper_phase"])[sp], _t(p["improper_phase"])[si]]) if len(si)
                  else _t(p["proper_phase"])[sp])
            if idx.shape[0] == 0:
                E = torch.zeros((), dtype=torch.float64)
            else:
                tprm = torch.stack([k, ph, per], dim=1)
                E = force.energy(_t(positions) * 10.0, _t(box) * 10.0, None, torsion_idx=idx, torsion_prm=tprm)
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


# ------------------------------------------------------------------------- nonbonded
def _lb_tables(sigma, epsilon, nbfix=None, sig_fix=None, eps_fix=None):
    """Type-pair tables (inter.py:58-72): eps_ij = sqrt(eps_i eps_j + 1e-32), sigma_ij = (s_i + s_j)/2,
    NBFix rows (t1, t2, k) override both orientations."""
    sig_tt = (sigma[:, None] + sigma[None, :]) * 0.5
    eps_tt = torch.sqrt(epsilon[:, None] * epsilon[None, :] + 1e-32)
    if nbfix is not None and len(nbfix):
        a, b, k = (torch.as_tensor(nbfix[:, c], dtype=torch.int64) for c in range(3))
        sig_tt = sig_tt.index_put((a, b), sig_fix[k]).index_put((b, a), sig_fix[k])
        eps_tt = eps_tt.index_put((a, b), eps_fix[k]).index_put((b, a), eps_fix[k])
    return sig_tt, eps_tt


def _coulomb_setup(method, topdata, r_cut, kwargs, default_ethresh):
    """(mode, kappa 1/nm, K) for the nonbonded method (classical.py:904-922, 1107-1151)."""
    if method == "PME":
        cell = topdata.getPeriodicBoxVectors()
        ethresh = kwargs.get("ethresh", default_ethresh)
        kappa, K1, K2, K3 = setup_ewald_parameters(r_cut, ethresh, cell, kwargs.get("PmeSpacing", 0.1),
                                                   kwargs.get("PmeCoeffMethod", "openmm"))
        return "pme", kappa, (K1, K2, K3)
    if method in ("CutoffPeriodic", "CutoffNonPeriodic"):
        return "rf", 0.0, (0, 0, 0)
    if method == "NoCutoff":
        return "nocutoff", 0.0, (0, 0, 0)
    raise ValueError("Illegal nonbonded method for NonbondedForce")


class NonbondedGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "NonbondedForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        meta = ffinfo["Forces"][self.name]["meta"]
        self.coulomb14scale = float(meta.get("coulomb14scale", 0.8333333333333334))
        self.lj14scale = float(meta.get("lj14scale", 0.5))
        self.key_type = None
        self.type_to_charge = {}
        nodes = ffinfo["Forces"][self.name]["node"]
        self.charge_in_residue = any(nd["name"] == "UseAttributeFromResidue" and nd["attrib"].get("name") == "charge"
                                     for nd in nodes)
        types, sigma, epsilon, masks = [], [], [], []
        for nd in nodes:
            if nd["name"] != "Atom":
                continue
            at = nd["attrib"]
            self.key_type = "type" if "type" in at else ("class" if "class" in at else None)
            types.append(at[self.key_type])
            sigma.append(float(at["sigma"]))
            epsilon.append(float(at["epsilon"]))
            masks.append(_mask(at))
            if not self.charge_in_residue:
                if "charge" not in at:
                    raise ValueError("No charge information found in NonbondedForce or Residues.")
                self.type_to_charge[at[self.key_type]] = float(at["charge"])
        self.atom_keys = types
        paramset.addParameter(np.array(sigma), "sigma", field=self.name, mask=np.array(masks))
        paramset.addParameter(np.array(epsilon), "epsilon", field=self.name, mask=np.array(masks))

    def getName(self):
        return self.name

    def _find_atype_key_index(self, atype):
        for n, i in enumerate(self.atom_keys):
            if i == atype:
                return n
        return None

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        method = method_name(nonbondedMethod)
        if method not in ("NoCutoff", "CutoffPeriodic", "CutoffNonPeriodic", "PME"):
            raise ValueError("Illegal nonbonded method for NonbondedForce")
        atoms = list(topdata.atoms())
        n = len(atoms)
        if self.charge_in_residue:
            charges = np.array([float(a.meta["charge"]) for a in atoms])
        else:
            charges = np.array([self.type_to_charge[a.meta[self.key_type]] for a in atoms])
        r_cut = _rc_nm(nonbondedCutoff)
        mode, kappa, K = _coulomb_setup(method, topdata, r_cut, kwargs, 1e-6)
        map_prm = []
        for a in atoms:
            p = self._find_atype_key_index(a.meta[self.key_type])
            if p is None:
                raise ValueError(f"Atom type {a.meta[self.key_type]} not found.")
            map_prm.append(p)
        map_prm = np.asarray(map_prm, dtype=np.int32)
        pbc = method in ("PME", "CutoffPeriodic")
        cov = topdata.buildCovMat()
        self.charges, self.map_prm, self.coul_mode, self.kappa_nm, self.K = charges, map_prm, mode, kappa, K
        self.r_cut, self.pbc = r_cut, pbc
        self.mscales_coul = (0.0, 0.0, self.coulomb14scale, 1.0, 1.0, 1.0)
        self.mscales_lj = (0.0, 0.0, self.lj14scale, 1.0, 1.0, 1.0)
        force = ClassicalForce(n, n_types=len(self.atom_keys), coulomb=mode, pbc=pbc, rc=r_cut * 10.0,
                               kappa=kappa / 10.0, K=K, cov_rows=cov.pairs(),
                               mscales_coul=(0.0, 0.0, self.coulomb14scale, 1.0, 1.0, 1.0),
                               mscales_lj=(0.0, 0.0, self.lj14scale, 1.0, 1.0, 1.0),
                               precision=kwargs.get("precision", "fp32"))
        self.pme_force = force
        disp_corr = None
        if kwargs.get("useDispersionCorrection", False):
            disp_corr = _DispersionCorrection(map_prm, len(self.atom_keys), cov, r_cut)
        self.disp_corr = disp_corr
        name, has_aux = self.name, _has_aux(kwargs)
        q = torch.as_tensor(charges, dtype=torch.float64)

        def potential_fn(positions, box, pairs, params, aux=None):
            p = params[name]
            sig, eps = _t(p["sigma"]), _t(p["epsilon"])
            sig_tt, eps_tt = _lb_tables(sig, eps)
            E = force.energy(_t(positions) * 10.0, _t(box) * 10.0, pairs, charges=q, atom_type=map_prm,
                             sigma_tt=sig_tt * 10.0, eps_tt=eps_tt)
            if disp_corr is not None:
                E = E + disp_corr(_t(box), eps, sig)
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


class _DispersionCorrection:
    """LennardJonesLongRangeForce (inter.py:97-131) with the pair-count matrix of
    classical.py:951-974: E = -2/3 pi N^2 / V <C6> / rc^3 (nm units)."""

    def __init__(self, map_prm, n_types, cov, r_cut):
        count_vec = np.bincount(map_prm, minlength=n_types).astype(np.int64)
        cm = np.zeros((n_types, n_types), dtype=np.int64)
        for i in range(n_types):
            for j in range(i, n_types):
                cm[i, j] = count_vec[i] * count_vec[j] if i != j else count_vec[i] * (count_vec[i] - 1) // 2
        rows = cov.pairs()
        for i, j, d in rows:
            if 0 < d <= 3:
                t1, t2 = sorted((map_prm[i], map_prm[j]))
                cm[t1, t2] -= 1
        self.count = torch.as_tensor(cm, dtype=torch.float64)
        self.n = len(map_prm)
        self.r_cut = r_cut

    def __call__(self, box, epsilon, sigma):
        eps_mat = torch.sqrt(epsilon[:, None] * epsilon[None, :])
        sig_mat = (sigma[:, None] + sigma[None, :]) * 0.5
        c6 = torch.sum(4 * eps_mat * sig_mat ** 6 * self.count) / torch.sum(self.count)
        vol = torch.linalg.det(box)
        return -2.0 / 3.0 * math.pi * self.n * self.n / vol * c6 / self.r_cut ** 3


class CoulombGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "CoulombForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        self.coulomb14scale = float(ffinfo["Forces"][self.name]["meta"]["coulomb14scale"])
        self._use_bcc = False
        bcc, masks = [], []
        for nd in ffinfo["Forces"][self.name]["node"]:
            if nd["name"] == "UseBondChargeCorrection":
                self._use_bcc = True
            if nd["name"] == "BondChargeCorrection":
                bcc.append(float(nd["attrib"]["bcc"]))
                masks.append(_mask(nd["attrib"]))
        paramset.addParameter(np.array(bcc), "bcc", field=self.name, mask=np.array(masks))

    def getName(self):
        return self.name

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        method = method_name(nonbondedMethod)
        if method not in ("NoCutoff", "CutoffPeriodic", "CutoffNonPeriodic", "PME"):
            raise ValueError("Illegal nonbonded method for CoulombForce")
        if self._use_bcc:
            raise NotImplementedError("BondChargeCorrection needs SMARTS matching of the topology (RDKit), "
                                      "which this package does not provide")
        atoms = list(topdata.atoms())
        charges = torch.as_tensor([float(a.meta["charge"]) for a in atoms], dtype=torch.float64)
        r_cut = _rc_nm(nonbondedCutoff)
        mode, kappa, K = _coulomb_setup(method, topdata, r_cut, kwargs, 1e-5)
        self.charges, self.coul_mode, self.kappa_nm, self.K = charges.numpy(), mode, kappa, K
        self.r_cut, self.pbc = r_cut, method in ("PME", "CutoffPeriodic")
        cov = topdata.buildCovMat()
        self.mscales_coul = (0.0, 0.0, self.coulomb14scale, 1.0, 1.0, 1.0)
        force = ClassicalForce(len(atoms), coulomb=mode, pbc=method in ("PME", "CutoffPeriodic"), rc=r_cut * 10.0,
                               kappa=kappa / 10.0, K=K, cov_rows=cov.pairs(), mscales_coul=self.mscales_coul,
                               precision=kwargs.get("precision", "fp32"))
        self.pme_force = force
        has_aux = _has_aux(kwargs)

        def potential_fn(positions, box, pairs, params, aux=None):
            E = force.energy(_t(positions) * 10.0, _t(box) * 10.0, pairs, charges=charges)
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


class LennardJonesGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "LennardJonesForce"
        self.ffinfo = ffinfo
        self.lj14scale = float(ffinfo["Forces"][self.name]["meta"]["lj14scale"])
        self.nbfix_to_idx = {}
        self.atype_to_idx = {}
        sig, eps, smask = [], [], []
        sfix, efix, fmask = [], [], []
        c2t = ffinfo["ClassToType"]
        for nd in ffinfo["Forces"][self.name]["node"]:
            at = nd["attrib"]
            if nd["name"] == "Atom":
                if "type" in at:
                    self.atype_to_idx[at["type"]] = len(sig)
                elif "class" in at:
                    for t in c2t[at["class"]]:
                        self.atype_to_idx[t] = len(sig)
                sig.append(float(at["sigma"]))
                eps.append(float(at["epsilon"]))
                smask.append(_mask(at))
            elif nd["name"] == "NBFixPair":
                if "type1" in at:
                    pairs = [(at["type1"], at["type2"])]
                else:
                    pairs = [(t1, t2) for t1 in c2t[at["class1"]] for t2 in c2t[at["class2"]]]
                for t1, t2 in pairs:
                    self.nbfix_to_idx.setdefault(t1, {})[t2] = len(sfix)
                    self.nbfix_to_idx.setdefault(t2, {})[t1] = len(sfix)
                sfix.append(float(at["sigma"]))
                efix.append(float(at["epsilon"]))
                fmask.append(_mask(at))
        paramset.addField(self.name)
        paramset.addParameter(np.array(sig), "sigma", field=self.name, mask=np.array(smask))
        paramset.addParameter(np.array(eps), "epsilon", field=self.name, mask=np.array(smask))
        paramset.addParameter(np.array(sfix), "sigma_nbfix", field=self.name, mask=np.array(fmask))
        paramset.addParameter(np.array(efix), "epsilon_nbfix", field=self.name, mask=np.array(fmask))
        self.n_types = len(sig)

    def getName(self):
        return self.name

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        method = method_name(nonbondedMethod)
        if method not in ("NoCutoff", "CutoffPeriodic", "CutoffNonPeriodic", "PME"):
            raise ValueError("Illegal nonbonded method for LennardJonesForce")
        atoms = list(topdata.atoms())
        map_prm = []
        for a in atoms:
            if a.meta["type"] not in self.atype_to_idx:
                raise ValueError(f"Atom type {a.meta['type']} not found.")
            map_prm.append(self.atype_to_idx[a.meta["type"]])
        map_prm = np.asarray(map_prm, dtype=np.int32)
        topdata._meta["lj_map_idx"] = map_prm
        nbfix = []
        for t1, d in self.nbfix_to_idx.items():
            for t2, k in d.items():
                nbfix.append((self.atype_to_idx[t1], self.atype_to_idx[t2], k))
        nbfix = np.asarray(nbfix, dtype=np.int64).reshape(-1, 3)
        r_cut = _rc_nm(nonbondedCutoff)
        cov = topdata.buildCovMat()
        self.map_prm, self.nbfix, self.r_cut = map_prm, nbfix, r_cut
        self.pbc = method in ("PME", "CutoffPeriodic")
        self.mscales_lj = (0.0, 0.0, self.lj14scale, 1.0, 1.0, 1.0)
        force = ClassicalForce(len(atoms), n_types=self.n_types, coulomb="none",
                               pbc=method in ("PME", "CutoffPeriodic"), rc=r_cut * 10.0, cov_rows=cov.pairs(),
                               mscales_lj=(0.0, 0.0, self.lj14scale, 1.0, 1.0, 1.0),
                               precision=kwargs.get("precision", "fp32"))
        self.force = force
        name, has_aux = self.name, _has_aux(kwargs)

        def potential_fn(positions, box, pairs, params, aux=None):
            p = params[name]
            sig_tt, eps_tt = _lb_tables(_t(p["sigma"]), _t(p["epsilon"]), nbfix, _t(p["sigma_nbfix"]),
                                        _t(p["epsilon_nbfix"]))
            E = force.energy(_t(positions) * 10.0, _t(box) * 10.0, pairs, atom_type=map_prm,
                             sigma_tt=sig_tt * 10.0, eps_tt=eps_tt)
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


_DMFFGenerators["HarmonicBondForce"] = HarmonicBondGenerator
_DMFFGenerators["HarmonicAngleForce"] = HarmonicAngleGenerator
_DMFFGenerators["PeriodicTorsionForce"] = PeriodicTorsionGenerator
_DMFFGenerators["NonbondedForce"] = NonbondedGenerator
_DMFFGenerators["CoulombForce"] = CoulombGenerator
_DMFFGenerators["LennardJonesForce"] = LennardJonesGenerator
