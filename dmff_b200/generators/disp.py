"""Dispersion generators: ADMPDispPmeForce and ADMPDispForce (dmff/generators/admp.py:22-397).

Same XML attributes and ParamSet names as the reference (A, B, Q, C6, C8, C10; mScale1n with
the trailing 1.0; pmax = 10), same unit conversions (C_n in kJ/mol nm^n -> c_n = sqrt(C_n 10^n)
in Angstrom units; A / 2625.5 to Hartree, B * 0.0529177249 to 1/bohr), same sign convention:
ADMPDispPmeForce returns -E_lr (admp.py:384) and ADMPDispForce returns E_sr - E_lr
(admp.py:208), with E_sr the Tang-Toennies damped short-range term (pairwise.py:100-118) and
E_lr the dispersion PME energy (disp_pme.py:80-130).  Both run on the GPU engine.
"""
import numpy as np
import torch

from ..admp.pme import setup_ewald_parameters
from ..api.hamiltonian import _DMFFGenerators, method_name
from ..api.paramset import ParamSet
from .admp import _rc_angstrom


def _mscales(meta, default=(0.0, 0.0, 0.0, 1.0, 1.0)):
    return [float(meta.get(f"mScale1{i}", default[i - 2])) for i in range(2, 7)] + [1.0]


class _DispBase:
    fields = ("C6", "C8", "C10")

    def __init__(self, ffinfo, paramset: ParamSet, name):
        self.name = name
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        self.ethresh = 5e-4
        self.pmax = 10
        meta = ffinfo["Forces"][self.name]["meta"]
        self.mScales = _mscales(meta)
        self.atom_keys = []
        vals = {f: [] for f in self.fields}
        masks = []
        self.key_type = "type"
        for node in ffinfo["Forces"][self.name]["node"]:
            if node["name"] != "Atom":
                continue
            at = node["attrib"]
            self.key_type = "type" if "type" in at else "class"
            self.atom_keys.append(at[self.key_type])
            for f in self.fields:
                vals[f].append(float(at[f]))
            masks.append(0.0 if at.get("mask", "").upper() == "TRUE" else 1.0)
        for f in self.fields:
            paramset.addParameter(np.array(vals[f]), f, field=self.name, mask=np.array(masks))
        self.force = None

    def getName(self):
        return self.name

    def _common(self, topdata, nonbondedMethod, nonbondedCutoff, kwargs):
        method = method_name(nonbondedMethod)
        if method not in ("CutoffPeriodic", "NoCutoff", "PME"):
            raise ValueError(f"Illegal nonbonded method for {self.name}")
        lpme = method != "CutoffPeriodic"  # admp.py:141-144
        atoms = list(topdata.atoms())
        idx = {k: n for n, k in enumerate(self.atom_keys)}
        map_atomtype = np.array([idx[a.meta[self.key_type]] for a in atoms], dtype=int)
        topdata._meta[self.name + "_map_atomtype"] = map_atomtype
        box = topdata.getPeriodicBoxVectors()
        box = np.asarray(box) * 10.0 if (lpme and box is not None) else np.ones((3, 3))
        rc = _rc_angstrom(nonbondedCutoff)
        if "ethresh" in kwargs:
            self.ethresh = kwargs["ethresh"]
        from ..admp.disp_pme import ADMPDispPmeForce
        cov = topdata.buildCovMat()
        force = ADMPDispPmeForce(box, rc, self.ethresh, self.pmax, lpme=lpme, cov_rows=cov.pairs(),
                                 tt_damping=self.tt, precision=kwargs.get("precision", "fp32"))
        self.force = force
        return force, map_atomtype, bool(kwargs.get("has_aux", False))

    @staticmethod
    def _c_list(p, mt):
        mt = torch.as_tensor(mt)
        return torch.stack([torch.sqrt(torch.as_tensor(p["C6"])[mt] * 1e6), torch.sqrt(torch.as_tensor(p["C8"])[mt] * 1e8),
                            torch.sqrt(torch.as_tensor(p["C10"])[mt] * 1e10)], dim=1)


class ADMPDispPmeGenerator(_DispBase):
    tt = False

    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "ADMPDispPmeForce")

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        force, mt, has_aux = self._common(topdata, nonbondedMethod, nonbondedCutoff, kwargs)
        name, mS = self.name, self.mScales

        def potential_fn(positions, box, pairs, params, aux=None):
            positions = torch.as_tensor(positions, dtype=torch.float64) * 10.0
            box = torch.as_tensor(box, dtype=torch.float64) * 10.0
            c_list = self._c_list(params[name], mt)
            E_lr = force.get_energy(positions, box, pairs, c_list, mS)
            return (-E_lr, aux) if has_aux else -E_lr

        self._jaxPotential = potential_fn
        return potential_fn


class ADMPDispGenerator(_DispBase):
    fields = ("A", "B", "Q", "C6", "C8", "C10")
    tt = True

    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "ADMPDispForce")
        self.mScales = _mscales(ffinfo["Forces"][self.name]["meta"])

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        force, mt, has_aux = self._common(topdata, nonbondedMethod, nonbondedCutoff, kwargs)
        name, mS = self.name, self.mScales

        def potential_fn(positions, box, pairs, params, aux=None):
            positions = torch.as_tensor(positions, dtype=torch.float64) * 10.0
            box = torch.as_tensor(box, dtype=torch.float64) * 10.0
            p = params[name]
            m = torch.as_tensor(mt)
            a_list = torch.as_tensor(p["A"])[m] / 2625.5
            b_list = torch.as_tensor(p["B"])[m] * 0.0529177249
            q_list = torch.as_tensor(p["Q"])[m]
            c_list = self._c_list(p, mt)
            E = force.get_energy(positions, box, pairs, c_list, mS, tt=(a_list, b_list, q_list))
            return (E, aux) if has_aux else E

        self._jaxPotential = potential_fn
        return potential_fn


_DMFFGenerators["ADMPDispPmeForce"] = ADMPDispPmeGenerator
_DMFFGenerators["ADMPDispForce"] = ADMPDispGenerator
