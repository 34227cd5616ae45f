"""ADMPQeqForce generator (dmff/generators/qeq.py).

Same XML (an ``ADMPQeqForce`` element with ``coulomb14scale`` and ``DampMod``, ``Atom`` entries
with ``type`` or ``class`` and ``chi``, ``J``, ``eta``, an optional ``mask``), the same ParamSet
names (chi, J, eta) and the same ``createPotential`` keywords (ethresh, PmeCoeffMethod,
PmeSpacing, neutral, slab, constQ, const_list / const_vals, has_aux) as the reference; without
an explicit constraint list every residue keeps its total initial charge (qeq.py generator,
createPotential).  The potential solves the charges on the GPU engines (``admp.qeq``).
"""
import numpy as np
import torch

from ..admp.pme import setup_ewald_parameters
from ..admp.qeq import ADMPQeqForce
from ..api.hamiltonian import _DMFFGenerators, method_name
from ..api.paramset import ParamSet


def _rc_nm(nonbondedCutoff):
    if hasattr(nonbondedCutoff, "value_in_unit"):
        import openmm.unit as unit
        return nonbondedCutoff.value_in_unit(unit.nanometer)
    return float(nonbondedCutoff)


class ADMPQeqGenerator:
    def __init__(self, ffinfo, paramset: ParamSet):
        self.name = "ADMPQeqForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        meta = ffinfo["Forces"][self.name]["meta"]
        self.coulomb14scale = float(meta["coulomb14scale"])
        self.damp_mod = int(meta["DampMod"]) if "DampMod" in meta else 3
        self.key_type = None
        keys, chi, J, eta, mask = [], [], [], [], []
        for node in ffinfo["Forces"][self.name]["node"]:
            at = node["attrib"]
            if self.key_type is None:
                if "type" in at:
                    self.key_type = "type"
                elif "class" in at:
                    self.key_type = "class"
                else:
                    raise ValueError("Cannot find key type for ADMPQeqForce.")
            elif self.key_type not in at:
                raise ValueError("Keyword 'class' or 'type' cannot be used together.")
            keys.append(at[self.key_type])
            chi.append(float(at["chi"]))
            J.append(float(at["J"]))
            eta.append(float(at["eta"]))
            mask.append(0.0 if at.get("mask", "").upper() == "TRUE" else 1.0)
        self.atom_keys = keys
        mask = np.array(mask)
        paramset.addParameter(np.array(chi), "chi", field=self.name, mask=mask)
        paramset.addParameter(np.array(J), "J", field=self.name, mask=mask)
        paramset.addParameter(np.array(eta), "eta", field=self.name, mask=mask)
        self._jaxPotential = None

    def getName(self):
        return self.name

    def overwrite(self, paramset):
        nodes = [i for i, nd in enumerate(self.ffinfo["Forces"][self.name]["node"]) if nd["name"] == "Atom"]
        p = paramset[self.name]
        m = paramset.mask[self.name]["chi"]
        for k, idx in enumerate(nodes):
            at = self.ffinfo["Forces"][self.name]["node"][idx]["attrib"]
            at["chi"], at["J"], at["eta"] = float(p["chi"][k]), float(p["J"][k]), float(p["eta"][k])
            if float(m[k]) < 0.999:
                at["mask"] = "true"

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        method = method_name(nonbondedMethod)
        if method not in ("NoCutoff", "PME"):
            raise ValueError("Illegal nonbonded method for NonbondedForce")
        no_cut = method == "NoCutoff"
        mscales = [0.0, 0.0, self.coulomb14scale, 1.0, 1.0, 1.0]
        r_cut = _rc_nm(nonbondedCutoff)
        if not no_cut:
            box = np.asarray(topdata.getPeriodicBoxVectors(), dtype=np.float64)
            kappa, K1, K2, K3 = setup_ewald_parameters(r_cut, kwargs.get("ethresh", 1e-5), box,
                                                       kwargs.get("PmeSpacing", 0.1),
                                                       kwargs.get("PmeCoeffMethod", "openmm"))
        else:
            kappa, K1, K2, K3 = 1.0, 1, 1, 1
        atoms = list(topdata.atoms())
        init_q = np.array([float(a.meta["charge"]) for a in atoms])
        index = {k: i for i, k in enumerate(self.atom_keys)}
        map_idx = np.array([index[a.meta[self.key_type]] for a in atoms], dtype=np.int64)
        if "const_list" in kwargs and "const_vals" in kwargs:
            const_list, const_vals = kwargs["const_list"], kwargs["const_vals"]
        else:
            const_list, const_vals = [], []
            for r in topdata.residues():
                idx = [a.index for a in r.atoms()]
                const_list.append(idx)
                const_vals.append(float(np.sum(init_q[idx])))
        has_aux = bool(kwargs.get("has_aux", False))
        force = ADMPQeqForce(init_q, r_cut, kappa, (K1, K2, K3), damp_mod=self.damp_mod, const_list=const_list,
                             const_vals=const_vals, neutral_flag=kwargs.get("neutral", True),
                             slab_flag=kwargs.get("slab", False), constQ=kwargs.get("constQ", True),
                             pbc_flag=not no_cut, has_aux=has_aux, precision=kwargs.get("precision", "fp64"))
        self.qeq_force = force
        energy = force.generate_get_energy()
        name = self.name
        m = torch.as_tensor(map_idx)

        def potential_fn(positions, box, pairs, params, aux=None):
            p = params[name]
            eta = torch.as_tensor(p["eta"], dtype=torch.float64)[m]
            chi = torch.as_tensor(p["chi"], dtype=torch.float64)[m]
            J = torch.as_tensor(p["J"], dtype=torch.float64)[m]
            if has_aux:
                return energy(positions, box, pairs, mscales, eta, chi, J, aux)
            return energy(positions, box, pairs, mscales, eta, chi, J)

        self._jaxPotential = potential_fn
        return potential_fn

    def getJaxPotential(self):
        return self._jaxPotential


_DMFFGenerators["ADMPQeqForce"] = ADMPQeqGenerator
