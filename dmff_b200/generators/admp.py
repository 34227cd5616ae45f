"""ADMP generators: XML -> ParamSet + potential_fn, backed by the B200 engine.

Mirrors dmff/generators/admp.py: ``ADMPPmeGenerator`` (866-1414) parses the same XML
attributes (lmax, m/p/dScale1n with the trailing 1.0, Multipole/Atom c0 dX.. qXX.., Polarize
polarizabilityXX.. thole; dipoles x10 and quadrupoles x300 into the Angstrom convention,
cart->harm conversion, pol x1000) and assigns local axes with the same rules; its
``potential_fn(positions_nm, box_nm, pairs, params, aux=None)`` returns a torch scalar.
"""
import numpy as np
import torch

from ..admp.pme import ADMPPmeForce
from ..api.hamiltonian import _DMFFGenerators, method_name
from ..api.paramset import ParamSet
from ..synthetic import cart2harm

ZThenX, Bisector, ZBisect, ThreeFold, ZOnly, NoAxisType = 0, 1, 2, 3, 4, 5


def _rc_angstrom(nonbondedCutoff):
    if hasattr(nonbondedCutoff, "value_in_unit"):
        try:
            import openmm.unit as unit  # noqa: F401  (only when the caller passes OpenMM quantities)
            return nonbondedCutoff.value_in_unit(unit.angstrom)
        except ImportError:
            pass
    return float(nonbondedCutoff) * 10.0


class ADMPPmeGenerator:
    def __init__(self, ffinfo: dict, paramset: ParamSet):
        self.name = "ADMPPmeForce"
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        self._jaxPotential = None
        self.multipole_types = []
        self.polarize_types = []
        self.ethresh = 5e-4
        self.step_pol = None
        self.pme_force = None
        meta = self.ffinfo["Forces"][self.name]["meta"]
        self.lmax = int(meta["lmax"])
        default_mscales = [0.0, 0.0, 1.0, 1.0, 1.0]
        default_pscales = [0.0, 0.0, 1.0, 1.0, 1.0]
        default_dscales = [1.0, 1.0, 1.0, 1.0, 1.0]
        self.mScales = [float(meta.get(f"mScale1{i}", default_mscales[i - 2])) for i in range(2, 7)] + [1.0]
        self.pScales = [float(meta.get(f"pScale1{i}", default_pscales[i - 2])) for i in range(2, 7)] + [1.0]
        self.dScales = [float(meta.get(f"dScale1{i}", default_dscales[i - 2])) for i in range(2, 7)] + [1.0]
        nodes = self.ffinfo["Forces"][self.name]["node"]
        polarize_nodes = [nd for nd in nodes if nd["name"] == "Polarize"]
        self.lpol = len(polarize_nodes) > 0
        multipole_nodes = [nd for nd in nodes if nd["name"] in ("Multipole", "Atom")]
        Q = np.zeros((len(multipole_nodes), 10))
        kxs, kys, kzs, masks = [], [], [], []
        self.key_type = "type"
        for k, nd in enumerate(multipole_nodes):
            at = nd["attrib"]
            self.key_type = "type" if "type" in at else "class"
            self.multipole_types.append(at[self.key_type])
            kxs.append(at.get("kx", ""))
            kys.append(at.get("ky", ""))
            kzs.append(at.get("kz", ""))
            Q[k, 0] = float(at["c0"])
            if self.lmax >= 1:
                Q[k, 1:4] = [float(at["dX"]), float(at["dY"]), float(at["dZ"])]
            if self.lmax >= 2:
                Q[k, 4:10] = [float(at[x]) for x in ("qXX", "qYY", "qZZ", "qXY", "qXZ", "qYZ")]
            masks.append(0.0 if at.get("mask", "").upper() == "TRUE" else 1.0)
        Q[:, 1:4] *= 10
        Q[:, 4:10] *= 300
        self.kStrings = {"kx": kxs, "ky": kys, "kz": kzs}
        if self.lpol:
            pol, thole, pmask = [], [], []
            for nd in polarize_nodes:
                at = nd["attrib"]
                self.polarize_types.append(at[self.key_type])
                pol.append((float(at["polarizabilityXX"]) + float(at["polarizabilityYY"])
                            + float(at["polarizabilityZZ"])) / 3.0)
                thole.append(float(at["thole"]))
                pmask.append(0.0 if at.get("mask", "").upper() == "TRUE" else 1.0)
            paramset.addParameter(np.array(pol) * 1000.0, "pol", field=self.name, mask=np.array(pmask))
            paramset.addParameter(np.array(thole), "thole", field=self.name, mask=np.array(pmask))
        n_h = (self.lmax + 1) ** 2
        Q_local = cart2harm(Q)[:, :n_h]
        paramset.addParameter(Q_local, "Q_local", field=self.name, mask=np.array(masks))

    def getName(self):
        return self.name

    @staticmethod
    def setAxisType(kIndices):
        """dmff/generators/admp.py:1118-1160."""
        kz, kx, ky = kIndices
        kyNeg = ky.startswith("-")
        ky = ky[1:] if kyNeg else ky
        kxNeg = kx.startswith("-")
        kx = kx[1:] if kxNeg else kx
        kzNeg = kz.startswith("-")
        kz = kz[1:] if kzNeg else kz
        axisType = ZThenX
        if not kz:
            axisType = NoAxisType
        if kz and not kx:
            axisType = ZOnly
        if (kz and kzNeg) or (kx and kxNeg):
            axisType = Bisector
        if kx and kxNeg and ky and kyNeg:
            axisType = ZBisect
        if kz and kzNeg and kx and kxNeg and ky and kyNeg:
            axisType = ThreeFold
        return axisType, [kz, kx, ky]

    def _assign_axes(self, topdata, cov):
        """Local-axis assignment, dmff/generators/admp.py:1209-1336 (same search order)."""
        atoms = list(topdata.atoms())
        n_atoms = len(atoms)
        key = self.key_type
        axis_types, axis_indices = {}, {}
        patched = np.zeros(n_atoms, dtype=int)
        by_type = {}
        for i, a in enumerate(atoms):
            by_type.setdefault(a.meta.get(key), []).append(i)
        for rev in range(len(self.multipole_types)):
            it = len(self.multipole_types) - rev - 1
            t = self.multipole_types[it]
            for ia in by_type.get(t, []):
                if patched[ia] > 0:
                    continue
                axisType, (kz, kx, ky) = self.setAxisType(
                    [self.kStrings["kz"][it], self.kStrings["kx"][it], self.kStrings["ky"][it]])
                zaxis = xaxis = yaxis = -1
                neighbors = cov.neighbors(ia, 1)
                if len(neighbors) < 1 and axisType != NoAxisType:
                    continue
                tp = lambda j: atoms[j].meta.get(key)
                if axisType == ZThenX:
                    zaxis = next((j for j in neighbors if tp(j) == kz), -1)
                    if zaxis < 0:
                        continue
                    xaxis = next((j for j in neighbors if j != zaxis and tp(j) == kx), -1)
                    if xaxis < 0:
                        xaxis = next((j for j in cov.neighbors(zaxis, 1) if j != ia and tp(j) == kx), -1)
                    if xaxis < 0:
                        continue
                elif axisType == ZOnly:
                    zaxis = next((j for j in neighbors if tp(j) == kz), -1)
                    if zaxis < 0:
                        continue
                elif axisType == Bisector:
                    zaxis = next((j for j in neighbors if tp(j) == kz), -1)
                    if zaxis < 0:
                        continue
                    xaxis = next((j for j in neighbors if j != zaxis and tp(j) == kx), -1)
                    if xaxis < 0:
                        continue
                elif axisType in (ZBisect, ThreeFold):
                    zaxis = next((j for j in neighbors if tp(j) == kz), -1)
                    if zaxis < 0:
                        continue
                    xaxis = next((j for j in neighbors if j != zaxis and tp(j) == kx), -1)
                    if xaxis < 0:
                        continue
                    yaxis = next((j for j in neighbors if j not in (zaxis, xaxis) and tp(j) == ky), -1)
                    if yaxis < 0:
                        continue
                elif axisType != NoAxisType:
                    continue
                axis_types[ia] = axisType
                axis_indices[ia] = [zaxis, xaxis, yaxis]
                patched[ia] = 1
        for ia in range(n_atoms):
            if patched[ia] < 0.5:
                raise ValueError("Atom %d not matched in forcefield!" % ia)
        return (np.array([axis_types[i] for i in range(n_atoms)], dtype=np.int32),
                np.array([axis_indices[i] for i in range(n_atoms)], dtype=np.int32))

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        method = method_name(nonbondedMethod)
        if method not in ("CutoffPeriodic", "CutoffNonPeriodic", "NoCutoff", "PME"):
            raise ValueError("Illegal nonbonded method for ADMPPmeForce")
        lpme = method == "PME"
        n_atoms = topdata.getNumAtoms()
        atoms = list(topdata.atoms())
        mt = {t: k for k, t in enumerate(self.multipole_types)}
        pt = {t: k for k, t in enumerate(self.polarize_types)}
        map_atomtype = np.array([mt[a.meta[self.key_type]] for a in atoms], dtype=int)
        map_poltype = np.array([pt[a.meta[self.key_type]] for a in atoms], dtype=int) if self.lpol else np.zeros(
            n_atoms, dtype=int)
        box = topdata.getPeriodicBoxVectors()
        box = np.asarray(box) * 10.0 if box is not None else np.eye(3)
        rc = _rc_angstrom(nonbondedCutoff)
        cov = topdata.buildCovMat()
        if self.lmax > 0:
            axis_types, axis_indices = self._assign_axes(topdata, cov)
        else:
            axis_types, axis_indices = np.full(n_atoms, NoAxisType, dtype=np.int32), None
        has_aux = bool(kwargs.get("has_aux", False))
        if "ethresh" in kwargs:
            self.ethresh = kwargs["ethresh"]
        if "step_pol" in kwargs:
            self.step_pol = kwargs["step_pol"]
        pme_force = ADMPPmeForce(
            box, map_atomtype, axis_types, axis_indices, rc, self.ethresh, self.lmax, self.lpol, lpme,
            self.step_pol, has_aux, cov_rows=cov.pairs(), precision=kwargs.get("precision", "fp32"),
            pol_solver=kwargs.get("pol_solver", "cg"), cg_tol=kwargs.get("cg_tol", 1e-6))
        self.pme_force = pme_force
        topdata._meta[self.name + "_map_atomtype"] = map_atomtype
        topdata._meta[self.name + "_map_poltype"] = map_poltype
        lpol, name = self.lpol, self.name
        mS, pS, dS = self.mScales, self.pScales, self.dScales

        def potential_fn(positions, box, pairs, params, aux=None):
            positions = torch.as_tensor(positions, dtype=torch.float64) * 10.0
            box = torch.as_tensor(box, dtype=torch.float64) * 10.0
            p = params[name]
            Q_local = torch.as_tensor(p["Q_local"])[torch.as_tensor(map_atomtype)]
            if lpol:
                pol = torch.as_tensor(p["pol"])[torch.as_tensor(map_poltype)]
                tholes = torch.as_tensor(p["thole"])[torch.as_tensor(map_poltype)]
                if has_aux:
                    U0 = aux["U_ind"] if (aux is not None and "U_ind" in aux) else torch.zeros((n_atoms, 3))
                    aux = {} if aux is None else aux
                    return pme_force.get_energy(positions, box, pairs, Q_local, pol, tholes, mS, pS, dS,
                                                U_init=U0, aux=aux)
                return pme_force.get_energy(positions, box, pairs, Q_local, pol, tholes, mS, pS, dS,
                                            U_init=pme_force.U_ind)
            energy = pme_force.get_energy(positions, box, pairs, Q_local, mS)
            return (energy, aux) if has_aux else energy

        self._jaxPotential = potential_fn
        return potential_fn

    def getJaxPotential(self):
        return self._jaxPotential


_DMFFGenerators["ADMPPmeForce"] = ADMPPmeGenerator
