"""Short-range ADMP generators: QqTtDampingForce, SlaterDampingForce, SlaterExForce and the
SlaterSrEs / SlaterSrPol / SlaterSrDisp / SlaterDhf terms (dmff/generators/admp.py:400-863).

Same XML attributes and ParamSet names as the reference (B, Q; B, C6, C8, C10; A, B; mScale1n with
the default (0, 0, 0, 1, 1) and the trailing 1.0; a ``mask`` attribute freezes a type), same
unit conversions inside the potential (positions and box nm -> A; B / 10 to 1/A; C_n ->
sqrt(C_n 10^n)), same signs (the SlaterSr* and SlaterDhf terms are the Slater exchange form with
a minus sign, admp.py:802-843).  Each potential sums its kernel over the pair rows on the GPU
engine's short-range pair kernel (``admp.pairwise.generate_pairwise_interaction``).
"""
import numpy as np
import torch

from ..admp.pairwise import (TT_damping_qq_kernel, generate_pairwise_interaction, slater_disp_damping_kernel,
                             slater_sr_kernel)
from ..api.hamiltonian import _DMFFGenerators
from ..api.paramset import ParamSet


class _ShortRangeBase:
    fields = ()
    kernel = None
    sign = 1.0

    def __init__(self, ffinfo, paramset: ParamSet, name):
        self.name = name
        self.ffinfo = ffinfo
        paramset.addField(self.name)
        meta = ffinfo["Forces"][self.name]["meta"]
        default = (0.0, 0.0, 0.0, 1.0, 1.0)
        self.mScales = [float(meta.get(f"mScale1{i}", default[i - 2])) for i in range(2, 7)] + [1.0]
        self.atom_keys = []
        self.key_type = None
        vals = {f: [] for f in self.fields}
        masks = []
        for node in ffinfo["Forces"][self.name]["node"]:
            if node["name"] != "Atom":
                continue
            at = node["attrib"]
            self.key_type = "type" if "type" in at else "class"
            self.atom_keys.append(at[self.key_type])
            for f in self.fields:
                vals[f].append(float(at[f]))
            masks.append(0.0 if at.get("mask", "").upper() == "TRUE" else 1.0)
        self.atom_keys = np.array(self.atom_keys)
        for f in self.fields:
            paramset.addParameter(np.array(vals[f]), f, field=self.name, mask=np.array(masks))
        self._jaxPotential = None

    def getName(self):
        return self.name

    def getJaxPotential(self):
        return self._jaxPotential

    def _per_atom(self, p, mt):
        """the kernel's per-atom parameters, in the order of its signature and A units"""
        raise NotImplementedError

    def createPotential(self, topdata, nonbondedMethod, nonbondedCutoff, **kwargs):
        atoms = list(topdata.atoms())
        map_atomtype = np.array([np.where(self.atom_keys == a.meta[self.key_type])[0][0] for a in atoms], dtype=int)
        topdata._meta[self.name + "_map_atomtype"] = map_atomtype
        pot_fn_sr = generate_pairwise_interaction(self.kernel, static_args={},
                                                  precision=kwargs.get("precision", "fp64"))
        has_aux = bool(kwargs.get("has_aux", False))
        name, mS, sign = self.name, self.mScales, self.sign
        mt = torch.as_tensor(map_atomtype)

        def potential_fn(positions, box, pairs, params, aux=None):
            positions = torch.as_tensor(positions, dtype=torch.float64) * 10.0
            box = torch.as_tensor(box, dtype=torch.float64) * 10.0
            e = pot_fn_sr(positions, box, pairs, mS, *self._per_atom(params[name], mt))
            e = e if sign == 1.0 else sign * e
            return (e, aux) if has_aux else e

        self._jaxPotential = potential_fn
        return potential_fn


def _p(p, k, mt):
    return torch.as_tensor(p[k], dtype=torch.float64)[mt]


class QqTtDampingGenerator(_ShortRangeBase):
    """E = -DIELECTRIC sum e^-br (1 + br) q_i q_j / r (admp.py:400-526)."""
    fields = ("B", "Q")
    kernel = staticmethod(TT_damping_qq_kernel)

    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "QqTtDampingForce")

    def _per_atom(self, p, mt):
        return _p(p, "B", mt) / 10.0, _p(p, "Q", mt)


class SlaterDampingGenerator(_ShortRangeBase):
    """Slater-ISA damped C6 / C8 / C10 dispersion (admp.py:529-669)."""
    fields = ("B", "C6", "C8", "C10")
    kernel = staticmethod(slater_disp_damping_kernel)

    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "SlaterDampingForce")

    def _per_atom(self, p, mt):
        return (_p(p, "B", mt) / 10.0, torch.sqrt(_p(p, "C6", mt) * 1e6), torch.sqrt(_p(p, "C8", mt) * 1e8),
                torch.sqrt(_p(p, "C10", mt) * 1e10))


class SlaterExGenerator(_ShortRangeBase):
    """Slater-ISA exchange, sum A_i A_j ((Br)^2 / 3 + Br + 1) e^-Br (admp.py:672-790)."""
    fields = ("A", "B")
    kernel = staticmethod(slater_sr_kernel)

    def __init__(self, ffinfo, paramset, default_name=None):
        super().__init__(ffinfo, paramset, default_name or "SlaterExForce")

    def _per_atom(self, p, mt):
        return _p(p, "A", mt), _p(p, "B", mt) / 10.0


class SlaterSrEsGenerator(SlaterExGenerator):
    """The exchange form with a minus sign (admp.py:795-843)."""
    sign = -1.0

    def __init__(self, ffinfo, paramset, default_name=None):
        super().__init__(ffinfo, paramset, default_name or "SlaterSrEsForce")


class SlaterSrPolGenerator(SlaterSrEsGenerator):
    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "SlaterSrPolForce")


class SlaterSrDispGenerator(SlaterSrEsGenerator):
    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "SlaterSrDispForce")


class SlaterDhfGenerator(SlaterSrEsGenerator):
    def __init__(self, ffinfo, paramset):
        super().__init__(ffinfo, paramset, "SlaterDhfForce")


_DMFFGenerators["QqTtDampingForce"] = QqTtDampingGenerator
_DMFFGenerators["SlaterDampingForce"] = SlaterDampingGenerator
_DMFFGenerators["SlaterExForce"] = SlaterExGenerator
_DMFFGenerators["SlaterSrEsForce"] = SlaterSrEsGenerator
_DMFFGenerators["SlaterSrPolForce"] = SlaterSrPolGenerator
_DMFFGenerators["SlaterSrDispForce"] = SlaterSrDispGenerator
_DMFFGenerators["SlaterDhfForce"] = SlaterDhfGenerator
