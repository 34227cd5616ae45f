"""Drop-ins for dmff/classical/inter.py: the nonbonded force objects a caller builds directly.

Same class names, constructor arguments and ``generate_get_energy()`` closures as the reference
(``LennardJonesForce`` inter.py:17-93, ``LennardJonesLongRangeForce`` 96-131,
``CoulNoCutoffForce`` 133-201, ``CoulReactionFieldForce`` 204-266, ``CoulombPMEForce``
269-335), in the reference's units (nm, e, kJ/mol; Ewald kappa in 1/nm).  The pair terms run in
the engine's CUDA pair kernel (``ClassicalForce``, libdmffb200.so): positions, box and lengths
are handed over in Angstrom, which leaves every energy unchanged.  The returned energies are
torch scalars; autograd gives dE/dpositions, dE/dbox and the adjoints of charges (and through
them ``bcc``), epsilon, sigma and the NBFix values.

Pair rows follow the reference: (i, j, nbond) with rows i >= j treated as padding, the scale of a
row read as ``mscales[nbond - 1]`` (nbond 0 takes the last entry), and no distance cutoff on the
rows given.  ``mscales`` is a six-entry vector; each distinct vector gets its own engine (it is
a compile-time table of the kernel), and it is not differentiated.
"""
import numpy as np
import torch

from ..admp.pme import DIELECTRIC
from .forces import ClassicalForce

ONE_4PI_EPS0 = DIELECTRIC * 0.1  # kJ/mol nm / e^2 (inter.py:14)


def _t(x):
    return torch.as_tensor(x, dtype=torch.float64)


def _mscales_key(mscales):
    m = tuple(float(x) for x in np.asarray(torch.as_tensor(mscales).detach().cpu(), dtype=np.float64).ravel())
    if len(m) != 6:
        raise ValueError(f"mscales must have 6 entries (1-2 ... 1-6 and beyond), got {len(m)}")
    return m


def _need_pairs(pairs):
    if pairs is None:
        raise ValueError("pairs (i, j, nbond) rows are required")
    return pairs


def _lj_tables(epsilon, sigma, map_nbfix, epsfix, sigfix):
    """Type-pair tables of inter.py:62-72: eps_ij = sqrt(eps_i eps_j + 1e-32), sigma_ij the
    arithmetic mean, then each NBFix row (t1, t2, k) sets both orientations, rows in order."""
    eps_tt = torch.sqrt(epsilon[:, None] * epsilon[None, :] + 1e-32)
    sig_tt = (sigma[:, None] + sigma[None, :]) * 0.5
    nb = np.asarray(map_nbfix if map_nbfix is not None else np.zeros((0, 3)), dtype=np.int64).reshape(-1, 3)
    for a, b, k in nb:
        idx = (torch.tensor([a, b]), torch.tensor([b, a]))
        eps_tt = eps_tt.index_put(idx, _t(epsfix)[k].expand(2))
        sig_tt = sig_tt.index_put(idx, _t(sigfix)[k].expand(2))
    return eps_tt, sig_tt


class LennardJonesForce:
    """Lennard-Jones over pair rows, Lorentz-Berthelot mixing with NBFix overrides (inter.py:17-93).

    ``isSwitch`` (the optional switching function of inter.py:51-55) is not built: the
    reference's generators always pass False."""

    def __init__(self, r_switch, r_cut, map_prm, map_nbfix, isSwitch: bool = False, isPBC: bool = True,
                 isNoCut: bool = False, precision="fp32", device=None) -> None:
        if isSwitch:
            raise NotImplementedError("LennardJonesForce(isSwitch=True) is not supported")
        self.isSwitch = isSwitch
        self.r_switch = r_switch
        self.r_cut = r_cut
        self.map_prm = np.asarray(map_prm, dtype=np.int32)
        self.map_nbfix = np.asarray(map_nbfix if map_nbfix is not None else np.zeros((0, 3)),
                                    dtype=np.int64).reshape(-1, 3)
        self.ifPBC = isPBC
        self.ifNoCut = isNoCut
        self.precision = precision
        self.device = device
        self._forces = {}

    def _force(self, n_types, mscales):
        key = (int(n_types), _mscales_key(mscales))
        f = self._forces.get(key)
        if f is None:
            f = ClassicalForce(len(self.map_prm), n_types=n_types, coulomb="none", pbc=self.ifPBC,
                               rc=float(self.r_cut) * 10.0, mscales_lj=key[1], precision=self.precision,
                               device=self.device)
            self._forces[key] = f
        return f

    def generate_get_energy(self):
        def get_energy(positions, box, pairs, epsilon, sigma, epsfix, sigfix, mscales, aux=None):
            epsilon, sigma = _t(epsilon), _t(sigma)
            f = self._force(epsilon.shape[0], mscales)
            eps_tt, sig_tt = _lj_tables(epsilon, sigma, self.map_nbfix, epsfix, sigfix)
            E = f.energy(_t(positions) * 10.0, _t(box) * 10.0, _need_pairs(pairs), atom_type=self.map_prm,
                         sigma_tt=sig_tt * 10.0, eps_tt=eps_tt)
            return E if aux is None else (E, aux)

        return get_energy


class LennardJonesLongRangeForce:
    """Long-range dispersion correction (inter.py:96-131):
    E = -2/3 pi N^2 / V * <4 eps_ij sigma_ij^6> / rc^3, the average taken over the type-pair
    count matrix.  A few type-pair operations on the host (torch); NBFix values set one
    orientation only, as the reference does."""

    def __init__(self, r_cut: float, map_prm, map_nbfix, countMat):
        self.r_cut = r_cut
        self.map_prm = map_prm
        self.map_nbfix = np.asarray(map_nbfix if map_nbfix is not None else np.zeros((0, 3)),
                                    dtype=np.int64).reshape(-1, 3)
        self.countMat = countMat
        self.numParticles = len(map_prm)

    def generate_get_energy(self):
        def get_energy(box, epsilon, sigma, epsfix, sigfix):
            epsilon, sigma = _t(epsilon), _t(sigma)
            eps_mat = torch.sqrt(epsilon[:, None] * epsilon[None, :])
            sig_mat = (sigma[:, None] + sigma[None, :]) * 0.5
            if len(self.map_nbfix):
                a = torch.as_tensor(self.map_nbfix[:, 0])
                b = torch.as_tensor(self.map_nbfix[:, 1])
                k = torch.as_tensor(self.map_nbfix[:, 2])
                eps_mat = eps_mat.index_put((a, b), _t(epsfix)[k])
                sig_mat = sig_mat.index_put((a, b), _t(sigfix)[k])
            cm = _t(self.countMat)
            c6 = torch.sum(4 * eps_mat * sig_mat ** 6 * cm) / torch.sum(cm)
            vol = torch.linalg.det(_t(box))
            n = self.numParticles
            return -2.0 / 3.0 * np.pi * n * n / vol * c6 / self.r_cut ** 3

        return get_energy


class _CoulombBase:
    """Charges = init_charges (+ topology_matrix @ bcc when a topology matrix is given), one
    engine per mscales vector; the energy is the engine's times 1 / epsilon_1."""

    coulomb = None

    def _setup(self, init_charges, topology_matrix, eps_1, pbc, rc_nm, kappa_nm=0.0, K=(0, 0, 0),
               eps_solv=78.5, precision="fp32", device=None):
        self.init_charges = init_charges
        self.top_mat = topology_matrix
        self.eps_1 = eps_1
        self._cfg = dict(pbc=pbc, rc=float(rc_nm) * 10.0, kappa=float(kappa_nm) / 10.0, K=tuple(int(k) for k in K),
                         eps_solvent=float(eps_solv), precision=precision, device=device)
        self._forces = {}

    def _force(self, n, mscales):
        key = _mscales_key(mscales)
        f = self._forces.get((n, key))
        if f is None:
            f = ClassicalForce(n, coulomb=self.coulomb, mscales_coul=key, **self._cfg)
            self._forces[(n, key)] = f
        return f

    def _charges(self, bcc):
        q = _t(self.init_charges).reshape(-1)
        if bcc is not None:
            q = q + (_t(self.top_mat) @ _t(bcc)).reshape(-1)
        return q

    def _energy(self, positions, box, pairs, bcc, mscales):
        q = self._charges(bcc)
        f = self._force(q.shape[0], mscales)
        E = f.energy(_t(positions) * 10.0, _t(box) * 10.0, _need_pairs(pairs), charges=q)
        return E if self.eps_1 == 1.0 else E / self.eps_1

    def generate_get_energy(self):
        if self.top_mat is None:
            def get_energy(positions, box, pairs, mscales):
                return self._energy(positions, box, pairs, None, mscales)
        else:
            def get_energy(positions, box, pairs, bcc, mscales):
                return self._energy(positions, box, pairs, bcc, mscales)
        return get_energy


class CoulNoCutoffForce(_CoulombBase):
    """q_i q_j / (4 pi eps0 eps_1 r) over the pair rows, no periodic image (inter.py:133-174)."""

    coulomb = "nocutoff"

    def __init__(self, init_charges, epsilon_1=1.0, topology_matrix=None, precision="fp32", device=None) -> None:
        self._setup(init_charges, topology_matrix, epsilon_1, False, 1.0, precision=precision, device=device)

    def generate_esp(self):
        """``get_esp(positions, grids[, bcc])`` -> sum_i ONE_4PI_EPS0 q_i / |r_i - g + 1e-16| per
        grid point (inter.py:176-201; the 1e-16 is added to each component, as there).  Host
        torch on the input's device, 4096 grid points at a time."""

        def esp(positions, grids, bcc):
            pos = _t(positions)
            g = _t(grids).to(pos.device)
            q = self._charges(bcc).to(pos.device)
            out = []
            for g0 in range(0, g.shape[0], 4096):
                r = torch.linalg.norm(pos[None, :, :] - g[g0:g0 + 4096, None, :] + 1e-16, dim=-1)
                out.append((ONE_4PI_EPS0 * q / r).sum(-1))
            return torch.cat(out)

        if self.top_mat is None:
            def get_esp(positions, grids):
                return esp(positions, grids, None)
        else:
            def get_esp(positions, grids, bcc):
                return esp(positions, grids, bcc)
        return get_esp


class CoulReactionFieldForce(_CoulombBase):
    """Reaction field (inter.py:204-266): q_i q_j / (4 pi eps0 eps_1) (1/r + k_rf r^2 - c_rf) with
    k_rf = (eps_solv - 1) / ((2 eps_solv + 1) rc^3) and c_rf = 3 eps_solv / ((2 eps_solv + 1) rc),
    minimum image when isPBC."""

    coulomb = "rf"

    def __init__(self, r_cut, init_charges, epsilon_1=1.0, epsilon_solv=78.5, isPBC=True, topology_matrix=None,
                 precision="fp32", device=None) -> None:
        self.r_cut = r_cut
        self.krf = (1.0 / r_cut ** 3) * (epsilon_solv - 1) / (2.0 * epsilon_solv + 1)
        self.crf = (1.0 / r_cut) * 3.0 * epsilon_solv / (2.0 * epsilon_solv + 1)
        self.exp_solv = epsilon_solv
        self.ifPBC = isPBC
        self._setup(init_charges, topology_matrix, epsilon_1, isPBC, r_cut, eps_solv=epsilon_solv,
                    precision=precision, device=device)


class CoulombPMEForce(_CoulombBase):
    """Point-charge PME (inter.py:269-335): the ADMP energy with lmax 0, i.e. real-space
    erfc-screened rows with the topological exclusions, the reciprocal sum on the K1 x K2 x K3
    mesh (order-6 B-splines) and the self term."""

    coulomb = "pme"

    def __init__(self, r_cut: float, init_charges, kappa: float, K, pme_order: int = 6, topology_matrix=None,
                 precision="fp32", device=None):
        if pme_order != 6:
            raise ValueError("PME order other than 6 is not supported")
        self.r_cut = r_cut
        self.lmax = 0
        self.kappa = kappa
        self.K1, self.K2, self.K3 = int(K[0]), int(K[1]), int(K[2])
        self.pme_order = pme_order
        self._setup(init_charges, topology_matrix, 1.0, True, r_cut, kappa_nm=kappa, K=K, precision=precision,
                    device=device)
