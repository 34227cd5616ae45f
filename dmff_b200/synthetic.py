"""Seeded synthetic inputs with the shapes of the ADMP benchmark workloads.

Water boxes: an m^3 lattice (m = ceil(n^(1/3)), spacing L/m; a seeded random subset of sites
when n < m^3), rigid waters (O-H 0.9572 A, H-O-H 104.52 deg) jittered by U(+-0.3 A) per axis
with a uniform random orientation, redrawn (seeded) while any intermolecular atom pair would be
closer than 1.7 A.  Without that rejection a 3.1 A lattice of randomly oriented waters has contacts
down to 0.8 A, where the polarizabilities of the benchmark (O 1.0, H 0.5 A^3) make the
induced-dipole matrix indefinite (a polarization catastrophe: the energy has no minimum in U).
Atom order per molecule is O, H1, H2.  Local frames follow
the water convention of the reference's examples: O is Bisector (z between O->H1 and O->H2, x
toward H2), H is ZThenX (z toward O, x toward the other H).  The covalent map holds O-H (1) and
H-H (2).  Per-type multipoles: charges O -0.8 / H +0.4, Cartesian dipoles ~ N(0, 0.1 e A) and
traceless quadrupoles ~ N(0, 0.1 e A^2) in the reference's internal Angstrom convention, turned
into harmonics with the reference's cart->harm matrices (dmff/admp/multipole.py:36-72).
"""
import math

import numpy as np

# dmff/admp/multipole.py:11-31
_RT3 = 1.73205080757
_INV_RT3 = 1.0 / _RT3
C1_C2H = np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0]], dtype=np.float64)
C2_C2H = np.array([
    [0, 0, 1, 0, 0, 0],
    [0, 0, 0, 0, 2 * _INV_RT3, 0],
    [0, 0, 0, 0, 0, 2 * _INV_RT3],
    [_INV_RT3, -_INV_RT3, 0, 0, 0, 0],
    [0, 0, 0, 2 * _INV_RT3, 0, 0],
], dtype=np.float64)

BISECTOR, ZTHENX = 1, 0


def cart2harm(theta):
    """Cartesian (c0, dX, dY, dZ, qXX, qYY, qZZ, qXY, qXZ, qYZ) -> 9 harmonic components."""
    theta = np.atleast_2d(np.asarray(theta, dtype=np.float64))
    out = np.zeros((theta.shape[0], 9))
    out[:, 0] = theta[:, 0]
    if theta.shape[1] >= 4:
        out[:, 1:4] = theta[:, 1:4] @ C1_C2H.T
    if theta.shape[1] >= 10:
        out[:, 4:9] = theta[:, 4:10] @ C2_C2H.T
    return out


def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


def _body():
    r, th = 0.9572, math.radians(104.52)
    return np.array([[0.0, 0.0, 0.0],
                     [r * math.sin(th / 2), 0.0, r * math.cos(th / 2)],
                     [-r * math.sin(th / 2), 0.0, r * math.cos(th / 2)]])


def water_positions(n_waters, L, rng, min_inter=1.7, max_tries=200):
    """Lattice centres + U(+-0.3 A) jitter + uniform random orientations.  Orientations are
    redrawn (same seeded stream) while any intermolecular atom pair is closer than ``min_inter``
    to an already placed molecule, so that no two waters overlap; a molecule that finds no such
    orientation in ``max_tries`` draws keeps its best one."""
    m = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    sites = np.array([(i, j, k) for i in range(m) for j in range(m) for k in range(m)], dtype=np.float64)
    if n_waters < m ** 3:
        sites = sites[np.sort(rng.choice(m ** 3, n_waters, replace=False))]
    centers = (sites + 0.5) * (L / m) + rng.uniform(-0.3, 0.3, size=(n_waters, 3))
    body = _body()
    R = _random_rotations(rng, n_waters)
    pos = centers[:, None, :] + np.einsum("nij,aj->nai", R, body)
    if min_inter is None or min_inter <= 0:
        return pos.reshape(-1, 3)
    # cell list over molecule centres (cell >= 6 A) to find nearby molecules
    nc = max(1, int(L // 6.0))
    cell = np.floor((centers % L) / (L / nc)).astype(int) % nc
    buckets = {}
    for k, c in enumerate(map(tuple, cell)):
        buckets.setdefault(c, []).append(k)
    placed = np.zeros(n_waters, dtype=bool)
    offs = [(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)] if nc >= 3 else None
    for k in range(n_waters):
        if offs is None:
            near = np.nonzero(placed)[0]
        else:
            c0 = cell[k]
            near = [q for o in offs for q in buckets.get(((c0[0] + o[0]) % nc, (c0[1] + o[1]) % nc, (c0[2] + o[2]) % nc), ())
                    if placed[q]]
            near = np.asarray(near, dtype=int)
        best, best_d = pos[k], -1.0
        for t in range(max_tries):
            cand = pos[k] if t == 0 else centers[k] + body @ _random_rotations(rng, 1)[0].T
            if len(near) == 0:
                best = cand
                break
            d = cand[:, None, None, :] - pos[near][None]
            d -= L * np.round(d / L)
            dmin = np.sqrt((d * d).sum(-1)).min()
            if dmin > best_d:
                best, best_d = cand, dmin
            if dmin >= min_inter:
                break
        pos[k] = best
        placed[k] = True
    return pos.reshape(-1, 3)


def water_topology(n_waters):
    n = 3 * n_waters
    o = np.arange(n_waters) * 3
    types = np.tile([0, 1, 1], n_waters)
    axis_types = np.tile([BISECTOR, ZTHENX, ZTHENX], n_waters).astype(np.int32)
    axis_indices = np.full((n, 3), -1, dtype=np.int32)
    axis_indices[o, 0], axis_indices[o, 1] = o + 1, o + 2
    axis_indices[o + 1, 0], axis_indices[o + 1, 1] = o, o + 2
    axis_indices[o + 2, 0], axis_indices[o + 2, 1] = o, o + 1
    cov = np.concatenate([np.stack([o, o + 1, np.ones_like(o)], 1), np.stack([o, o + 2, np.ones_like(o)], 1),
                          np.stack([o + 1, o + 2, 2 * np.ones_like(o)], 1)])
    cov = cov[np.lexsort((cov[:, 1], cov[:, 0]))].astype(np.int32)
    return types, axis_types, axis_indices, cov


def type_multipoles(rng, charges=(-0.8, 0.4), sd_dip=0.1, sd_quad=0.1):
    rows = []
    for q in charges:
        d = rng.normal(0.0, sd_dip, size=3)
        qxx, qyy, qxy, qxz, qyz = rng.normal(0.0, sd_quad, size=5)
        rows.append([q, d[0], d[1], d[2], qxx, qyy, -qxx - qyy, qxy, qxz, qyz])
    return cart2harm(np.array(rows))


def water_box(n_waters, L, seed, lmax=2, pol=False, rc=6.0, ethresh=5e-4, pol_O=1.0, pol_H=0.5, thole=0.33,
              min_inter=1.7):
    """System dict for an ADMP water box (positions / box in Angstrom)."""
    rng = np.random.default_rng(seed)
    pos = water_positions(n_waters, L, rng, min_inter=min_inter)
    types, axis_types, axis_indices, cov = water_topology(n_waters)
    Qt = type_multipoles(rng)
    if lmax < 2:
        Qt[:, 4:] = 0.0
    if lmax < 1:
        Qt[:, 1:4] = 0.0
    kappa = math.sqrt(-math.log(2 * ethresh)) / rc
    K = int(math.ceil(2 * kappa * L / 3 / ethresh ** 0.2))
    sysd = dict(
        n_atoms=3 * n_waters, pos=pos, box=np.eye(3) * L, types=types, axis_types=axis_types,
        axis_indices=axis_indices, cov_rows=cov, Q_type=Qt, Q_local=Qt[types], lmax=lmax, lpol=pol, rc=rc,
        ethresh=ethresh, kappa=kappa, K=(K, K, K),
        mscales=np.array([0.0, 0.0, 1.0, 1.0, 1.0, 1.0]),
        pscales=np.array([0.0, 0.0, 1.0, 1.0, 1.0, 1.0]),
        dscales=np.array([1.0, 1.0, 1.0, 1.0, 1.0, 1.0]),
    )
    if pol:
        sysd["pol"] = np.where(types == 0, pol_O, pol_H).astype(np.float64)
        sysd["thole"] = np.full(3 * n_waters, thole, dtype=np.float64)
    return sysd


def workload(name):
    """The named benchmark workloads."""
    if name == "c0":
        return water_box(216, 18.6, seed=0, lmax=2, pol=False, rc=6.0)
    if name == "c1":
        return water_box(4096, 49.7, seed=1, lmax=2, pol=True, rc=8.0)
    if name == "c2":
        return water_box(2048, 40.0, seed=2, lmax=2, pol=True, rc=8.0)
    raise KeyError(name)


def serving_sizes(n_requests=2000, seed=3, lo=100, hi=10000):
    """Log-uniform molecule counts of the serving stream."""
    rng = np.random.default_rng(seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size=n_requests)).astype(int)


def pairs_nbond(pairs, cov_rows, n_atoms):
    """Fill the third column of (i, j) rows from sparse covalent rows (i < j, nbond)."""
    key = cov_rows[:, 0].astype(np.int64) * n_atoms + cov_rows[:, 1]
    order = np.argsort(key)
    key, nb = key[order], cov_rows[order, 2]
    q = pairs[:, 0].astype(np.int64) * n_atoms + pairs[:, 1]
    pos = np.clip(np.searchsorted(key, q), 0, max(len(key) - 1, 0))
    out = np.zeros(len(pairs), dtype=np.int64)
    if len(key):
        hit = key[pos] == q
        out[hit] = nb[pos[hit]]
    return out


def disp_params(n_waters, seed=2, b_per_A=3.5):
    """Dispersion / Tang-Toennies parameters of the differentiation workload: per-type C6, C8, C10
    log-normal (sigma 0.5) around 1e-3, 1e-4, 1e-5 kJ/mol nm^n; TT b = 3.5 / A (B = 35 / nm);
    A and Q of the reference's water force field (examples/water_fullpol/forcefield.xml)."""
    rng = np.random.default_rng(seed)
    C = np.stack([np.exp(rng.normal(np.log(m), 0.5, size=2)) for m in (1e-3, 1e-4, 1e-5)], axis=1)  # [type, 3]
    types = np.tile([0, 1, 1], n_waters)
    Ct = C[types]
    c_list = np.sqrt(Ct * np.array([1e6, 1e8, 1e10]))
    A = np.array([1203470.743, 83.2283563])[types] / 2625.5
    B = np.full(len(types), b_per_A * 10.0 * 0.0529177249)
    Q = np.array([-0.741706, 0.370853])[types]
    return dict(C_type=C, c_list=c_list, a=A, b=B, q=Q, mscales=np.array([0.0, 0.0, 0.0, 1.0, 1.0, 1.0]))


def _chain_walk(rng, n_beads, start, bond=1.53, ang=(100.0, 120.0), min_dist=3.0, max_tries=200):
    """Random-walk chain: bond length ``bond``, bond angles U(ang), uniform dihedrals; a new bead is
    redrawn while it sits within ``min_dist`` of a bead three or more places back."""
    pos = [np.asarray(start, dtype=np.float64)]
    d = rng.normal(size=3)
    pos.append(pos[0] + bond * d / np.linalg.norm(d))
    for k in range(2, n_beads):
        best, best_d = None, -1.0
        for _ in range(max_tries):
            a, b = pos[k - 1], pos[k - 2]
            u = (b - a) / np.linalg.norm(b - a)
            th = math.radians(rng.uniform(*ang))
            ph = rng.uniform(0, 2 * math.pi)
            t = rng.normal(size=3)
            t -= t.dot(u) * u
            t /= np.linalg.norm(t)
            w = np.cross(u, t)
            v = math.cos(th) * u + math.sin(th) * (math.cos(ph) * t + math.sin(ph) * w)
            p = a + bond * v
            dmin = min([np.linalg.norm(p - q) for q in pos[:k - 2]], default=1e9)
            if dmin > best_d:
                best, best_d = p, dmin
            if dmin >= min_dist:
                break
        pos.append(best)
    return np.array(pos)


def polymer_water_box(n_chains, n_beads, n_waters, L, seed=4, rc=10.0, ethresh=1e-5):
    """Classical polymer + water system (positions / box in Angstrom, kJ/mol).

    ``n_chains`` linear chains of ``n_beads`` beads (random walk: bonds 1.53 A, angles U(100, 120) deg,
    redrawn within 3 A of earlier beads), bead charges N(0, 0.3 e) shifted to zero net charge per
    chain, one LJ type per chain position with sigma U(3.0, 3.8) A and eps U(0.2, 0.8) kJ/mol;
    harmonic bonds (k 2000 kJ/mol/A^2, r0 U(1.48, 1.58) A), angles (k 400 kJ/mol/rad^2, theta0 110 deg) and
    3-term periodic torsions (n = 1, 2, 3; k U(0.5, 2) kJ/mol, phase 0 or pi).  Waters: point
    charges O -0.834 / H +0.417 (O-H 0.9572 A, H-O-H 104.52 deg) on a seeded subset of an m^3
    lattice with random orientations, O LJ sigma 3.15061 A / eps 0.6364 kJ/mol, H none.  Atom order:
    chains first, then waters (O, H1, H2).  Covalent map from the bonds (chains: path lengths up to
    6; waters: O-H 1, H-H 2).  Coulomb PME kappa / K from ethresh by the reference's 'openmm'
    formula; scales 1-4: LJ 0.5, Coulomb 0.8333 (0 for 1-2, 1-3)."""
    from .api.topology import covalent_rows
    rng = np.random.default_rng(seed)
    nb = n_chains * n_beads
    chains = [_chain_walk(rng, n_beads, rng.uniform(0, L, size=3)) for _ in range(n_chains)]
    wpos = water_positions(n_waters, L, rng, min_inter=None) if n_waters else np.zeros((0, 3))
    pos = np.concatenate(chains + [wpos]) if n_chains else wpos
    n = nb + 3 * n_waters
    q = []
    for _ in range(n_chains):
        c = rng.normal(0.0, 0.3, size=n_beads)
        q.append(c - c.mean())
    q = np.concatenate(q + [np.tile([-0.834, 0.417, 0.417], n_waters)])
    sig_b = rng.uniform(3.0, 3.8, size=n_beads)
    eps_b = rng.uniform(0.2, 0.8, size=n_beads)
    sig = np.concatenate([sig_b, [3.15061, 0.0]])
    eps = np.concatenate([eps_b, [0.6364, 0.0]])
    types = np.concatenate([np.tile(np.arange(n_beads), n_chains),
                            np.tile([n_beads, n_beads + 1, n_beads + 1], n_waters)]).astype(np.int32)
    bonds, angles, tors = [], [], []
    for c in range(n_chains):
        o = c * n_beads
        bonds += [(o + k, o + k + 1) for k in range(n_beads - 1)]
        angles += [(o + k, o + k + 1, o + k + 2) for k in range(n_beads - 2)]
        tors += [(o + k, o + k + 1, o + k + 2, o + k + 3) for k in range(n_beads - 3)]
    wb = []
    for w in range(n_waters):
        o = nb + 3 * w
        wb += [(o, o + 1), (o, o + 2)]
    bonds = np.asarray(bonds, dtype=np.int32).reshape(-1, 2)
    angles = np.asarray(angles, dtype=np.int32).reshape(-1, 3)
    tors = np.asarray(tors, dtype=np.int32).reshape(-1, 4)
    cov = covalent_rows(n, np.concatenate([bonds, np.asarray(wb, dtype=np.int32).reshape(-1, 2)]))
    bond_prm = np.stack([np.full(len(bonds), 2000.0), rng.uniform(1.48, 1.58, size=len(bonds))], axis=1)
    angle_prm = np.tile([400.0, math.radians(110.0)], (len(angles), 1))
    t_idx = np.repeat(tors, 3, axis=0)
    t_prm = np.stack([rng.uniform(0.5, 2.0, size=len(t_idx)), rng.choice([0.0, math.pi], size=len(t_idx)),
                      np.tile([1.0, 2.0, 3.0], len(tors))], axis=1)
    kappa = math.sqrt(-math.log(2 * ethresh)) / rc
    K = int(math.ceil(2 * kappa * L / 3 / ethresh ** 0.2))
    return dict(n_atoms=n, pos=pos, box=np.eye(3) * L, charges=q, types=types, sigma=sig, epsilon=eps,
                sigma_tt=(sig[:, None] + sig[None, :]) * 0.5, eps_tt=np.sqrt(eps[:, None] * eps[None, :] + 1e-32),
                cov_rows=cov.astype(np.int32), bonds=bonds, bond_prm=bond_prm, angles=angles, angle_prm=angle_prm,
                torsions=t_idx, torsion_prm=t_prm, rc=rc, ethresh=ethresh, kappa=kappa, K=(K, K, K),
                mscales_coul=np.array([0.0, 0.0, 0.8333333333333334, 1.0, 1.0, 1.0]),
                mscales_lj=np.array([0.0, 0.0, 0.5, 1.0, 1.0, 1.0]))


def water_positions_fast(n_waters, L, rng, min_inter=1.7, max_rounds=400):
    """Vectorised variant of ``water_positions`` for streams of many boxes: lattice centres with
    U(+-0.3 A) jitter and uniform random orientations; in rounds, one molecule of every pair with
    an intermolecular atom contact below ``min_inter`` (periodic k-d tree query; the later one in
    even rounds, the earlier one in odd rounds) gets a new jitter and orientation.  After 50 rounds
    a molecule still in contact also moves to the free lattice site with the fewest occupied
    neighbours when the box has one (a
    seeded subset of the m^3 sites is used when n < m^3), and from round 100 on the re-drawn
    molecules sit on their sites without jitter.  Raises when contacts remain after
    ``max_rounds`` rounds, so that no box with overlapping molecules is ever returned."""
    from scipy.spatial import cKDTree
    m = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    all_sites = np.array([(i, j, k) for i in range(m) for j in range(m) for k in range(m)], dtype=np.float64)
    used = np.arange(m ** 3)
    if n_waters < m ** 3:
        used = np.sort(rng.choice(m ** 3, n_waters, replace=False))
    free = np.setdiff1d(np.arange(m ** 3), used)
    base = (all_sites[used] + 0.5) * (L / m)
    centers = base + rng.uniform(-0.3, 0.3, size=(n_waters, 3))
    body = _body()
    R = _random_rotations(rng, n_waters)
    pos = centers[:, None, :] + np.einsum("nij,aj->nai", R, body)
    for rnd in range(max_rounds):
        flat = pos.reshape(-1, 3) % L
        pr = cKDTree(flat, boxsize=L).query_pairs(min_inter, output_type="ndarray")
        mol = pr // 3
        mol = mol[mol[:, 0] != mol[:, 1]]
        if len(mol) == 0:
            return pos.reshape(-1, 3)
        bad = np.unique(mol.max(axis=1) if rnd % 2 == 0 else mol.min(axis=1))
        if rnd >= 50 and len(free):
            # move to the free sites with the fewest occupied face neighbours (ties at random)
            occ = np.zeros(m ** 3, dtype=bool)
            occ[used] = True
            for mv in rng.permutation(bad)[: len(free)]:
                fs = all_sites[free].astype(np.int64)
                cnt = np.zeros(len(free), dtype=np.int64)
                for ax in range(3):
                    for sh in (-1, 1):
                        nb_ = fs.copy()
                        nb_[:, ax] = (nb_[:, ax] + sh) % m
                        cnt += occ[(nb_[:, 0] * m + nb_[:, 1]) * m + nb_[:, 2]]
                best = np.flatnonzero(cnt == cnt.min())
                pick = best[rng.integers(len(best))]
                occ[used[mv]] = False
                occ[free[pick]] = True
                used[mv], free[pick] = free[pick], used[mv]
                base[mv] = (all_sites[used[mv]] + 0.5) * (L / m)
        jitter = 0.3 if rnd < 100 else 0.0  # late rounds: the re-drawn molecules sit on their sites
        centers[bad] = base[bad] + rng.uniform(-jitter, jitter, size=(len(bad), 3))
        pos[bad] = centers[bad][:, None, :] + np.einsum("nij,aj->nai", _random_rotations(rng, len(bad)), body)
    raise RuntimeError(f"water_positions_fast: contacts below {min_inter} A remain after {max_rounds} rounds "
                       f"({n_waters} waters, L = {L:.2f} A)")


def serving_system(n_waters, index, density=0.0334, rc=8.0, ethresh=5e-4, lmax=2, seed=3):
    """One request of the serving stream: a polarizable water box of ``n_waters`` molecules at
    ``density`` molecules/A^3 (L = (n / density)^(1/3)), built as ``water_box`` (per-type multipoles
    of seed ``seed``, O 1.0 / H 0.5 A^3, Thole 0.33) with positions from ``water_positions_fast``
    seeded by (seed, index).  Boxes narrower than 2 rc use rc' = 0.5 L (1 - 1e-6), with kappa and K
    re-derived from rc' ('openmm' formula)."""
    L = (n_waters / density) ** (1.0 / 3.0)
    rcx = min(rc, 0.5 * L * (1 - 1e-6))
    rng_t = np.random.default_rng(seed)
    Qt = type_multipoles(rng_t)
    if lmax < 2:
        Qt[:, 4:] = 0.0
    if lmax < 1:
        Qt[:, 1:4] = 0.0
    rng = np.random.default_rng([seed, int(index)])
    pos = water_positions_fast(n_waters, L, rng)
    types, axis_types, axis_indices, cov = water_topology(n_waters)
    kappa = math.sqrt(-math.log(2 * ethresh)) / rcx
    K = int(math.ceil(2 * kappa * L / 3 / ethresh ** 0.2))
    return dict(n_atoms=3 * n_waters, pos=pos, box=np.eye(3) * L, types=types, axis_types=axis_types,
                axis_indices=axis_indices, cov_rows=cov, Q_type=Qt, Q_local=Qt[types], lmax=lmax, lpol=True, rc=rcx,
                ethresh=ethresh, kappa=kappa, K=(K, K, K), mscales=np.array([0.0, 0.0, 1.0, 1.0, 1.0, 1.0]),
                pscales=np.array([0.0, 0.0, 1.0, 1.0, 1.0, 1.0]), dscales=np.ones(6),
                pol=np.where(types == 0, 1.0, 0.5).astype(np.float64), thole=np.full(3 * n_waters, 0.33))


def serving_arrivals(n_requests, rate, seed=33):
    """Poisson arrival times (s) of the serving stream at ``rate`` requests/s."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n_requests))
