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
