"""ORACLE — test infrastructure only, never the product path.

A float64 PyTorch (CPU) restatement of the reference's charge-equilibration potential,
ADMPQeqForce (dmff/admp/qeq.py) and its generator (dmff/generators/qeq.py), for checking the
GPU implementation in ``dmff_b200.admp.qeq``.  Only ``tests/`` may import this module.

The reference finds the charges q and Lagrange multipliers lambda where the gradient of
E_full(q, lambda) vanishes with a MINPACK root finder (jaxopt.ScipyRootFinding 'hybr', tol
1e-10, qeq.py:375-381), then evaluates E_full there with the solution held fixed
(stop_gradient, qeq.py:395).  Every term of E_full is a polynomial of degree two in
b = (q, lambda), so its gradient is affine: G(b) = H b + G(0).  This oracle builds H column by
column from exact gradient differences, H e_k = G(e_k) - G(0) (autograd gradients), and solves
H b = -G(0) directly — the same stationary point by a different method.  Parity is pinned by
the reference's own golden energies (tests/test_admp/test_qeq.py: -37.84692763 for qeq.xml /
qeq.pdb, 4817.295171 for qeq2.xml / qeq2.pdb).
"""
import math

import numpy as np
import torch

from oracle.admp_ref import DIELECTRIC, DTYPE, Ck_1, energy_pme, generate_pme_recip, pair_buffer_scales, \
    regularize_pairs


def padding_consts(const_list, max_idx):
    """qeq.py:57-63: groups padded to a rectangle with the index n."""
    width = max([len(c) for c in const_list]) if const_list else 0
    out = np.zeros((len(const_list), width), dtype=np.int64) + max_idx
    for g, c in enumerate(const_list):
        out[g, :len(c)] = c
    return torch.as_tensor(out)


def group_sum(v, groups):
    """qeq.py:42-54: sum of v over each group, padding indices (>= n) masked."""
    n = v.shape[0]
    mask = (groups < n).to(DTYPE)
    idx = torch.clamp(groups, max=n - 1)
    return (v[idx] * mask).sum(dim=1)


def E_constQ(q, lagmt, groups, const_vals):
    """qeq.py:66-69."""
    return torch.sum((group_sum(q, groups) - const_vals) * lagmt)


def E_constP(q, lagmt, groups, const_vals):
    """qeq.py:72-75."""
    return torch.sum(group_sum(q, groups) * const_vals)


def _eta_pair(s, ds):
    """qeq.py:193-201 (eta_piecewise): erfc(ds / s) where s > 1e-4, else 0."""
    keep = s > 1e-4
    return torch.where(keep, torch.erfc(ds / torch.where(keep, s, torch.ones_like(s))), torch.zeros_like(s))


def _eta_inv(eta):
    """qeq.py:206-214 (etainv_piecewise)."""
    keep = eta > 1e-4
    return torch.where(keep, 1.0 / torch.where(keep, eta, torch.ones_like(eta)), torch.zeros_like(eta))


def E_sr2(pos, box, pairs, q, eta, ds, buffer_scales):
    """qeq.py:85-95 (DampMod 2)."""
    s = torch.sqrt(2 * (eta[pairs[:, 0]] ** 2 + eta[pairs[:, 1]] ** 2))
    pre_pair = -_eta_pair(s, ds) * DIELECTRIC
    pre_self = _eta_inv(eta) / math.sqrt(2 * math.pi) * DIELECTRIC
    e_pair = pre_pair * q[pairs[:, 0]] * q[pairs[:, 1]] / ds * buffer_scales
    e_pair = torch.where(buffer_scales < 1e-4, torch.zeros_like(e_pair), e_pair)
    return torch.sum(e_pair) + torch.sum(pre_self * q * q)


def E_sr3(pos, box, pairs, q, eta, ds, buffer_scales):
    """qeq.py:98-112 (DampMod 3)."""
    s = torch.sqrt(eta[pairs[:, 0]] ** 2 + eta[pairs[:, 1]] ** 2 + 1e-64)
    pre_pair = -_eta_pair(s, ds) * DIELECTRIC
    pre_self = _eta_inv(eta) / math.sqrt(2 * math.pi) * DIELECTRIC
    e_pair = pre_pair * q[pairs[:, 0]] * q[pairs[:, 1]] / ds
    e_pair = torch.where(buffer_scales < 1e-4, torch.zeros_like(e_pair), e_pair)
    return torch.sum(e_pair) + torch.sum(pre_self * q * q)


def E_site2(chi, J, q):
    """qeq.py:120-123."""
    return torch.sum((chi * q + 0.5 * J * q ** 2) * 96.4869)


def E_site3(chi, J, q):
    """qeq.py:126-129."""
    return torch.sum(chi * q * 4.184 + J * q ** 2 * DIELECTRIC * 2 * math.pi)


def E_corr(pos, box, q, kappa, neutral_flag=True):
    """qeq.py:132-152 (slab correction).  ``box[3]`` of the reference indexes past the 3 x 3 box;
    JAX clamps the index, so the row used is box[2]."""
    V = torch.linalg.det(box)
    pre_corr = 2 * math.pi / V * DIELECTRIC
    Mz = torch.sum(q * pos[:, 2])
    Q_tot = torch.sum(q)
    Lz = torch.linalg.norm(box[2])
    e = pre_corr * (Mz ** 2 - Q_tot * torch.sum(q * pos[:, 2] ** 2) - Q_tot ** 2 * Lz ** 2 / 12)
    if neutral_flag:
        e = e + (-math.pi / (2 * V * kappa ** 2) * DIELECTRIC) * Q_tot ** 2
    return e


def ds_pairs(positions, box, pairs, pbc_flag):
    """qeq.py:170-182."""
    dpos = positions[pairs[:, 0]] - positions[pairs[:, 1]]
    if pbc_flag:
        f = dpos @ torch.linalg.inv(box)
        f = f - torch.floor(f + 0.5)
        dpos = f @ box
    return torch.linalg.norm(dpos + 1e-64, dim=1)


class ADMPQeqForce:
    """qeq.py:217-405 with the direct solve described in the module docstring."""

    def __init__(self, init_q, r_cut, kappa, K, damp_mod=3, const_list=(), const_vals=(), neutral_flag=True,
                 slab_flag=False, constQ=True, pbc_flag=True, has_aux=False):
        const_vals = np.asarray(const_vals, dtype=np.float64)
        if neutral_flag and len(const_vals):
            const_vals = const_vals - np.sum(const_vals) / len(const_vals)
        self.const_vals = torch.as_tensor(const_vals, dtype=DTYPE)
        n = len(init_q)
        self.groups = padding_consts(list(const_list), n)
        self.init_q = torch.as_tensor(np.asarray(init_q, dtype=np.float64))
        self.n_const = len(const_list)
        self.damp_mod = damp_mod
        self.constQ = constQ
        self.neutral_flag = neutral_flag
        self.slab_flag = slab_flag
        self.pbc_flag = pbc_flag
        self.e_constraint = E_constQ if constQ else E_constP
        self.e_sr = {1: lambda *a: 0.0, 2: E_sr2, 3: E_sr3}[damp_mod]
        self.e_site = {1: lambda *a: 0.0, 2: E_site2, 3: E_site3}[damp_mod]
        self.kappa = kappa if pbc_flag else 0.0
        self._K = tuple(int(k) for k in K)
        if pbc_flag:
            recip = generate_pme_recip(Ck_1, kappa / 10, False, 6, K[0], K[1], K[2], 0)

            def coul(positions, box, pairs, q, mscales):
                return energy_pme(positions * 10, box * 10, pairs, q.reshape(-1, 1), None, None, None, mscales, None,
                                  None, None, None, recip, kappa / 10, K[0], K[1], K[2], 0, False)
        else:
            def coul(positions, box, pairs, q, mscales):
                rp = regularize_pairs(pairs[:, :2])
                mask = pair_buffer_scales(pairs[:, :2])
                ms = mscales[pairs[:, 2] - 1]
                dr = positions[rp[:, 0]] - positions[rp[:, 1]]
                d = torch.linalg.norm(dr + 1e-64, dim=1)
                return torch.sum(q[rp[:, 0]] * q[rp[:, 1]] * ms * DIELECTRIC * 0.1 / d * mask)
        self.coul = coul

    def E_full(self, q, lagmt, chi, J, pos, box, pairs, eta, ds, buffer_scales, mscales):
        """qeq.py:310-322."""
        e = self.e_constraint(q, lagmt, self.groups, self.const_vals)
        e = e + self.e_sr(pos * 10, box * 10, pairs, q, eta, ds * 10, buffer_scales)
        e = e + self.e_site(chi, J, q)
        e = e + self.coul(pos, box, pairs, q, mscales)
        if self.slab_flag:
            e = e + E_corr(pos * 10, box * 10, q, self.kappa / 10, self.neutral_flag)
        return e

    def solve(self, positions, box, pairs, mscales, eta, chi, J):
        """The stationary point b* = (q*, lambda*) of E_full."""
        pairs = torch.as_tensor(np.asarray(pairs)).long()
        n = self.init_q.shape[0]
        # rows with i < j < n: the others carry zero buffer scale in every term (padding rows
        # index n; the reference's gathers clamp them, its masks drop them)
        pairs = pairs[(pairs[:, 0] < pairs[:, 1]) & (pairs[:, 1] < n)]
        ds = ds_pairs(positions, box, pairs, self.pbc_flag)
        bs = pair_buffer_scales(pairs[:, :2]).to(DTYPE)
        m = self.n_const
        ms = torch.as_tensor(np.asarray(mscales, dtype=np.float64))

        def grad_at(b):
            with torch.enable_grad():
                b = b.clone().requires_grad_(True)
                e = self.E_full(b[:n], b[n:], chi, J, positions, box, pairs, eta, ds, bs, ms)
                (g,) = torch.autograd.grad(e, b)
            return g.detach()

        g0 = grad_at(torch.zeros(n + m, dtype=DTYPE))
        H = torch.zeros((n + m, n + m), dtype=DTYPE)
        for k in range(n + m):
            ek = torch.zeros(n + m, dtype=DTYPE)
            ek[k] = 1.0
            H[:, k] = grad_at(ek) - g0
        H = 0.5 * (H + H.T)
        # E_constP leaves lambda out of E_full: its block is zero; any lambda solves it
        free = torch.ones(n + m, dtype=torch.bool)
        if self.e_constraint is E_constP:
            free[n:] = False
        b = torch.zeros(n + m, dtype=DTYPE)
        idx = torch.nonzero(free).reshape(-1)
        b[idx] = torch.linalg.solve(H[idx][:, idx], -g0[idx])
        return b[:n], b[n:], ds, bs, ms, pairs

    def get_energy(self, positions, box, pairs, mscales, eta, chi, J):
        """Energy at the stationary point (kJ/mol); differentiable in positions, box and the
        parameters with the solution held fixed (the reference's stop_gradient).  Returns
        (energy, q*, lambda*)."""
        with torch.no_grad():
            q, lam, ds, bs, ms, pr = self.solve(positions.detach(), box.detach(), pairs, mscales, eta.detach(),
                                                chi.detach(), J.detach())
        ds = ds_pairs(positions, box, pr, self.pbc_flag)
        e = self.E_full(q, lam, chi, J, positions, box, pr, eta, ds, bs, ms)
        return e, q, lam
