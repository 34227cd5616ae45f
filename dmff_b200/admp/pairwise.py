"""Generic pairwise interactions with the names of dmff/admp/pairwise.py.

``generate_pairwise_interaction(kernel, static_args)`` returns
``pair_int(positions, box, pairs, mScales, *atomic_params)``: the sum over pair rows of
``kernel(r, m, p1_i, p1_j, p2_i, p2_j, ...) * [i < j]`` (pairwise.py:47-95).  ``r`` is the
minimum-image distance and ``m = mScales[nbond - 1]``, nbond read from the rows' last column.

The reference's built-in kernels (``TT_damping_qq_c6_kernel``, ``TT_damping_qq_kernel``,
``slater_disp_damping_kernel``, ``slater_sr_kernel``, pairwise.py:100-171) run on the GPU in the
engine's short-range pair kernel (``PairwiseEngine``, dmffb_pairwise_*): closed-form energies,
forces, box gradient and per-atom parameter adjoints, autograd through ``_PairwiseEnergy`` (double
backward by central differences of those analytic first derivatives).  Any other elementwise torch
function of those tensors runs vectorised over all rows on the rows' device, differentiated by
autograd.
"""
import numpy as np
import torch

from ..utils import pair_buffer_scales, regularize_pairs
from .spatial import pbc_shift

DIELECTRIC = 1389.35455846


def distribute_scalar(params, index):
    """params[index] (pairwise.py:22-41)."""
    return params[index]


distribute_v3 = distribute_multipoles = distribute_dispcoeff = distribute_scalar


def distribute_matrix(multipoles, index1, index2):
    """multipoles[index1, index2] (pairwise.py:44-45)."""
    return multipoles[index1, index2]


def generate_pairwise_interaction(pair_int_kernel, static_args, precision="fp64"):
    """The pair-sum calculator for ``pair_int_kernel`` (pairwise.py:47-95); ``static_args`` is
    kept for the reference's signature.  Built-in kernels evaluate on the GPU in ``precision``."""
    kind = _builtin_kind(pair_int_kernel)
    if kind is not None:
        return _cuda_pair_int(kind, precision)

    def pair_int(positions, box, pairs, mScales, *atomic_params):
        pos = torch.as_tensor(positions, dtype=torch.float64)
        dev = pos.device
        rows = (pairs if torch.is_tensor(pairs) else torch.as_tensor(pairs)).to(dev).long()
        ij = regularize_pairs(rows[:, :2])
        buf = pair_buffer_scales(rows[:, :2]).to(torch.float64)
        m = torch.as_tensor(mScales, dtype=torch.float64).to(dev)[rows[:, -1] - 1] * buf
        b = torch.as_tensor(box, dtype=torch.float64).to(dev)
        dr = pbc_shift(pos[ij[:, 0]] - pos[ij[:, 1]], b, torch.linalg.inv(b))
        r = torch.linalg.norm(dr, dim=1)
        per_pair = []
        for p in atomic_params:
            p = torch.as_tensor(p).to(dev)
            per_pair += [p[ij[:, 0]], p[ij[:, 1]]]
        return torch.sum(pair_int_kernel(r, m, *per_pair) * buf)

    return pair_int


def TT_damping_qq_c6_kernel(dr, m, ai, aj, bi, bj, qi, qj, ci, cj):
    """Tang–Toennies short range with charge penetration and damped C6 (pairwise.py:100-117):
    2625.5 A e^{-br} - 2625.5 e^{-br} (1 + br) q / r + f_6(br) c / dr^6, with
    A = sqrt(a_i a_j), b = sqrt(b_i b_j), q = q_i q_j, c = c_i c_j, r = dr in bohr and
    f_6 the sixth-order damping sum; times m."""
    a = torch.sqrt(ai * aj)
    b = torch.sqrt(bi * bj)
    r = dr * 1.889726878
    br = b * r
    e = torch.exp(-br)
    f6 = 1 + br + br ** 2 / 2 + br ** 3 / 6 + br ** 4 / 24 + br ** 5 / 120 + br ** 6 / 720
    return (2625.5 * a * e - 2625.5 * e * (1 + br) * qi * qj / r + e * f6 * ci * cj / dr ** 6) * m


def TT_damping_qq_kernel(dr, m, bi, bj, qi, qj):
    """Charge-penetration term only (pairwise.py:121-128): -DIELECTRIC e^{-br} (1 + br) q / dr,
    b = sqrt(b_i b_j), r = dr; times m."""
    b = torch.sqrt(bi * bj)
    br = b * dr
    return -DIELECTRIC * torch.exp(-br) * (1 + br) * qi * qj / dr * m


def slater_disp_damping_kernel(dr, m, bi, bj, c6i, c6j, c8i, c8j, c10i, c10j):
    """Slater-ISA damping of C6/C8/C10 dispersion (pairwise.py:131-156): sum_n f_n(x) c_n / r^n with
    f_n = e^-x sum_{k<=n} x^k / k!, x = br - (2 (br)^2 + 3 br) / ((br)^2 + 3 br + 3),
    b = sqrt(b_i b_j), c_n = c_n,i c_n,j; times m."""
    b = torch.sqrt(bi * bj)
    br = b * dr
    x = br - (2 * br * br + 3 * br) / (br * br + 3 * br + 3)
    s6 = 1 + x + x ** 2 / 2 + x ** 3 / 6 + x ** 4 / 24 + x ** 5 / 120 + x ** 6 / 720
    s8 = s6 + x ** 7 / 5040 + x ** 8 / 40320
    s10 = s8 + x ** 9 / 362880 + x ** 10 / 3628800
    e = torch.exp(-x)
    return (e * s6 * c6i * c6j / dr ** 6 + e * s8 * c8i * c8j / dr ** 8 + e * s10 * c10i * c10j / dr ** 10) * m


def slater_sr_kernel(dr, m, ai, aj, bi, bj):
    """Slater-ISA short range (pairwise.py:159-171): a_i a_j ((br)^2 / 3 + br + 1) e^-br,
    b = sqrt(b_i b_j); times m."""
    b = torch.sqrt(bi * bj)
    br = b * dr
    return ai * aj * (br * br / 3 + br + 1) * torch.exp(-br) * m


# ----------------------------------------------------------------------------- CUDA path
def _builtin_kind(kernel):
    from .. import _lib as L
    return {TT_damping_qq_kernel: L.DMFFB_SR_TT_QQ, slater_disp_damping_kernel: L.DMFFB_SR_SLATER_DISP,
            slater_sr_kernel: L.DMFFB_SR_SLATER, TT_damping_qq_c6_kernel: L.DMFFB_SR_TT_QQ_C6}.get(kernel)


_ENGINES = {}


def _engine_for(kind, n, mscales, sign, precision, device):
    from ..engine import PairwiseEngine
    key = (kind, n, tuple(float(x) for x in mscales), float(sign), precision, str(device))
    eng = _ENGINES.get(key)
    if eng is None:
        # the pair rows are always given here; rc only sizes the unused internal list
        eng = PairwiseEngine(n, kind, rc=1.0, mscales=mscales, sign=sign, precision=precision, device=device)
        _ENGINES[key] = eng
    return eng


def _rows3(pairs, n, device):
    rows = pairs if torch.is_tensor(pairs) else torch.as_tensor(np.asarray(pairs))
    rows = rows.to(device=device, dtype=torch.int64)
    if rows.dim() != 2 or rows.shape[0] == 0:
        return torch.zeros((0, 3), dtype=torch.int32, device=device)
    nb = rows[:, -1] if rows.shape[1] > 2 else torch.zeros_like(rows[:, 0])
    return torch.stack([rows[:, 0], rows[:, 1], nb], dim=1).to(torch.int32).contiguous()


def _cuda_pair_int(kind, precision, sign=1.0):
    def pair_int(positions, box, pairs, mScales, *atomic_params):
        if not torch.cuda.is_available():
            raise RuntimeError("the built-in pairwise kernels run on the GPU engine; no CUDA device is available")
        pos = torch.as_tensor(positions, dtype=torch.float64)
        boxt = torch.as_tensor(box, dtype=torch.float64)
        n = pos.shape[0]
        ms = [float(x) for x in torch.as_tensor(mScales).detach().cpu().reshape(-1)]
        dev = torch.device("cuda", torch.cuda.current_device()) if not pos.is_cuda else pos.device
        eng = _engine_for(kind, n, ms, sign, precision, dev)
        rows = _rows3(pairs, n, dev)
        params = [torch.as_tensor(p, dtype=torch.float64) for p in atomic_params]
        return _PairwiseEnergy.apply(pos, boxt, rows, {"eng": eng, "kind": kind, "ms": ms, "sign": sign,
                                                       "precision": precision}, *params)

    return pair_int


def _pairwise_first(eng, pos, box, rows, params, want_p):
    """(energy, [dE/dpos, dE/dbox, dE/dp_1, ...]) of one engine evaluation."""
    eng.set_params(torch.stack([p.detach().to(torch.float64).reshape(-1) for p in params]))
    eng.set_param_grads(want_p)
    res, F = eng.compute(pos.detach().to(device=eng.device, dtype=torch.float64).contiguous(), box.detach(), rows)
    first = [-F.clone(), torch.tensor(list(res.box_grad), dtype=torch.float64).reshape(3, 3)]
    if want_p:
        pg = eng.param_grads()
        first += [pg[k].clone() for k in range(eng.nparam)]
    else:
        first += [None] * eng.nparam
    return res, first


class _PairwiseEnergy(torch.autograd.Function):
    """E(positions, box, per-atom parameters) of a built-in short-range kernel on the GPU engine;
    the first derivatives come out of ``_PairwiseFirstDerivs`` (differentiable in turn)."""

    @staticmethod
    def forward(ctx, positions, box, rows, cfg, *params):
        want_p = any(ctx.needs_input_grad[4:])
        res, first = _pairwise_first(cfg["eng"], positions, box, rows, params, want_p)
        ctx.payload = {"cfg": cfg, "rows": rows, "first": first}
        ctx.save_for_backward(positions, box, *params)
        return torch.tensor(res.energy, dtype=torch.float64, device=positions.device)

    @staticmethod
    def backward(ctx, g):
        saved = ctx.saved_tensors
        d = _PairwiseFirstDerivs.apply(ctx.payload, *saved)
        out = [None if t is None else t * g.to(t.device) for t in d]
        for k in range(2, len(out)):
            if not ctx.needs_input_grad[2 + k]:
                out[k] = None
        return (out[0], out[1], None, None, *out[2:])


class _PairwiseFirstDerivs(torch.autograd.Function):
    @staticmethod
    def forward(ctx, payload, positions, box, *params):
        ctx.payload = payload
        ctx.save_for_backward(positions, box, *params)
        like = (positions, box) + params
        return tuple(torch.zeros_like(t, dtype=torch.float64) if v is None else v.to(t.device).reshape(t.shape).clone()
                     for v, t in zip(payload["first"], like))

    @staticmethod
    def backward(ctx, *cot):
        from .._hvp import central_hvp
        saved = ctx.saved_tensors
        p = ctx.payload
        cfg = p["cfg"]
        eng = _engine_for(cfg["kind"], saved[0].shape[0], cfg["ms"], cfg["sign"], "fp64", cfg["eng"].device)

        def grad_at(z):
            _, first = _pairwise_first(eng, z[0], z[1], p["rows"], z[2:], True)
            return [first[0].to(z[0].device), first[1].to(z[1].device)] + [
                v.to(t.device).reshape(t.shape) for v, t in zip(first[2:], z[2:])]

        scales = [1.0, 1.0] + [max(float(t.detach().abs().max()), 1e-12) for t in saved[2:]]
        hv, _ = central_hvp(grad_at, [t.detach() for t in saved], [None if c is None else c.detach() for c in cot],
                            scales)
        return (None, *hv)
