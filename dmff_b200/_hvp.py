"""Directional derivatives of first-derivative maps, for the second-order (double-backward) passes
of the energies whose first derivatives the engine computes analytically and that involve no
implicit solve (dispersion PME with Tang-Toennies damping, the classical terms).

For an energy E(z) with engine gradient G(z) = dE/dz, the vector-Jacobian product of G with a
cotangent c is the Hessian-vector product H c (the Hessian is symmetric), computed here as the
central difference (G(z + e c) - G(z - e c)) / (2 e).  The step e puts every block of z at most
``eps`` of its own scale away from the evaluation point (positions and box: 1 A), with the pair
list held fixed, so the error is O(e^2) in FP64 arithmetic.
"""
import torch


def central_hvp(grad_at, point, direction, scales, eps=1e-4):
    """``grad_at(list of tensors) -> list of gradient tensors`` (same shapes as ``point``);
    ``direction`` a list of tensors or None (zero); ``scales`` the natural size of each block.
    Returns (list of H c blocks, step)."""
    rate = 0.0
    for d, sc in zip(direction, scales):
        if d is not None and d.numel():
            rate = max(rate, float(d.detach().abs().max()) / max(float(sc), 1e-12))
    if rate == 0.0:
        return [torch.zeros_like(p) if p is not None else None for p in point], 0.0
    e = eps / rate

    def shifted(a):
        return [None if p is None else (p if d is None else p + a * d.to(p.device, p.dtype))
                for p, d in zip(point, direction)]

    gp = grad_at(shifted(e))
    gm = grad_at(shifted(-e))
    return [None if a is None else (a - b) / (2.0 * e) for a, b in zip(gp, gm)], e
