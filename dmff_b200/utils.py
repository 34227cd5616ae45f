"""Helpers with the names of dmff/utils.py, for code that imports them next to the force objects.

``regularize_pairs`` and ``pair_buffer_scales`` give the pair-row conventions that the engine's
kernels apply themselves: a row with j <= i is padding.  They run in torch on the rows' device.
``jit_condition`` is the identity decorator here: the compute is compiled CUDA, not traced.
"""
import numpy as np
import torch


class DMFFException(BaseException):
    """The reference's exception type (utils.py:6-7)."""


def dict_to_jnp(inp: dict):
    """Nested dict of arrays -> the same dict of float64 torch tensors (utils.py:45-52)."""
    out = {}
    for k, v in inp.items():
        out[k] = dict_to_jnp(v) if isinstance(v, dict) else torch.as_tensor(np.asarray(v) if not torch.is_tensor(v)
                                                                              else v, dtype=torch.float64)
    return out


def jit_condition(*args, **kwargs):
    """Decorator factory of utils.py:55-64; no tracing here, so it returns the function."""
    def deco(func):
        return func
    return deco


def _rows(p):
    return p.long() if torch.is_tensor(p) else torch.as_tensor(np.asarray(p)).long()


def regularize_pairs(p):
    """Rows (i, j) with j <= i become (i - 1, j - 2), so that padding rows index in range
    (utils.py:67-76)."""
    p = _rows(p)
    pad = (p[:, 1] - p[:, 0] <= 0).long()
    return torch.stack([p[:, 0] - pad, p[:, 1] - 2 * pad], dim=1)


def pair_buffer_scales(p):
    """1 for rows with i < j, 0 for padding rows (utils.py:79-84)."""
    p = _rows(p)
    return (p[:, 0] < p[:, 1]).long()


def convertStr2Float(string: str):
    """float(string), or the string itself when it is not a number (utils.py:100-107)."""
    try:
        return float(string)
    except ValueError:
        return string


def findItemInList(item, targetList):
    """Index of the first element equal to ``item``, or -1 (utils.py:110-114)."""
    for n, t in enumerate(targetList):
        if item == t:
            return n
    return -1
