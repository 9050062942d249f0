"""Quadrature helpers of the density / current integrals (torch, any device).

``gauss_xw`` mirrors negf/negf_utils.py:136-160 (Gauss-Legendre nodes and
weights mapped to [xl, xu]).  ``simpson`` is the composite Simpson rule for
irregularly spaced samples with the last-interval correction for an even
number of points (Cartwright 2017, eq. 8 rearranged for the final interval),
the rule scipy.integrate.simpson applies; the reference integrates the
Landauer current with it (negf/device_property.py:366-369).  Written in torch
so the current integration runs on the GPU in FP64.
"""
import numpy as np
import torch


def gauss_xw(xl, xu, n=100):
    """Gauss-Legendre points and weights on [xl, xu] (same layout as the reference), in the
    floating dtype of ``xu`` as the reference computes them (a float32 ``xu``, e.g. from
    ``torch.scalar_tensor`` of a Python float, gives float32 nodes and weights)."""
    xu = torch.as_tensor(xu)
    if not xu.is_floating_point():
        xu = xu.to(torch.float64)
    xl = torch.as_tensor(xl, dtype=xu.dtype, device=xu.device)
    nd = xu.ndim
    x, w = np.polynomial.legendre.leggauss(n)
    x = torch.tensor(x, dtype=xu.dtype, device=xu.device)[(...,) + (None,) * nd]
    w = torch.tensor(w, dtype=xu.dtype, device=xu.device)[(...,) + (None,) * nd]
    half = 0.5 * (xu - xl)
    return x * half + 0.5 * (xu + xl), w * half


def _simpson_pairs(y, x):
    """Composite Simpson over consecutive interval pairs of (y, x) (odd sample count)."""
    h = torch.diff(x, dim=-1)
    h0, h1 = h[..., 0::2], h[..., 1::2]
    hs = h0 + h1
    r = h0 / h1
    y0, y1, y2 = y[..., 0:-2:2], y[..., 1:-1:2], y[..., 2::2]
    return (hs / 6.0 * (y0 * (2.0 - 1.0 / r) + y1 * (hs * hs / (h0 * h1)) + y2 * (2.0 - r))).sum(-1)


def simpson(y, x):
    """Integrate samples ``y`` over ``x`` (last axis) by composite Simpson's rule."""
    y = torch.as_tensor(y)
    x = torch.as_tensor(x, dtype=y.dtype if y.is_floating_point() else torch.float64, device=y.device)
    N = y.shape[-1]
    if N < 2:
        return torch.zeros(y.shape[:-1], dtype=y.dtype, device=y.device)
    if N == 2:
        return 0.5 * (x[..., 1] - x[..., 0]) * (y[..., 0] + y[..., 1])
    if N % 2 == 1:
        return _simpson_pairs(y, x)
    res = _simpson_pairs(y[..., :-1], x[..., :-1])
    ha, hb = x[..., -2] - x[..., -3], x[..., -1] - x[..., -2]
    alpha = (2.0 * hb ** 2 + 3.0 * ha * hb) / (6.0 * (ha + hb))
    beta = (hb ** 2 + 3.0 * ha * hb) / (6.0 * ha)
    eta = hb ** 3 / (6.0 * ha * (ha + hb))
    return res + alpha * y[..., -1] + beta * y[..., -2] - eta * y[..., -3]
