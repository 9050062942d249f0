"""Differentiable transmission: a hand-written adjoint RGF behind torch autograd.

``transmission(...)`` returns T(E) for a batch of energies; its backward runs
the adjoint pass of the RGF kernel (``NEGF_ADJOINT``), which re-sweeps the
device and accumulates, for the loss L = sum_E w_E T(E) with w = dL/dT,

  dL/dX_pq = 2 sum_E w_E W_qp^H,   W_qp = G_qN M G_1p,   M = Gamma_R G_1N^H Gamma_L,
  X = H + Sigma - z S  (so dL/dH_pq = dL/dX_pq and dL/dS_pq = -2 sum_E w_E conj(z_E) W_qp^H),

plus the explicit Gamma terms of the self-energies, dT/dSigma_L = -2i G_1N
Gamma_R G_1N^H (and its mirror for Sigma_R).  G_qN comes from the backward
sweep, the first block row from G_1p = P_p G_pp with P_{p+1} = P_p g_p U_p.
The re-sweep keeps nothing from the forward call; one backward costs about
1.7x a forward sweep.  Inside the adjoint launch every left-connected g_q of
the item stays in the item's scratch slot, or, with ``checkpoint=s`` on
``transmission_and_grad`` / ``rgf_plan.run``, only g_0, g_s, g_2s, ... and one
segment of s blocks, each segment recomputed from its checkpoint when the
backward sweep and the adjoint pass reach it (sqrt(K) checkpointing for
blocks too large to keep).

``transmission_dos(...)`` returns T(E) and DOS(E) (the reference's _cal_dos_,
device_property.py:408-439: -(2/pi) Im Tr[G S] with the block-tridiagonal
trace), both differentiable: the DOS weighted by occupation x quadrature
weights is the summed onsite density n, and its gradient comes from a
z-tangent sweep in the same adjoint launch.  Tr[G S] = d/dz log det(zS - H -
Sigma), so with Y = G S G = -dG/dz
  dn/dH_pq = i c conj(Y_qp),  dn/dS_pq = i c (conj(G_qp) - conj(z) conj(Y_qp)),
  dn/dSigma_pq = i c conj(Y_qp),   c = -(2/pi) w_E,
and only the block-tridiagonal blocks of Y are needed; the tangent sweep
differentiates the forward recursion (dg_q = -g_q dK_q g_q) and the backward
blocks, about 16 more block products per block.

Gradients follow torch's convention for complex leaves (dL/dRe + i dL/dIm),
so they compose with autograd through the caller's tight-binding model; the
Landauer current is a differentiable Simpson sum over T (``current``).
No counterpart in the reference, which offers only torch autograd through its
Python ``recursive_gf``.
"""
from typing import Sequence

import torch

from . import rgf_plan
from .negf_utils import simpson


class _TransmissionFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, energy, eta, E_ref, K, precision, refine, left_se, right_se, *blocks):
        hd, hu, hl, sd, su, sl = _split(blocks, K)
        geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(hd, hu, hl, sd, su, sl)], device=left_se.device,
                                 detect_zero_offdiag=False)
        res = rgf_plan.run(geom, [energy], [left_se], [right_se], eta=eta, E_ref=E_ref, outputs=(), trans=True,
                           precision=precision, refine=refine)
        ctx.geom = geom
        ctx.eta, ctx.E_ref, ctx.K, ctx.precision = eta, E_ref, K, precision
        ctx.save_for_backward(energy, left_se, right_se)
        return res.trans.clone()

    @staticmethod
    def backward(ctx, gT):
        energy, left_se, right_se = ctx.saved_tensors
        res = rgf_plan.run(ctx.geom, [energy], [left_se], [right_se], eta=ctx.eta, E_ref=ctx.E_ref, outputs=(),
                           adjoint_w=gT.detach().to(torch.float64), precision=ctx.precision)
        g = res.grads
        K = ctx.K
        block_grads = g["hd"] + g["hu"] + g["hl"] + g["sd"] + g["su"] + g["sl"]
        assert len(block_grads) == 6 * K - 4
        return (None, None, None, None, None, None, g["se_l"], g["se_r"]) + tuple(block_grads)


class _TransmissionDosFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, energy, eta, E_ref, K, precision, left_se, right_se, *blocks):
        hd, hu, hl, sd, su, sl = _split(blocks, K)
        geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(hd, hu, hl, sd, su, sl)], device=left_se.device,
                                 detect_zero_offdiag=False)
        res = rgf_plan.run(geom, [energy], [left_se], [right_se], eta=eta, E_ref=E_ref, outputs=(), trans=True,
                           dos=True, precision=precision)
        ctx.geom = geom
        ctx.eta, ctx.E_ref, ctx.K, ctx.precision = eta, E_ref, K, precision
        ctx.save_for_backward(energy, left_se, right_se)
        return res.trans.clone(), res.dos.clone()

    @staticmethod
    def backward(ctx, gT, gD):
        energy, left_se, right_se = ctx.saved_tensors
        B = energy.shape[0]
        z = torch.zeros(B, dtype=torch.float64, device=left_se.device)
        wt = gT.detach().to(torch.float64) if gT is not None else z
        wd = gD.detach().to(torch.float64) if gD is not None else z
        res = rgf_plan.run(ctx.geom, [energy], [left_se], [right_se], eta=ctx.eta, E_ref=ctx.E_ref, outputs=(),
                           adjoint_w=wt, adjoint_w_dos=wd, precision=ctx.precision)
        g = res.grads
        block_grads = g["hd"] + g["hu"] + g["hl"] + g["sd"] + g["su"] + g["sl"]
        return (None, None, None, None, None, g["se_l"], g["se_r"]) + tuple(block_grads)


def _split(blocks, K):
    hd = list(blocks[0:K])
    hu = list(blocks[K:2 * K - 1])
    hl = list(blocks[2 * K - 1:3 * K - 2])
    sd = list(blocks[3 * K - 2:4 * K - 2])
    su = list(blocks[4 * K - 2:5 * K - 3])
    sl = list(blocks[5 * K - 3:6 * K - 4])
    return hd, hu, hl, sd, su, sl


def transmission(hd: Sequence[torch.Tensor], hu: Sequence[torch.Tensor], hl: Sequence[torch.Tensor],
                 sd: Sequence[torch.Tensor], su: Sequence[torch.Tensor], sl: Sequence[torch.Tensor],
                 energy: torch.Tensor, left_se: torch.Tensor, right_se: torch.Tensor, eta: float = 0.0,
                 E_ref: float = 0.0, precision: str = "fp64", refine: bool = False) -> torch.Tensor:
    """T(E) [B] of one BTD device, differentiable w.r.t. every 2-D block and both
    ``[B, n, n]`` self-energies (CUDA tensors).

    ``precision="mixed"`` runs the forward sweep and the adjoint pass on the
    tcgen05 3xTF32 products (gradients at FP32-product accuracy); ``refine``
    refines the forward T(E) with an FP64 residual."""
    K = len(hd)
    if not (len(sd) == K and len(hu) == len(hl) == len(su) == len(sl) == K - 1):
        raise ValueError("inconsistent block lists")
    energy = torch.as_tensor(energy).to(torch.complex128).reshape(-1).detach()
    blocks = list(hd) + list(hu) + list(hl) + list(sd) + list(su) + list(sl)
    return _TransmissionFn.apply(energy, float(eta), float(E_ref), K, precision, bool(refine), left_se, right_se,
                                 *blocks)


def transmission_dos(hd: Sequence[torch.Tensor], hu: Sequence[torch.Tensor], hl: Sequence[torch.Tensor],
                     sd: Sequence[torch.Tensor], su: Sequence[torch.Tensor], sl: Sequence[torch.Tensor],
                     energy: torch.Tensor, left_se: torch.Tensor, right_se: torch.Tensor, eta: float = 0.0,
                     E_ref: float = 0.0, precision: str = "fp64"):
    """(T(E), DOS(E)), each [B], of one BTD device, both differentiable w.r.t. every
    2-D block and both ``[B, n, n]`` self-energies (CUDA tensors).  The DOS is the
    reference's (spin factor 2, block-tridiagonal trace of G S); a weighted sum of
    it over an energy window is the summed onsite density, so losses such as
    current + density (Landauer I from T, n from DOS) take one adjoint launch."""
    K = len(hd)
    if not (len(sd) == K and len(hu) == len(hl) == len(su) == len(sl) == K - 1):
        raise ValueError("inconsistent block lists")
    energy = torch.as_tensor(energy).to(torch.complex128).reshape(-1).detach()
    blocks = list(hd) + list(hu) + list(hl) + list(sd) + list(su) + list(sl)
    return _TransmissionDosFn.apply(energy, float(eta), float(E_ref), K, precision, left_se, right_se, *blocks)


def transmission_and_grad(hd: Sequence[torch.Tensor], hu: Sequence[torch.Tensor], hl: Sequence[torch.Tensor],
                          sd: Sequence[torch.Tensor], su: Sequence[torch.Tensor], sl: Sequence[torch.Tensor],
                          energy: torch.Tensor, left_se: torch.Tensor, right_se: torch.Tensor,
                          weights: torch.Tensor, eta: float = 0.0, E_ref: float = 0.0, precision: str = "fp64",
                          refine: bool = False, dos_weights=None, checkpoint=0):
    """T(E) and the gradient of L = sum_E w_E T(E) for weights known in advance, in one launch.

    The adjoint pass sweeps the device itself and reduces T(E) on the way, so
    a loss that is linear in T with fixed weights (the Landauer current's
    Fermi-window quadrature weights, a weighted sum of transmissions) needs no
    separate forward call: this costs one adjoint launch instead of the
    forward + backward launches of ``transmission`` under autograd.  Returns
    ``(T [B], grads)`` with ``grads`` keyed ``hd, hu, hl, sd, su, sl`` (lists
    of blocks) and ``se_l, se_r`` ([B, n, n], each energy's dL/dSigma), in
    torch's complex-gradient convention, equal to what autograd through
    ``transmission`` gives for ``(w * T).sum()``.  ``refine`` refines the
    column G_{:,N} (mixed precision) before T and the gradient are formed.
    ``dos_weights`` ([B]) add the gradient of sum_E wd_E DOS(E) (the summed
    onsite density for occupation x quadrature weights) to the same launch.  ``checkpoint``
    (an interval s, or "sqrt") keeps only every s-th left-connected block of the forward sweep
    and recomputes the others segment by segment (rgf_plan.run), for devices whose full set of
    blocks does not fit the per-SM scratch."""
    K = len(hd)
    if not (len(sd) == K and len(hu) == len(hl) == len(su) == len(sl) == K - 1):
        raise ValueError("inconsistent block lists")
    energy = torch.as_tensor(energy).to(torch.complex128).reshape(-1).detach()
    w = torch.as_tensor(weights, dtype=torch.float64).reshape(-1).detach()
    if w.shape[0] != energy.shape[0]:
        raise ValueError(f"{w.shape[0]} weights for {energy.shape[0]} energies")
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks([t.detach() for t in hd], [t.detach() for t in hu],
                                                    [t.detach() for t in hl], [t.detach() for t in sd],
                                                    [t.detach() for t in su], [t.detach() for t in sl])],
                             device=left_se.device, detect_zero_offdiag=False)
    wd = None
    if dos_weights is not None:
        wd = torch.as_tensor(dos_weights, dtype=torch.float64).reshape(-1).detach()
        if wd.shape[0] != energy.shape[0]:
            raise ValueError(f"{wd.shape[0]} DOS weights for {energy.shape[0]} energies")
    res = rgf_plan.run(geom, [energy], [left_se.detach()], [right_se.detach()], eta=eta, E_ref=E_ref, outputs=(),
                       adjoint_w=w, adjoint_w_dos=wd, precision=precision, refine=refine,
                       refine_steps=3 if refine else 1, checkpoint=checkpoint)
    return res.trans.clone(), res.grads


class _LeadSelfEnergyFn(torch.autograd.Function):
    """Sigma(E) of one lead, differentiable through the converged decimation fixed point.

    Forward: the CUDA Lopez-Sancho decimation (one launch for every energy) gives
    g_s and Sigma.  Backward: g_s is the fixed point of
        f(g) = (z S - H - tau g tau')^-1,  tau = z S01 - H01,  tau' = z S01^H - H01^H
    (the residual the reference checks, negf/surface_green.py:142-145), so with
    V = dL/dg_s (from Sigma = (E S_DL - H_DL) g_s[:b,:b] (E S_DL^H - H_DL^H), or the
    bulk form (E S - H) - g_s^-1) the implicit-function adjoint is
        Lambda = V + P^H Lambda Q^H,   P = g_s tau,  Q = tau' g_s,
    a Stein equation solved by doubling (Lambda += A Lambda B, A <- A^2, B <- B^2:
    2^j terms after j steps, the Lopez-Sancho convergence, since the spectral
    radii of P and Q are below one for eta > 0), and dL/dtheta is the
    Lambda-weighted derivative of f at the fixed point plus the explicit
    dependence of Sigma on H_DL, S_DL, H and S.  The whole backward (V, the
    doubling, the inverse of f's argument and the parameter terms, summed over
    energies) is one launch of ``negf_lead_adjoint_run``."""

    @staticmethod
    def forward(ctx, energies, eta, E_ref, bulk, hL, hLL, sL, sLL, hDL, sDL):
        from . import surface_green as sg
        lead = sg.LeadBlocks(hL=hL.detach(), hLL=hLL.detach(), sL=sL.detach(), sLL=sLL.detach(),
                             hDL=None if hDL is None else hDL.detach(), sDL=None if sDL is None else sDL.detach())
        arena = sg.LeadArena([lead], device=hL.device)
        E = energies.detach().cpu().numpy()
        res = sg.self_energies(arena, [0] * len(E), E, eta, E_ref=E_ref, want_gs=True)
        gs = torch.stack(res.gs)
        sig = torch.stack(res.sigma)
        if hDL is None and bulk:
            Eb = (energies.to(hL.device) + E_ref).view(-1, 1, 1)
            sig = Eb * sL.detach() - hL.detach() - sig
        ctx.save_for_backward(energies, gs, hL, hLL, sL, sLL, hDL, sDL)
        ctx.eta, ctx.E_ref, ctx.bulk = eta, E_ref, bulk
        return sig

    @staticmethod
    def backward(ctx, gsig):
        from .products import lead_adjoint
        energies, gs, hL, hLL, sL, sLL, hDL, sDL = ctx.saved_tensors
        form = 0 if hDL is not None else (1 if ctx.bulk else 2)
        E = energies.detach().cpu().numpy() + ctx.E_ref
        dH, dH01, dS, dS01, dHDL, dSDL = lead_adjoint(hL.detach(), hLL.detach(), sL.detach(), sLL.detach(),
                                                      None if hDL is None else hDL.detach(),
                                                      None if sDL is None else sDL.detach(),
                                                      E, ctx.eta, gs, gsig, form)
        # a real parameter receives the real part (the backward of its promotion to complex)
        cast = lambda g, t: None if g is None else (g if t.is_complex() else g.real).to(t.dtype)
        return (None, None, None, None, cast(dH, hL), cast(dH01, hLL), cast(dS, sL), cast(dS01, sLL),
                cast(dHDL, hDL), cast(dSDL, sDL))


def lead_self_energy(hL: torch.Tensor, hLL: torch.Tensor, sL: torch.Tensor, sLL: torch.Tensor,
                     energies: torch.Tensor, eta: float, hDL: torch.Tensor = None, sDL: torch.Tensor = None,
                     E_ref: float = 0.0, bulk: bool = False) -> torch.Tensor:
    """Sigma(E) [B, nc, nc] of one lead at real energies ``energies`` [B] (relative to ``E_ref``),
    differentiable w.r.t. H, H_01, S, S_01, H_DL and S_DL (2-D CUDA tensors).

    The same quantity as ``surface_green.selfEnergy`` (negf/surface_green.py:9-91:
    decimation at z = E + E_ref + i eta, Sigma = (E S_DL - H_DL) g_s[:b,:b]
    (E S_DL^H - H_DL^H) with E = energy + E_ref, or the bulk forms without H_DL),
    for every energy in one decimation launch.  Its gradient goes through the
    converged surface Green's function by implicit differentiation, so
    tight-binding parameters of the leads can be fitted together with the
    device's: pass the result as ``left_se`` / ``right_se`` to ``transmission``
    or ``transmission_dos``.  Raises as ``selfEnergy`` does when the decimation
    fails its residual check."""
    e = torch.as_tensor(energies, dtype=torch.float64).reshape(-1).to(torch.complex128)
    return _LeadSelfEnergyFn.apply(e, float(eta), float(E_ref), bool(bulk), hL, hLL, sL, sLL, hDL, sDL)


def current(T: torch.Tensor, energy: torch.Tensor, f_left: torch.Tensor, f_right: torch.Tensor) -> torch.Tensor:
    """Landauer current sum(E) (f_L - f_R) T by Simpson's rule (no 2e/h prefactor, as the reference)."""
    e = torch.as_tensor(energy, dtype=torch.float64, device=T.device).real
    return simpson((f_left - f_right).to(T.dtype) * T, e)
