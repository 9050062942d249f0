"""Fused transport observables for one block-tridiagonal device.

``transmission_dos`` is the batched replacement for the reference pattern
``DeviceProperty.cal_green_function(...)`` followed by the ``tc`` / ``dos`` /
``ldos`` properties (negf/device_property.py:137-296, :374-470): T(E) and the
DOS (and optionally the per-orbital LDOS) come out of one RGF sweep without
materialising any Green's-function block.  Host tensors in give host tensors
out; the H/S blocks and self-energies are copied to the GPU inside the call.
"""
from typing import Optional, Sequence

import torch

from . import rgf_plan


def transmission_dos(hd: Sequence[torch.Tensor], hu: Sequence[torch.Tensor], hl: Sequence[torch.Tensor],
                     sd: Sequence[torch.Tensor], su: Sequence[torch.Tensor], sl: Sequence[torch.Tensor],
                     energy: torch.Tensor, left_se: torch.Tensor, right_se: torch.Tensor, eta: float = 0.0,
                     E_ref: float = 0.0, orbital_dos: bool = False,
                     geometry: Optional[rgf_plan.Geometry] = None, device: str = "cuda", events=None,
                     precision: str = "fp64", refine: bool = False, refine_steps: int = 1):
    """T(E) [B], DOS(E) [B] (spin factor 2) and optionally -Im diag(GS)/pi [B, n_orb].

    ``energy`` is a 1-D ``[B]`` tensor (real or complex); ``left_se`` /
    ``right_se`` are ``[B, n, n]`` lead self-energies embedded in the first /
    last block corners; ``eta`` is the device broadening (``eta_device``).
    Pass a prebuilt ``geometry`` to reuse the packed H/S arena across calls.
    ``precision="mixed"`` computes the block products on the tcgen05 3xTF32
    path (FP32-accurate); ``refine=True`` adds the FP64-residual refinement
    of G_{:,N} that brings T(E) back to FP64-level accuracy (the DOS is not
    refined).
    """
    out_dev = energy.device
    geom = geometry or rgf_plan.Geometry([rgf_plan.DeviceBlocks(hd, hu, hl, sd, su, sl)], device=device)
    dev = geom.device
    E = energy.to(dev, non_blocking=True)
    seL = left_se.to(dev, non_blocking=True)
    seR = right_se.to(dev, non_blocking=True)
    res = rgf_plan.run(geom, [E], [seL], [seR], eta=eta, E_ref=E_ref, outputs=(), trans=True, dos=True,
                       orb_dos=orbital_dos, events=events, precision=precision, refine=refine,
                       refine_steps=refine_steps)
    B = int(E.shape[0])
    T, D = res.trans, res.dos
    orb = res.orb_dos.view(B, -1) if orbital_dos else None
    if out_dev.type != "cuda":
        T, D = T.to(out_dev), D.to(out_dev)
        orb = orb.to(out_dev) if orb is not None else None
    return T, D, orb
