"""Lead surface Green's functions and self-energies on the B200.

Drop-in for negf/surface_green.py: ``selfEnergy`` and ``surface_green`` keep
the reference signatures, argument meaning, return types and error behaviour
(``ArithmeticError`` when the Lopez-Sancho residual check fails, ``RuntimeError``
after more than 100 decimation steps, a logged warning for a residual above
1e-8).  The decimation itself runs in the CUDA kernel ``negf_lopez_sancho_run``;
``self_energies`` evaluates many (lead, energy) pairs in one launch, which is how
the runner's per-(k, E) self-energy loop (negf/lead_property.py:599-683) maps
onto the GPU.
"""
import ctypes
import logging
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib

log = logging.getLogger(__name__)
C128 = torch.complex128
LS_TOL = 1.0e-40      # negf/surface_green.py:139
LS_MAX_ITER = 100     # negf/surface_green.py:156 (the 101st step raises)


@dataclass
class LeadBlocks:
    """One lead principal layer: H, S, H_01, S_01 [n, n]; H_DL, S_DL [nc, b] or None."""
    hL: torch.Tensor
    hLL: torch.Tensor
    sL: torch.Tensor
    sLL: torch.Tensor
    hDL: Optional[torch.Tensor] = None
    sDL: Optional[torch.Tensor] = None


@dataclass
class DecimationResult:
    sigma: List[torch.Tensor]        # per item: [nc, nc] (or [n, n] bulk form)
    gs: Optional[List[torch.Tensor]] # per item: [n, n] when requested
    status: np.ndarray
    iters: np.ndarray
    resid: np.ndarray


def _c128(x):
    if isinstance(x, np.ndarray):
        x = torch.from_numpy(x)
    return torch.as_tensor(x).to(C128)


class LeadArena:
    """Packed lead blocks on the GPU (energy independent; build once per k-point)."""

    def __init__(self, leads: Sequence[LeadBlocks], device="cuda"):
        dev = torch.device(device)
        self.device = dev
        pieces, table = [], []
        cursor = 0

        def put(t):
            nonlocal cursor
            f = _c128(t).to(dev).reshape(-1)
            pieces.append(f)
            off = cursor
            cursor += f.numel()
            return off

        self.max_n = 0
        self.shapes = []
        for ld in leads:
            n = int(ld.hL.shape[-1])
            rec = np.zeros((), dtype=_lib.LEAD_DTYPE)
            rec["n"] = n
            rec["h"], rec["s"] = put(ld.hL), put(ld.sL)
            rec["h01"], rec["s01"] = put(ld.hLL), put(ld.sLL)
            if ld.hDL is not None:
                nc, b = int(ld.hDL.shape[0]), int(ld.hDL.shape[1])
                if b > n:
                    raise ValueError(f"H_DL has {b} columns, more than the principal layer ({n})")
                sdl = ld.sDL if ld.sDL is not None else torch.zeros_like(_c128(ld.hDL))
                rec["nc"], rec["b"] = nc, b
                rec["hdl"], rec["sdl"] = put(ld.hDL), put(sdl)
                self.shapes.append((n, nc))
                # the self-energy products are nc x b and nc x nc: slot buffers are sized by max(n, nc)
                self.max_n = max(self.max_n, nc)
            else:
                rec["nc"], rec["b"] = 0, n
                rec["hdl"] = rec["sdl"] = -1
                self.shapes.append((n, n))
            table.append(rec)
            self.max_n = max(self.max_n, n)
        if self.max_n > _lib.NEGF_MAX_BLOCK:
            raise ValueError(f"lead block {self.max_n} exceeds the supported maximum {_lib.NEGF_MAX_BLOCK}")
        self.arena = torch.cat(pieces)
        self.table = np.array(table, dtype=_lib.LEAD_DTYPE)


@_lib.on_given_stream
def self_energies(arena: LeadArena, lead_index: Sequence[int], energies, eta, E_ref=0.0, want_gs=False,
                  want_sigma=True, tol=LS_TOL, max_iter=LS_MAX_ITER, check=True, n_slots=None, stream=None):
    """Decimate every (lead_index[i], energies[i]) pair in one launch.

    ``energies`` are complex (E relative to ``E_ref``); the decimation uses
    z = E + E_ref + i*eta and the self-energy product E + E_ref (reference
    :65-86).  ``eta`` is a scalar or per item.  Returns a DecimationResult.
    """
    _lib.require_cuda()
    lib = _lib.load()
    dev = arena.device
    E = np.asarray(energies, dtype=np.complex128).reshape(-1) + complex(E_ref)
    idx = np.asarray(lead_index, dtype=np.int64).reshape(-1)
    if idx.shape[0] != E.shape[0]:
        raise ValueError("one lead index per energy")
    B = E.shape[0]
    eta_a = np.broadcast_to(np.asarray(eta, dtype=np.float64), (B,))
    sig_sizes = [arena.shapes[i][1] for i in idx]
    sig_off = np.concatenate([[0], np.cumsum([s * s for s in sig_sizes])]).astype(np.int64)
    sig_buf = torch.empty(max(int(sig_off[-1]), 1), dtype=C128, device=dev)
    gs_sizes = [arena.shapes[i][0] for i in idx]
    gs_off = np.concatenate([[0], np.cumsum([s * s for s in gs_sizes])]).astype(np.int64)
    gs_buf = torch.empty(max(int(gs_off[-1]), 1), dtype=C128, device=dev) if want_gs else None
    items = np.zeros(B, dtype=_lib.LS_ITEM_DTYPE)
    items["lead"] = idx
    items["e_re"], items["e_im"] = E.real, E.imag
    items["eta"] = eta_a
    items["sigma"] = (sig_buf.data_ptr() + sig_off[:-1] * 16) if want_sigma else 0
    items["gs"] = (gs_buf.data_ptr() + gs_off[:-1] * 16) if want_gs else 0
    items["out"] = np.arange(B)
    # heaviest first
    order = np.argsort(-np.array([arena.shapes[i][0] for i in idx]), kind="stable")
    items = items[order]
    u8 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    leads_t, items_t = u8(arena.table), u8(items)
    status = torch.empty(B, dtype=torch.int32, device=dev)
    iters = torch.empty(B, dtype=torch.int32, device=dev)
    resid = torch.empty(B, dtype=torch.float64, device=dev)
    p = _lib.NegfLsProblem()
    p.leads, p.items, p.n_items, p.max_n = leads_t.data_ptr(), items_t.data_ptr(), B, arena.max_n
    p.arena = arena.arena.data_ptr()
    p.status, p.iters, p.resid = status.data_ptr(), iters.data_ptr(), resid.data_ptr()
    p.tol, p.max_iter = float(tol), int(max_iter)
    p.n_slots = n_slots or max(1, min(B, lib.negf_sm_count()))
    need = lib.negf_lopez_sancho_scratch_bytes(ctypes.byref(p))
    scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    p.scratch, p.scratch_bytes = scratch.data_ptr(), scratch.numel()
    _lib.check(lib.negf_lopez_sancho_run(ctypes.byref(p), _lib.stream_handle(stream)), "negf_lopez_sancho_run")
    st = status.cpu().numpy()
    res = DecimationResult(
        sigma=[sig_buf[sig_off[i]:sig_off[i + 1]].view(sig_sizes[i], sig_sizes[i]) for i in range(B)]
        if want_sigma else None,
        gs=[gs_buf[gs_off[i]:gs_off[i + 1]].view(gs_sizes[i], gs_sizes[i]) for i in range(B)] if want_gs else None,
        status=st, iters=iters.cpu().numpy(), resid=resid.cpu().numpy())
    if check:
        raise_for_status(st, res.resid, E)
    return res


def raise_for_status(status, resid, E):
    """Map per-item status codes to the reference's exceptions and warnings."""
    for i, s in enumerate(status):
        if s == _lib.NEGF_WARN_LS_CONVERGENCE:
            log.warning(f"Lopez-Sancho scheme not-so-well converged at E = {E[i].real:.4f} eV: {resid[i]}")
        elif s == _lib.NEGF_ERR_LS_RESIDUAL:
            log.error(f"Lopez-Sancho {resid[i]:.8f} Error: gs iteration at E = {E[i].real:.4f}")
            raise ArithmeticError("Criteria not met. Please check output...")
        elif s == _lib.NEGF_ERR_LS_NOT_CONVERGED:
            log.error("Lopez-scheme not converged after 100 iteration.")
            raise RuntimeError("Lopez-scheme not converged.")
        elif s == _lib.NEGF_ERR_SINGULAR:
            raise ArithmeticError(f"Lopez-Sancho: singular matrix at E = {E[i].real:.4f} eV")
        elif s == _lib.NEGF_ERR_ARGUMENT:
            raise ValueError(f"Lopez-Sancho: item {i} has a lead larger than the problem's max_n")


def selfEnergy(hL, hLL, sL, sLL, ee, hDL=None, sDL=None, etaLead=1e-8, Bulk=False,
               E_ref=0.0, dtype=np.complex128, device='cpu', method='Lopez-Sancho', numba_jit=None):
    """Self-energy and surface Green's function of a lead at one energy.

    Same contract as negf/surface_green.py:9-91: returns ``(Sig, SGF)`` as
    complex128 torch tensors on ``device``.  ``Sig = (E sDL - hDL) SGF[:b,:b]
    (E sDL^H - hDL^H)`` with ``E = ee + E_ref``; without ``hDL`` the bulk form
    ``(E sL - hL) - SGF^-1`` (``SGF^-1`` itself when ``Bulk``).  ``method``
    other than Lopez-Sancho (the reference's GEP) is not provided.
    """
    if method == 'GEP':
        raise NotImplementedError("the GEP surface Green's function is not provided by dpnegf_b200")
    ee_t = ee.detach().cpu().numpy() if torch.is_tensor(ee) else np.asarray(ee)
    E_ref_v = E_ref.detach().cpu().numpy() if torch.is_tensor(E_ref) else E_ref
    e = complex(np.asarray(ee_t).reshape(-1)[0]) + complex(np.asarray(E_ref_v).reshape(-1)[0])
    lead = LeadBlocks(hL=_c128(hL), hLL=_c128(hLL), sL=_c128(sL), sLL=_c128(sLL),
                      hDL=None if hDL is None else _c128(hDL), sDL=None if sDL is None else _c128(sDL))
    arena = LeadArena([lead])
    res = self_energies(arena, [0], [e], etaLead, want_gs=True)
    gs, sig = res.gs[0], res.sigma[0]
    if hDL is None and Bulk:
        # the kernel's bulk form is (E sL - hL) - g_s^-1; the reference's Bulk returns g_s^-1
        sig = e * lead.sL.to(sig.device) - lead.hL.to(sig.device) - sig
    return sig.to(device), gs.to(device)


def surface_green(H, h01, S, s01, ee, method='Lopez-Sancho', numba_jit=None):
    """Surface Green's function g_s at complex energy ``ee`` (negf/surface_green.py:229-279).

    Returns a numpy complex128 array like the reference.
    """
    if method == 'GEP':
        raise NotImplementedError("the GEP surface Green's function is not provided by dpnegf_b200")
    lead = LeadBlocks(hL=_c128(H), hLL=_c128(h01), sL=_c128(S), sLL=_c128(s01))
    arena = LeadArena([lead])
    # ee already carries the broadening: decimate at z = ee exactly
    res = self_energies(arena, [0], [complex(ee)], 0.0, want_gs=True, want_sigma=False)
    return res.gs[0].cpu().numpy()
