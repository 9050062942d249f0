"""Product chains around the sweep, on the library's CUDA kernels.

``gamma_sum``     out = sum_i w_i Re(G_i[:, c0:c0+k] Gamma_i G_i[:, c0:c0+k]^H): the
                  non-equilibrium density matrix of ``Ozaki.integrate``
                  (negf/density.py:183-195) in two launches (per-energy products, then one
                  GEMM over every energy in order).
``coupling_sigma`` Sigma_i = (E_i S_DL - H_DL) g_i[:b,:b] (E_i S_DL^H - H_DL^H) for surface
                  Green's functions the caller supplies (the Bloch-unfolded leads of
                  negf/lead_property.py:330-379), through the decimation kernel's own
                  coupling product.
``lead_adjoint``  the gradient of a loss through a lead's self-energies by implicit
                  differentiation of the converged decimation, one launch for every energy.

No CPU fallback: each raises without the CUDA library or a GPU.
"""
import ctypes

import numpy as np
import torch

from . import _lib

C128 = torch.complex128
LEADADJ_TOL = 1.0e-32    # doubling stops once max|P| max|Q| drops below this
LEADADJ_MAX_ITER = 64    # 2^64 terms of the Neumann series at most


def _u8(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)


def _rows_contiguous(t):
    """A view whose rows are contiguous (stride 1 in the last dimension), copying only if needed."""
    return t if t.stride(-1) == 1 else t.contiguous()


@_lib.on_given_stream
def gamma_sum(G: torch.Tensor, gamma: torch.Tensor, c0: int, w: torch.Tensor, stream=None) -> torch.Tensor:
    """sum_i w_i Re(G_i[:, c0:c0+k] gamma_i G_i[:, c0:c0+k]^H) as a real [n, n] tensor.

    ``G`` [B, n, m] and ``gamma`` [B, k, k] complex128 CUDA tensors (views allowed when their rows
    are contiguous), ``w`` [B] real weights.  Bitwise reproducible (fixed summation order)."""
    if G.ndim != 3 or gamma.ndim != 3 or G.shape[0] != gamma.shape[0]:
        raise ValueError("G [B, n, m] and gamma [B, k, k] with the same B")
    B, n, m = G.shape
    k = gamma.shape[-1]
    if gamma.shape[-2] != k or c0 < 0 or c0 + k > m:
        raise ValueError(f"gamma {tuple(gamma.shape)} does not fit columns {c0}..{c0 + k} of G {tuple(G.shape)}")
    dev = G.device
    G = _rows_contiguous(G.to(C128).resolve_conj())
    gam = _rows_contiguous(gamma.to(dev, C128).resolve_conj())
    w = torch.as_tensor(w, dtype=torch.float64).reshape(-1).to(dev).contiguous()
    if w.shape[0] != B:
        raise ValueError(f"{w.shape[0]} weights for {B} energies")
    _lib.require_cuda()
    lib = _lib.load()
    out = torch.empty(n, n, dtype=torch.float64, device=dev)
    p = _lib.NegfGammaSum()
    p.g, p.g_stride, p.ldg = G.data_ptr(), G.stride(0), G.stride(1)
    p.gamma, p.gamma_stride, p.ldgam = gam.data_ptr(), gam.stride(0), gam.stride(1)
    p.w, p.out = w.data_ptr(), out.data_ptr()
    p.n_items, p.n, p.c0, p.k = B, n, int(c0), k
    need = lib.negf_gamma_sum_scratch_bytes(ctypes.byref(p))
    scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    p.scratch, p.scratch_bytes = scratch.data_ptr(), scratch.numel()
    _lib.check(lib.negf_gamma_sum_run(ctypes.byref(p), _lib.stream_handle(stream)), "negf_gamma_sum_run")
    return out


@_lib.on_given_stream
def coupling_sigma(g: torch.Tensor, hdl: torch.Tensor, sdl: torch.Tensor, energies, E_ref=0.0,
                   stream=None) -> torch.Tensor:
    """Sigma_i = (E_i S_DL - H_DL) g_i[:b,:b] (E_i S_DL^H - H_DL^H), E_i = energies_i + E_ref.

    ``g`` [B, N, N] complex128 CUDA tensor, ``hdl``/``sdl`` [nc, b] (b <= N; ``sdl`` may be None).
    One launch of the decimation kernel in its coupling-product mode; returns [B, nc, nc]."""
    dev = g.device
    g = g.to(C128).resolve_conj().contiguous()
    B, N = g.shape[0], g.shape[-1]
    hdl = torch.as_tensor(hdl).to(dev, C128).resolve_conj().contiguous()
    sdl = torch.zeros_like(hdl) if sdl is None else torch.as_tensor(sdl).to(dev, C128).resolve_conj().contiguous()
    nc, b = hdl.shape
    if b > N or sdl.shape != hdl.shape:
        raise ValueError(f"H_DL {tuple(hdl.shape)} / S_DL {tuple(sdl.shape)} do not fit g of size {N}")
    E = np.asarray(energies, dtype=np.complex128).reshape(-1) + complex(E_ref)
    if E.shape[0] != B:
        raise ValueError(f"{E.shape[0]} energies for {B} surface Green's functions")
    _lib.require_cuda()
    lib = _lib.load()
    arena = torch.cat([hdl.reshape(-1), sdl.reshape(-1)])
    lead = np.zeros((), dtype=_lib.LEAD_DTYPE)
    lead["n"], lead["nc"], lead["b"] = N, nc, b
    lead["hdl"], lead["sdl"] = 0, nc * b
    sig = torch.empty(B, nc, nc, dtype=C128, device=dev)
    items = np.zeros(B, dtype=_lib.LS_ITEM_DTYPE)
    items["mode"] = _lib.LS_SIGMA_FROM_GS
    items["e_re"], items["e_im"] = E.real, E.imag
    items["sigma"] = sig.data_ptr() + np.arange(B, dtype=np.uint64) * (nc * nc * 16)
    items["gs"] = g.data_ptr() + np.arange(B, dtype=np.uint64) * (N * N * 16)
    items["out"] = np.arange(B)
    leads_t, items_t = _u8(lead.reshape(1), dev), _u8(items, dev)
    status = torch.empty(B, dtype=torch.int32, device=dev)
    p = _lib.NegfLsProblem()
    p.leads, p.items, p.n_items, p.max_n = leads_t.data_ptr(), items_t.data_ptr(), B, max(nc, b)
    p.arena, p.status = arena.data_ptr(), status.data_ptr()
    p.max_iter = 0
    p.n_slots = max(1, min(B, lib.negf_sm_count()))
    need = lib.negf_lopez_sancho_scratch_bytes(ctypes.byref(p))
    scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    p.scratch, p.scratch_bytes = scratch.data_ptr(), scratch.numel()
    _lib.check(lib.negf_lopez_sancho_run(ctypes.byref(p), _lib.stream_handle(stream)), "negf_lopez_sancho_run")
    st = status.cpu().numpy()
    if (st != _lib.NEGF_OK).any():
        raise _lib.NegfError(f"coupling product: status {st[st != _lib.NEGF_OK][0]} (malformed sizes)")
    return sig


@_lib.on_given_stream
def lead_adjoint(hL, hLL, sL, sLL, hDL, sDL, E, eta, gs, gsig, form, tol=LEADADJ_TOL, max_iter=LEADADJ_MAX_ITER,
                 stream=None, info=None):
    """dL/d(hL, hLL, sL, sLL, hDL, sDL) through Sigma(E) of one lead (PyTorch's complex convention).

    ``E`` [B] complex (energy + E_ref), ``gs`` [B, n, n] the converged surface Green's functions at
    E + i eta, ``gsig`` [B, nc, nc] (form 0) or [B, n, n] (forms 1, 2) the incoming gradient of
    Sigma.  form 0: Sigma = (E S_DL - H_DL) g[:b,:b] (E S_DL^H - H_DL^H); 1: Sigma = g^-1;
    2: Sigma = E S - H - g^-1.  Returns six tensors (None for hDL/sDL when not given); a dict
    passed as ``info`` receives the doubling steps per energy under "iters"."""
    if form not in (0, 1, 2):
        raise ValueError(f"form must be 0, 1 or 2, not {form!r}")
    if form == 0 and hDL is None:
        raise ValueError("form 0 (the coupling form) needs H_DL")
    dev = gs.device
    c = lambda t: torch.as_tensor(t).to(dev, C128).resolve_conj().contiguous()
    hL, hLL, sL, sLL = c(hL), c(hLL), c(sL), c(sLL)
    n = hL.shape[-1]
    gs = c(gs)
    gsig = c(gsig)
    B = gs.shape[0]
    pieces = [hL.reshape(-1), sL.reshape(-1), hLL.reshape(-1), sLL.reshape(-1)]
    lead = _lib.NegfLead()
    lead.n, lead.h, lead.s, lead.h01, lead.s01 = n, 0, n * n, 2 * n * n, 3 * n * n
    lead.hdl = lead.sdl = -1
    nc = b = 0
    if form == 0:
        hdl = c(hDL)
        sdl = torch.zeros_like(hdl) if sDL is None else c(sDL)
        nc, b = hdl.shape
        pieces += [hdl.reshape(-1), sdl.reshape(-1)]
        lead.nc, lead.b, lead.hdl, lead.sdl = nc, b, 4 * n * n, 4 * n * n + nc * b
        if gsig.shape[-2:] != (nc, nc):
            raise ValueError(f"dL/dSigma {tuple(gsig.shape)} is not [B, {nc}, {nc}]")
    elif gsig.shape[-2:] != (n, n):
        raise ValueError(f"dL/dSigma {tuple(gsig.shape)} is not [B, {n}, {n}]")
    E = np.asarray(torch.as_tensor(E).detach().cpu().numpy(), dtype=np.complex128).reshape(-1)
    if E.shape[0] != B or gs.shape[-2:] != (n, n) or gsig.ndim != 3 or gsig.shape[0] != B:
        raise ValueError(f"{E.shape[0]} energies, g_s {tuple(gs.shape)} and dL/dSigma {tuple(gsig.shape)} "
                         f"for a {n}-wide lead: one [n, n] g_s and one dL/dSigma per energy")
    _lib.require_cuda()
    lib = _lib.load()
    arena = torch.cat(pieces)
    items = np.zeros(B, dtype=_lib.LEADADJ_ITEM_DTYPE)
    items["e_re"], items["e_im"] = E.real, E.imag
    items["gs"] = gs.data_ptr() + np.arange(B, dtype=np.uint64) * (n * n * 16)
    items["gsig"] = gsig.data_ptr() + np.arange(B, dtype=np.uint64) * (gsig.shape[-1] * gsig.shape[-2] * 16)
    items_t = _u8(items, dev)
    grad = torch.empty(4 * n * n + 2 * nc * b, dtype=C128, device=dev)
    status = torch.empty(B, dtype=torch.int32, device=dev)
    iters = torch.empty(B, dtype=torch.int32, device=dev)
    p = _lib.NegfLeadAdjProblem()
    p.lead, p.arena, p.items, p.n_items, p.form = lead, arena.data_ptr(), items_t.data_ptr(), B, int(form)
    p.eta, p.tol, p.max_iter = float(eta), float(tol), int(max_iter)
    p.n_slots = max(1, min(B, lib.negf_sm_count()))
    p.grad, p.status, p.iters = grad.data_ptr(), status.data_ptr(), iters.data_ptr()
    need = lib.negf_lead_adjoint_scratch_bytes(ctypes.byref(p))
    scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    p.scratch, p.scratch_bytes = scratch.data_ptr(), scratch.numel()
    _lib.check(lib.negf_lead_adjoint_run(ctypes.byref(p), _lib.stream_handle(stream)), "negf_lead_adjoint_run")
    st = status.cpu().numpy()
    if info is not None:
        info["iters"] = iters.cpu().numpy()
    if (st == _lib.NEGF_ERR_SINGULAR).any():
        raise torch.linalg.LinAlgError("lead adjoint: singular g_s or (zS - H - tau g_s tau')")
    if (st != _lib.NEGF_OK).any():
        raise _lib.NegfError("lead adjoint: non-finite doubling (the decimation fixed point is not contractive)")
    n2 = n * n
    out = [grad[i * n2:(i + 1) * n2].view(n, n) for i in range(4)]
    if form == 0:
        o = 4 * n2
        out += [grad[o:o + nc * b].view(nc, b), grad[o + nc * b:o + 2 * nc * b].view(nc, b) if sDL is not None else None]
    else:
        out += [None, None]
    return tuple(out)
