"""Fused T(E)/DOS sweep through ``negf_rgf_run_static`` (include/negf_b200.h).

For callers that cannot allocate device memory while the sweep runs (a host
transport code that owns the GPU through its own pool, or a plugin that only
receives input and output buffers): the library takes its scratch from a fixed
64 MiB array per GPU instead of a caller buffer.  The descriptor tables and
the output tensors are still the caller's; these helpers build them with torch
before the call, the C entry point itself allocates nothing.

Every call runs with the geometry's GPU current and waits for the stream it
launched on before it returns, so the descriptor tables it releases are no
longer read by the kernel.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .rgf_plan import Geometry

NEGF_ERR_SCRATCH_LIMIT = -4


def _bind(lib):
    lib.negf_rgf_run_static.restype = ctypes.c_int
    lib.negf_rgf_run_static.argtypes = [ctypes.POINTER(_lib.NegfRgfProblem), ctypes.c_void_p]
    lib.negf_rgf_static_scratch_bytes.restype = ctypes.c_size_t
    lib.negf_rgf_static_scratch_bytes.argtypes = []
    lib.negf_rgf_static_slots.restype = ctypes.c_int
    lib.negf_rgf_static_slots.argtypes = [ctypes.POINTER(_lib.NegfRgfProblem)]
    return lib


def static_scratch_bytes():
    return int(_bind(_lib.load()).negf_rgf_static_scratch_bytes())


def static_slots(prob):
    """Work slots ``negf_rgf_run_static`` runs for the problem ``prob`` (a NegfRgfProblem), or a
    negative status when even one slot does not fit."""
    return int(_bind(_lib.load()).negf_rgf_static_slots(ctypes.byref(prob)))


def _launch(lib, prob, dev, stream):
    """negf_rgf_run_static on ``dev`` (made current) and ``stream`` (default: its current stream);
    waits for that stream.  Returns the call-level status."""
    with torch.cuda.device(dev):
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        code = lib.negf_rgf_run_static(ctypes.byref(prob), ctypes.c_void_p(s.cuda_stream))
        s.synchronize()
    return code


def run_plan_static(plan, stream=None):
    """Run a deferred sweep (``rgf_plan.run(..., defer=True)``) with the library's static scratch
    in place of the plan's own; any output selection of the plan.  Returns (result, code)."""
    lib = _bind(_lib.load())
    dev = plan.result.status.device
    code = _launch(lib, plan.prob, dev, stream) if plan.n_items else 0
    return plan.result, code


def transmission_dos_static(geom: Geometry, energy: torch.Tensor, left_se: torch.Tensor,
                            right_se: torch.Tensor, eta=0.0, E_ref=0.0, n_slots=None, stream=None):
    """T(E) and DOS of the single device in ``geom`` at ``energy`` ([B]); returns (T, DOS, status, code).

    ``code`` is the call-level status of negf_rgf_run_static (0 on success).  The call runs on
    ``geom.device`` (made current for the call) and on ``stream`` if given, else that device's
    current stream.
    """
    _lib.require_cuda()
    lib = _bind(_lib.load())
    if len(geom.devs) != 1:
        raise ValueError("one device per call")
    dev = geom.device
    B = int(energy.shape[0])
    seL = left_se.to(device=dev, dtype=torch.complex128).contiguous()
    seR = right_se.to(device=dev, dtype=torch.complex128).contiguous()
    z = energy.to(torch.complex128).cpu().numpy().reshape(-1) + complex(E_ref) + 1j * float(eta)
    rows = np.arange(B, dtype=np.int64)
    items = np.zeros(B, dtype=_lib.ITEM_DTYPE)
    items["row"] = rows
    items["z_re"], items["z_im"] = z.real, z.imag
    nsl, nsr = int(seL.shape[-1]), int(seR.shape[-1])
    items["se_l"] = seL.data_ptr() + rows * nsl * nsl * 16
    items["se_r"] = seR.data_ptr() + rows * nsr * nsr * 16
    items["nse_l"], items["nse_r"] = nsl, nsr
    items["out"] = rows
    u8 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    blocks_t, devs_t, items_t = u8(geom.blocks), u8(geom.devs), u8(items)
    T = torch.empty(B, dtype=torch.float64, device=dev)
    D = torch.empty(B, dtype=torch.float64, device=dev)
    status = torch.empty(B, dtype=torch.int32, device=dev)
    p = _lib.NegfRgfProblem()
    p.blocks, p.devices, p.items = blocks_t.data_ptr(), devs_t.data_ptr(), items_t.data_ptr()
    p.n_items, p.max_n, p.max_g_slab = B, geom.max_n, geom.max_g_slab
    p.hs = geom.hs.data_ptr()
    p.trans, p.dos, p.status = T.data_ptr(), D.data_ptr(), status.data_ptr()
    p.flags = _lib.TRANS | _lib.DOS
    with torch.cuda.device(dev):
        p.n_slots = n_slots or max(1, min(B, lib.negf_sm_count()))
    code = _launch(lib, p, dev, stream)
    del blocks_t, devs_t, items_t
    return T, D, status, code
