"""Host-side planner for the batched RGF kernel (``negf_rgf_run``).

Packs one or more block-tridiagonal devices into a single complex128 arena on
the GPU, lays out the requested outputs, builds the block / device / item
descriptor tables and launches the persistent sweep.  Every (device, energy)
pair is one work item; items are handed to the kernel largest-first so that
uneven batches (different block sizes and lengths) balance across the SMs.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib

C128 = torch.complex128


@dataclass
class DeviceBlocks:
    """One BTD device: 2-D complex blocks, ``hu/hl/su/sl`` have K-1 entries."""
    hd: Sequence[torch.Tensor]
    hu: Sequence[torch.Tensor]
    hl: Sequence[torch.Tensor]
    sd: Sequence[torch.Tensor]
    su: Sequence[torch.Tensor]
    sl: Sequence[torch.Tensor]

    @property
    def dims(self):
        return [int(h.shape[-1]) for h in self.hd]


class Geometry:
    """Packed H/S arena + block table for a list of devices (energy independent).

    Build once per k-point (or per set of devices) and reuse across energy
    batches; this mirrors the reference caching H/S per (k, V)
    (negf/device_property.py:179-224).
    """

    def __init__(self, devices: List[DeviceBlocks], device="cuda", detect_zero_offdiag=True):
        dev = torch.device(device)
        self.device = dev
        self.devices = devices
        blocks, devs, copies = [], [], []
        offdiag = []  # (block index, field, arena offset, numel) of H/S coupling blocks
        cursor = 0

        def put(t):
            nonlocal cursor
            off = cursor
            copies.append((off, t))
            cursor += t.numel()
            return off

        self.max_n = 0
        self.max_g_slab = 0
        for d in devices:
            K = len(d.hd)
            if not (len(d.sd) == K and len(d.hu) == len(d.hl) == len(d.su) == len(d.sl) == K - 1):
                raise ValueError("inconsistent block lists")
            dims = d.dims
            blk0 = len(blocks)
            g = 0
            orb = 0
            gc = 0
            gu = 0
            for q in range(K):
                n = dims[q]
                if tuple(d.hd[q].shape[-2:]) != (n, n) or tuple(d.sd[q].shape[-2:]) != (n, n):
                    raise ValueError(f"block {q}: H/S must be square [{n},{n}]")
                b = np.zeros((), dtype=_lib.BLOCK_DTYPE)
                b["n"] = n
                b["n_next"] = dims[q + 1] if q + 1 < K else 0
                b["hd"] = put(d.hd[q])
                b["sd"] = put(d.sd[q])
                b["sdT"] = put(d.sd[q].mT)
                for name in ("hu", "su", "hl", "sl", "suT", "slT"):
                    b[name] = -1
                if q + 1 < K:
                    nn = dims[q + 1]
                    for name, lst, shape in (("hu", d.hu, (n, nn)), ("su", d.su, (n, nn)),
                                             ("hl", d.hl, (nn, n)), ("sl", d.sl, (nn, n))):
                        t = lst[q]
                        if tuple(t.shape[-2:]) != shape:
                            raise ValueError(f"{name}[{q}] has shape {tuple(t.shape)}, expected {shape}")
                        b[name] = put(t)
                        offdiag.append((len(blocks), name, int(b[name]), t.numel()))
                    for name, t in (("suT", d.su[q].mT), ("slT", d.sl[q].mT)):
                        b[name] = put(t)
                        offdiag.append((len(blocks), name, int(b[name]), t.numel()))
                b["orb0"] = orb
                b["g"] = g
                b["gc"] = gc
                b["gu"] = gu
                gc += n * dims[-1]
                if q + 1 < K:
                    gu += n * dims[q + 1]
                for f in ("o_grd", "o_grl", "o_gru", "o_grlc", "o_grleft", "o_gnd", "o_gnl", "o_gnu",
                          "o_ginleft", "s_in", "o_gpd", "o_gpl", "o_gpu", "o_gipleft", "s_out"):
                    b[f] = -1
                blocks.append(b)
                g += n * n
                orb += n
                self.max_n = max(self.max_n, n)
            dv = np.zeros((), dtype=_lib.DEVICE_DTYPE)
            dv["n_blocks"] = K
            dv["blk0"] = blk0
            dv["n_orb"] = orb
            dv["o_gtrans"] = -1
            dv["g_slab"] = g
            devs.append(dv)
            self.max_g_slab = max(self.max_g_slab, g)
            self.col_slab = max(getattr(self, "col_slab", 0), gc)
            self.u_slab = max(getattr(self, "u_slab", 0), gu)
        if self.max_n > _lib.NEGF_MAX_BLOCK:
            raise ValueError(f"block size {self.max_n} exceeds the supported maximum {_lib.NEGF_MAX_BLOCK}")
        # one host->device copy per block straight into the arena
        self.hs = torch.empty(max(cursor, 1), dtype=C128, device=dev)
        for off, t in copies:
            src = t.detach()
            if src.dtype != C128:
                src = src.to(C128)
            self.hs[off:off + src.numel()].view(src.shape).copy_(src, non_blocking=True)
        self.blocks = np.array(blocks, dtype=_lib.BLOCK_DTYPE)
        self.devs = np.array(devs, dtype=_lib.DEVICE_DTYPE)
        if detect_zero_offdiag and offdiag:
            # zero coupling blocks (orthogonal basis: su = sl = 0) are skipped by the kernel
            amax = torch.stack([self.hs[o:o + n].abs().amax() for _, _, o, n in offdiag])
            for (bi, name, _, _), z in zip(offdiag, (amax == 0).tolist()):
                if z:
                    self.blocks[bi][name] = -1

    @property
    def n_orb(self):
        return [int(x) for x in self.devs["n_orb"]]


def check_status(status: torch.Tensor):
    """Raise for the first failing item of a per-item status vector."""
    st = status.cpu()
    if (st != 0).any():
        bad = int((st != 0).nonzero()[0, 0])
        code = int(st[bad])
        if code == _lib.NEGF_ERR_SINGULAR:
            raise torch.linalg.LinAlgError(
                f"RGF: a left-connected block is singular (item {bad}); the matrix is not invertible")
        if code == _lib.NEGF_ERR_TIMEOUT:
            raise _lib.NegfError(f"RGF: a tensor-core completion wait expired (item {bad})")
        raise _lib.NegfError(f"RGF failed for item {bad} with status {code}")


@dataclass
class RgfPlan:
    """A prepared sweep (``run(..., defer=True)``): descriptors, scratch and outputs stay allocated."""
    prob: object
    keep: list
    n_items: int
    result: "RgfResult"

    def launch(self, stream=None):
        """Enqueue the sweep on ``stream`` (default: the current stream).  No host synchronisation and
        no allocation, so the call can be captured in a CUDA graph once the plan has run eagerly."""
        if self.n_items:
            _lib.check(_lib.load().negf_rgf_run(ctypes.byref(self.prob), _lib.stream_handle(stream)),
                       "negf_rgf_run")

    def check(self):
        if self.n_items:
            check_status(self.result.status)


@dataclass
class RgfResult:
    trans: Optional[torch.Tensor]    # [n_items] T(E), item order = device-major, energy-minor
    orb_dos: Optional[torch.Tensor]  # concatenated per-item [n_orb] -Im diag(GS)/pi
    dos: Optional[torch.Tensor]      # [n_items] DOS with spin factor 2
    status: torch.Tensor
    blocks: list                     # per device: tag -> list of [B, ...] tensors (tensor for g_trans)
    phase_cycles: Optional[torch.Tensor] = None  # [n_slots, NEGF_PHASES] SM cycles per phase
    orb_g: Optional[torch.Tensor] = None    # concatenated per-item [n_orb] diag(G_qq) (complex)
    orb_ar: Optional[torch.Tensor] = None   # concatenated per-item [n_orb] diag(G_qN Gamma_R G_qN^H)
    grads: Optional[dict] = None            # adjoint: block gradients and per-energy dT/dSigma


_FAMILY = {  # output tag -> (flag, block field, shape fn (n_q, n_next, n_last))
    "grd": (_lib.OUT_GRD, "o_grd", lambda n, nn, nl: (n, n), False),
    "grl": (_lib.OUT_GRL, "o_grl", lambda n, nn, nl: (nn, n), True),
    "gru": (_lib.OUT_GRU, "o_gru", lambda n, nn, nl: (n, nn), True),
    "gr_lc": (_lib.OUT_GR_LC, "o_grlc", lambda n, nn, nl: (n, nl), False),
    "gr_left": (_lib.OUT_GR_LEFT, "o_grleft", lambda n, nn, nl: (n, n), False),
    "gnd": (_lib.LESSER, "o_gnd", lambda n, nn, nl: (n, n), False),
    "gnl": (_lib.LESSER, "o_gnl", lambda n, nn, nl: (nn, n), True),
    "gnu": (_lib.LESSER, "o_gnu", lambda n, nn, nl: (n, nn), True),
    "gin_left": (_lib.LESSER, "o_ginleft", lambda n, nn, nl: (n, n), False),
    "gpd": (_lib.GREATER, "o_gpd", lambda n, nn, nl: (n, n), False),
    "gpl": (_lib.GREATER, "o_gpl", lambda n, nn, nl: (nn, n), True),
    "gpu": (_lib.GREATER, "o_gpu", lambda n, nn, nl: (n, nn), True),
    "gip_left": (_lib.GREATER, "o_gipleft", lambda n, nn, nl: (n, n), False),
}


@_lib.on_given_stream
def run(geom: Geometry, energies: List[torch.Tensor], se_l: List[Optional[torch.Tensor]],
        se_r: List[Optional[torch.Tensor]], eta=0.0, E_ref=0.0, outputs=("g_trans", "grd", "grl", "gru"),
        trans=False, orb_dos=False, dos=False, orb_g=False, orb_ar=False,
        s_in: Optional[List[List[Optional[torch.Tensor]]]] = None,
        s_out: Optional[List[List[Optional[torch.Tensor]]]] = None,
        n_slots=None, check=True, stream=None, phase=False, events=None, adjoint_w=None, adjoint_w_dos=None,
        precision="fp64", refine=False, refine_steps=1, defer=False, inv_ob=None, inverse=None, checkpoint=0):
    """Run the batched sweep.

    ``energies[d]`` is a 1-D tensor of B_d energies for device d; ``se_l[d]``
    / ``se_r[d]`` are ``[B_d, n, n]`` self-energies (or None).  ``outputs``
    names the block tensors to materialise (tags of recursive_gf's tuple);
    ``s_in[d]`` is the per-block list of ``[B_d, n_q, n_q]`` lesser inputs
    (None entries are zero blocks) and switches the lesser sweep on; ``s_out``
    (same layout) switches the greater sweep on (gpd, gpl, gpu, gip_left).
    ``events=(start, end)`` are CUDA events recorded on the launch stream
    immediately around the kernel (device time of the sweep alone).
    ``adjoint_w`` ([B] weights of T(E), single device) switches the adjoint
    on: the result carries d(sum w T)/d(hd, hu, hl, sd, su, sl) and per-energy
    dT/dSigma_L, dT/dSigma_R weighted by w (torch's complex convention).
    ``adjoint_w_dos`` ([B] weights of DOS(E), with or without ``adjoint_w``)
    adds the gradient of sum w_d DOS to the same results: the summed onsite
    density over the energies when the weights are occupation x quadrature.
    ``precision="mixed"`` runs every block product on the tcgen05 3xTF32 GEMM
    (FP32-accurate products; pivoting, panels and storage stay FP64);
    ``refine=True`` (with ``trans``) adds ``refine_steps`` FP64-residual
    refinement steps of the column G_{:,N} that T(E) is read from.
    ``inverse="block"`` inverts each Schur complement by recursive
    2x2 blocks (pivoted Gauss-Jordan only on 64-wide leaves, all updates on
    the block GEMM), which needs nonsingular leading sub-blocks: eta > 0
    guarantees them for Hermitian H, positive-definite S and retarded
    self-energies.  Every block inverse is checked by a residual probe and
    an item whose check fails is redone with the pivoted Gauss-Jordan
    inverse, so other inputs (eta = 0, arbitrary matrices) stay exact.
    ``inverse="gj"`` uses the pivoted Gauss-Jordan inverse throughout; by
    default the autotuned scheme for this GPU, block size and precision, else
    "block".
    ``inv_ob`` is the inverse's outer block width (32..512); by default the
    autotuned value for this GPU, block size and precision (``autotune.lookup``),
    else 128.
    ``checkpoint`` (adjoint only): 0 keeps every left-connected g_q of an item in its scratch slot;
    s > 0 keeps g_0, g_s, g_2s, ... and one segment of s blocks, recomputing each segment from its
    checkpoint when the backward sweep and the adjoint pass reach it (``"sqrt"``: s = ceil(sqrt(K))),
    so the g storage per slot is (ceil(K/s) + s) max_n^2 instead of sum n_q^2 (twice that with
    ``adjoint_w_dos``, whose z-tangents are checkpointed alike); results are identical.
    ``defer=True`` builds everything but launches nothing and returns an
    ``RgfPlan``: its ``launch()`` re-runs the sweep on the same descriptors,
    scratch and output tensors (a queue reset and one kernel, so it can be
    captured in a CUDA graph) and its ``result`` views the outputs.
    """
    if precision not in ("fp64", "mixed"):
        raise ValueError(f"precision must be 'fp64' or 'mixed', not {precision!r}")
    _lib.require_cuda()
    lib = _lib.load()
    dev = geom.device
    nd = len(geom.devs)
    outputs = set(outputs)
    lesser = s_in is not None
    if lesser:
        outputs |= {"gnd", "gnl", "gnu", "gin_left"}
    greater = s_out is not None
    if greater:
        outputs |= {"gpd", "gpl", "gpu", "gip_left"}
    flags = 0
    for tag in outputs:
        if tag == "g_trans":
            flags |= _lib.OUT_GTRANS
        elif tag in _FAMILY:
            flags |= _FAMILY[tag][0]
        else:
            raise ValueError(f"unknown output {tag}")
    if trans:
        flags |= _lib.TRANS
    if orb_dos:
        flags |= _lib.ORB_DOS
    if dos:
        flags |= _lib.DOS
    if orb_g:
        flags |= _lib.ORB_GDIAG
    if orb_ar:
        flags |= _lib.ORB_AR
    if lesser:
        flags |= _lib.LESSER
    if greater:
        flags |= _lib.GREATER
    adjoint = adjoint_w is not None or adjoint_w_dos is not None
    if adjoint_w_dos is not None:
        flags |= _lib.ADJ_DOS
    if adjoint:
        if nd != 1:
            raise ValueError("the adjoint runs on a single device")
        flags |= _lib.ADJOINT | _lib.TRANS
        trans = True
    if precision == "mixed":
        flags |= _lib.MIXED
    if refine:
        if not trans:
            raise ValueError("refine improves T(E): it needs trans=True")
        flags |= _lib.REFINE
    ckpt = 0
    if checkpoint:
        if not adjoint:
            raise ValueError("checkpoint applies to the adjoint pass (adjoint_w / adjoint_w_dos)")
        if refine or lesser or greater or "gr_left" in outputs:
            raise ValueError("checkpointing does not combine with refine, lesser, greater or gr_left outputs")
        K0 = int(geom.devs[0]["n_blocks"])
        ckpt = int(np.ceil(np.sqrt(K0))) if checkpoint == "sqrt" else int(checkpoint)
        if ckpt < 1:
            raise ValueError(f"checkpoint interval must be >= 1, not {checkpoint!r}")

    blocks = geom.blocks.copy()
    devs = geom.devs.copy()
    out_cursor = 0
    layout = []  # per device: tag -> list of (offset, shape, B)
    sin_pieces = []
    sin_cursor = 0
    sout_pieces = []
    sout_cursor = 0
    item_parts, cost_parts = [], []
    keep_alive = []
    orb_cursor = 0
    item_cursor = 0
    for d in range(nd):
        K = int(devs[d]["n_blocks"])
        b0 = int(devs[d]["blk0"])
        dims = [int(blocks[b0 + q]["n"]) for q in range(K)]
        E = energies[d]
        B = int(E.shape[0])
        lay = {}
        nl = dims[-1]
        for tag in ("grd", "grl", "gru", "gr_lc", "gr_left", "gnd", "gnl", "gnu", "gin_left",
                    "gpd", "gpl", "gpu", "gip_left"):
            if tag not in outputs:
                continue
            _, field, shp, offd = _FAMILY[tag]
            lst = []
            for q in range(K - 1 if offd else K):
                nn = dims[q + 1] if q + 1 < K else 0
                shape = shp(dims[q], nn, nl)
                blocks[b0 + q][field] = out_cursor
                lst.append((out_cursor, shape, B))
                out_cursor += B * shape[0] * shape[1]
            lay[tag] = lst
        if "g_trans" in outputs:
            devs[d]["o_gtrans"] = out_cursor
            lay["g_trans"] = (out_cursor, (dims[0], nl), B)
            out_cursor += B * dims[0] * nl
        layout.append(lay)
        # self-energies are read in place: one device pointer per item
        ptr_l = ptr_r = 0
        nsl = nsr = 0
        stride_l = stride_r = 0
        for side in (0, 1):
            t = (se_l if side == 0 else se_r)[d]
            if t is None:
                continue
            t = t.to(device=dev, dtype=C128)
            if t.ndim == 2:
                t = t.unsqueeze(0).expand(B, -1, -1)
            if t.shape[0] != B or t.shape[-1] != t.shape[-2]:
                raise ValueError(f"self-energy of shape {tuple(t.shape)} does not match {B} energies")
            t = t.contiguous() if t.stride(0) != 0 else t[:1].contiguous()
            keep_alive.append(t)
            ns = int(t.shape[-1])
            stride = ns * ns * 16 if t.shape[0] == B and t.stride(0) != 0 else 0
            if side == 0:
                ptr_l, nsl, stride_l = t.data_ptr(), ns, stride
            else:
                ptr_r, nsr, stride_r = t.data_ptr(), ns, stride
        if lesser:
            for q in range(K):
                t = s_in[d][q]
                if t is None:
                    continue
                t = t.to(device=dev, dtype=C128)
                if t.ndim == 2:
                    t = t.unsqueeze(0).expand(B, -1, -1)
                if tuple(t.shape) != (B, dims[q], dims[q]):
                    raise ValueError(f"s_in[{q}] has shape {tuple(t.shape)}, expected {(B, dims[q], dims[q])}")
                blocks[b0 + q]["s_in"] = sin_cursor
                sin_pieces.append(t.reshape(-1))
                sin_cursor += B * dims[q] * dims[q]
        if greater:
            for q in range(K):
                t = s_out[d][q]
                if t is None:
                    continue
                t = t.to(device=dev, dtype=C128)
                if t.ndim == 2:
                    t = t.unsqueeze(0).expand(B, -1, -1)
                if tuple(t.shape) != (B, dims[q], dims[q]):
                    raise ValueError(f"s_out[{q}] has shape {tuple(t.shape)}, expected {(B, dims[q], dims[q])}")
                blocks[b0 + q]["s_out"] = sout_cursor
                sout_pieces.append(t.reshape(-1))
                sout_cursor += B * dims[q] * dims[q]
        z = (E.to(torch.complex128).cpu().numpy().reshape(-1) + complex(E_ref)) + 1j * float(eta)
        n_orb = int(devs[d]["n_orb"])
        rows = np.arange(B, dtype=np.int64)
        it = np.zeros(B, dtype=_lib.ITEM_DTYPE)
        if adjoint:
            if adjoint_w is not None:
                it["w_t"] = torch.as_tensor(adjoint_w, dtype=torch.float64).reshape(-1).cpu().numpy()
            if adjoint_w_dos is not None:
                it["w_d"] = torch.as_tensor(adjoint_w_dos, dtype=torch.float64).reshape(-1).cpu().numpy()
            gseL_t = torch.empty((B, nsl, nsl), dtype=C128, device=dev) if nsl else None
            gseR_t = torch.empty((B, nsr, nsr), dtype=C128, device=dev) if nsr else None
            keep_alive += [x for x in (gseL_t, gseR_t) if x is not None]
            it["gse_l"] = (gseL_t.data_ptr() + rows * nsl * nsl * 16) if nsl else 0
            it["gse_r"] = (gseR_t.data_ptr() + rows * nsr * nsr * 16) if nsr else 0
        it["dev"] = d
        it["row"] = rows
        it["z_re"] = z.real
        it["z_im"] = z.imag
        it["se_l"] = (ptr_l + rows * stride_l) if ptr_l else 0
        it["se_r"] = (ptr_r + rows * stride_r) if ptr_r else 0
        it["nse_l"] = nsl
        it["nse_r"] = nsr
        it["out"] = item_cursor + rows
        it["orb"] = orb_cursor + rows * n_orb
        item_parts.append(it)
        cost_parts.append(np.full(B, sum(n ** 3 for n in dims), dtype=np.int64))
        item_cursor += B
        orb_cursor += B * n_orb
    n_items = item_cursor
    if n_items:
        all_items = np.concatenate(item_parts)
        # largest work first; stable, so equal costs keep energy order
        item_arr = all_items[np.argsort(-np.concatenate(cost_parts), kind="stable")]
    else:
        item_arr = np.zeros(0, dtype=_lib.ITEM_DTYPE)

    u8 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    blocks_t = u8(blocks)
    devs_t = u8(devs)
    items_t = u8(item_arr) if n_items else torch.zeros(1, dtype=torch.uint8, device=dev)
    sin_t = torch.cat(sin_pieces) if sin_pieces else torch.zeros(1, dtype=C128, device=dev)
    sout_t = torch.cat(sout_pieces) if sout_pieces else torch.zeros(1, dtype=C128, device=dev)
    out_t = torch.empty(max(out_cursor, 1), dtype=C128, device=dev)
    trans_t = torch.empty(max(item_cursor, 1), dtype=torch.float64, device=dev) if trans else None
    orb_t = torch.empty(max(orb_cursor, 1), dtype=torch.float64, device=dev) if orb_dos else None
    dos_t = torch.empty(max(item_cursor, 1), dtype=torch.float64, device=dev) if dos else None
    orbg_t = torch.empty(max(orb_cursor, 1), dtype=C128, device=dev) if orb_g else None
    orbar_t = torch.zeros(max(orb_cursor, 1), dtype=torch.float64, device=dev) if orb_ar else None
    status_t = torch.empty(max(item_cursor, 1), dtype=torch.int32, device=dev)
    if n_slots is None:
        n_slots = max(1, min(n_items, lib.negf_sm_count()))
    prob = _lib.NegfRgfProblem()
    prob.blocks = blocks_t.data_ptr()
    prob.devices = devs_t.data_ptr()
    prob.items = items_t.data_ptr()
    prob.n_items = n_items
    prob.max_n = geom.max_n
    prob.max_g_slab = geom.max_g_slab
    prob.hs = geom.hs.data_ptr()
    prob.s_in = sin_t.data_ptr()
    prob.s_out = sout_t.data_ptr()
    prob.out = out_t.data_ptr()
    prob.trans = trans_t.data_ptr() if trans else None
    prob.orb_dos = orb_t.data_ptr() if orb_dos else None
    prob.dos = dos_t.data_ptr() if dos else None
    prob.orb_g = orbg_t.data_ptr() if orb_g else None
    prob.orb_ar = orbar_t.data_ptr() if orb_ar else None
    prob.status = status_t.data_ptr()
    prob.flags = flags
    prob.n_slots = n_slots
    if refine or adjoint:
        prob.col_slab = max(int(geom.col_slab), 1)
    prob.refine_steps = int(refine_steps)
    if ckpt:
        prob.ckpt = ckpt
        prob.ckpt_blocks = int(geom.devs[0]["n_blocks"])
    if inv_ob is None or inverse is None:
        from . import autotune
        tuned = autotune.lookup(geom.max_n, precision)
        if inv_ob is None:
            inv_ob = tuned.get("inv_ob", 0)
        if inverse is None:
            inverse = tuned.get("inverse", "block")
    prob.inv_ob = int(inv_ob)
    if inverse not in ("gj", "block"):
        raise ValueError(f"inverse must be 'gj' or 'block', not {inverse!r}")
    prob.inv_mode = 1 if inverse == "block" else 0
    need = lib.negf_rgf_scratch_bytes(ctypes.byref(prob))
    scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    prob.scratch = scratch.data_ptr()
    prob.scratch_bytes = scratch.numel()
    grad_t = None
    if adjoint:
        g_slab = int(geom.devs[0]["g_slab"])
        grad_slab = 2 * g_slab + 4 * int(geom.u_slab)
        grad_t = torch.zeros((n_slots, max(grad_slab, 1)), dtype=C128, device=dev)
        prob.grad = grad_t.data_ptr()
        prob.grad_slab = grad_slab
        need = lib.negf_rgf_scratch_bytes(ctypes.byref(prob))
        if need > scratch.numel():
            scratch = torch.empty(need, dtype=torch.uint8, device=dev)
            prob.scratch = scratch.data_ptr()
            prob.scratch_bytes = scratch.numel()
    phase_t = None
    if phase:
        phase_t = torch.zeros((n_slots, len(_lib.PHASES)), dtype=torch.int64, device=dev)
        prob.phase_cycles = phase_t.data_ptr()
    if defer:
        if adjoint:
            raise ValueError("the adjoint pass is not available as a deferred plan")
        keep = [blocks_t, devs_t, items_t, sin_t, sout_t, out_t, trans_t, orb_t, dos_t, orbg_t, orbar_t, status_t,
                scratch, phase_t, geom.hs] + keep_alive
    # otherwise the staging tensors may be released on return: the caching
    # allocator only hands their memory to work ordered after this launch
    if not defer:
        if events is not None:
            events[0].record(stream)
        _lib.check(lib.negf_rgf_run(ctypes.byref(prob), _lib.stream_handle(stream)), "negf_rgf_run")
        if events is not None:
            events[1].record(stream)

    res_blocks = []
    for d in range(nd):
        lay = layout[d]
        dd = {}
        for tag, v in lay.items():
            if tag == "g_trans":
                off, shape, B = v
                dd[tag] = out_t[off:off + B * shape[0] * shape[1]].view(B, *shape)
            else:
                dd[tag] = [out_t[off:off + B * s[0] * s[1]].view(B, *s) for off, s, B in v]
        res_blocks.append(dd)
    if defer:
        return RgfPlan(prob=prob, keep=keep, n_items=n_items, result=RgfResult(
            trans=trans_t[:item_cursor] if trans else None, orb_dos=orb_t[:orb_cursor] if orb_dos else None,
            dos=dos_t[:item_cursor] if dos else None, status=status_t[:item_cursor], blocks=res_blocks,
            phase_cycles=phase_t, orb_g=orbg_t[:orb_cursor] if orb_g else None,
            orb_ar=orbar_t[:orb_cursor] if orb_ar else None))
    if check and n_items:
        check_status(status_t[:n_items])
    grads = None
    if adjoint:
        gsum = grad_t.sum(0)
        K = int(geom.devs[0]["n_blocks"])
        dims = [int(geom.blocks[q]["n"]) for q in range(K)]
        g_slab = int(geom.devs[0]["g_slab"])
        u_slab = int(geom.u_slab)
        base = {"hd": 0, "sd": g_slab, "hu": 2 * g_slab, "su": 2 * g_slab + u_slab,
                "hl": 2 * g_slab + 2 * u_slab, "sl": 2 * g_slab + 3 * u_slab}
        grads = {}
        for name in ("hd", "sd"):
            grads[name] = [gsum[base[name] + int(geom.blocks[q]["g"]):][:dims[q] ** 2].view(dims[q], dims[q])
                           for q in range(K)]
        for name in ("hu", "su"):
            grads[name] = [gsum[base[name] + int(geom.blocks[q]["gu"]):][:dims[q] * dims[q + 1]]
                           .view(dims[q], dims[q + 1]) for q in range(K - 1)]
        for name in ("hl", "sl"):
            grads[name] = [gsum[base[name] + int(geom.blocks[q]["gu"]):][:dims[q] * dims[q + 1]]
                           .view(dims[q + 1], dims[q]) for q in range(K - 1)]
        grads["se_l"] = gseL_t
        grads["se_r"] = gseR_t
    return RgfResult(trans=trans_t[:item_cursor] if trans else None,
                     orb_dos=orb_t[:orb_cursor] if orb_dos else None,
                     dos=dos_t[:item_cursor] if dos else None,
                     status=status_t[:item_cursor], blocks=res_blocks, phase_cycles=phase_t,
                     orb_g=orbg_t[:orb_cursor] if orb_g else None,
                     orb_ar=orbar_t[:orb_cursor] if orb_ar else None, grads=grads)
