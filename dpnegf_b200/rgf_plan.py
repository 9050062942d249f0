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


def _flat(t, dev):
    return t.to(device=dev, dtype=C128).reshape(-1)


def _all_zero(ts, dev):
    """Which of the tensors are identically zero (one host sync for all)."""
    if not ts:
        return []
    m = torch.stack([t.to(dev).abs().amax() if t.numel() else torch.zeros((), dtype=torch.float64, device=dev)
                     for t in ts])
    return (m == 0).tolist()


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
        pieces, blocks, devs = [], [], []
        cursor = 0

        def put(t):
            nonlocal cursor
            off = cursor
            f = _flat(t, dev)
            pieces.append(f)
            cursor += f.numel()
            return off

        zero_flags = None
        if detect_zero_offdiag:
            offd = [t for d in devices for t in list(d.su) + list(d.sl) + list(d.hu) + list(d.hl)]
            zero_flags = iter(_all_zero(offd, dev))
        self.max_n = 0
        self.max_g_slab = 0
        for d in devices:
            K = len(d.hd)
            if not (len(d.sd) == K and len(d.hu) == len(d.hl) == len(d.su) == len(d.sl) == K - 1):
                raise ValueError("inconsistent block lists")
            dims = d.dims
            if zero_flags is not None:
                zsu = [next(zero_flags) for _ in d.su]
                zsl = [next(zero_flags) for _ in d.sl]
                zhu = [next(zero_flags) for _ in d.hu]
                zhl = [next(zero_flags) for _ in d.hl]
            else:
                zsu = zsl = zhu = zhl = [False] * (K - 1)
            blk0 = len(blocks)
            g = 0
            orb = 0
            for q in range(K):
                n = dims[q]
                if tuple(d.hd[q].shape[-2:]) != (n, n) or tuple(d.sd[q].shape[-2:]) != (n, n):
                    raise ValueError(f"block {q}: H/S must be square [{n},{n}]")
                b = np.zeros((), dtype=_lib.BLOCK_DTYPE)
                b["n"] = n
                b["n_next"] = dims[q + 1] if q + 1 < K else 0
                b["hd"] = put(d.hd[q])
                b["sd"] = put(d.sd[q])
                for name in ("hu", "su", "hl", "sl"):
                    b[name] = -1
                if q + 1 < K:
                    nn = dims[q + 1]
                    for name, lst, zl, shape in (("hu", d.hu, zhu, (n, nn)), ("su", d.su, zsu, (n, nn)),
                                                 ("hl", d.hl, zhl, (nn, n)), ("sl", d.sl, zsl, (nn, n))):
                        t = lst[q]
                        if tuple(t.shape[-2:]) != shape:
                            raise ValueError(f"{name}[{q}] has shape {tuple(t.shape)}, expected {shape}")
                        b[name] = -1 if zl[q] else put(t)
                b["orb0"] = orb
                b["g"] = g
                for f in ("o_grd", "o_grl", "o_gru", "o_grlc", "o_grleft", "o_gnd", "o_gnl", "o_gnu",
                          "o_ginleft", "s_in"):
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
        if self.max_n > _lib.NEGF_MAX_BLOCK:
            raise ValueError(f"block size {self.max_n} exceeds the supported maximum {_lib.NEGF_MAX_BLOCK}")
        self.hs = torch.cat(pieces) if pieces else torch.zeros(1, dtype=C128, device=dev)
        self.blocks = np.array(blocks, dtype=_lib.BLOCK_DTYPE)
        self.devs = np.array(devs, dtype=_lib.DEVICE_DTYPE)

    @property
    def n_orb(self):
        return [int(x) for x in self.devs["n_orb"]]


@dataclass
class RgfResult:
    trans: Optional[torch.Tensor]
    orb_dos: Optional[torch.Tensor]
    status: torch.Tensor
    blocks: dict  # per device: tag -> list of [B, ...] tensors (or tensor for g_trans)


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
}


def run(geom: Geometry, energies: List[torch.Tensor], se_l: List[Optional[torch.Tensor]],
        se_r: List[Optional[torch.Tensor]], eta=0.0, E_ref=0.0, outputs=("g_trans", "grd", "grl", "gru"),
        trans=False, orb_dos=False, s_in: Optional[List[List[Optional[torch.Tensor]]]] = None,
        n_slots=None, check=True, stream=None):
    """Run the batched sweep.

    ``energies[d]`` is a 1-D tensor of B_d energies for device d; ``se_l[d]``
    / ``se_r[d]`` are ``[B_d, n, n]`` self-energies (or None).  ``outputs``
    names the block tensors to materialise (tags of recursive_gf's tuple);
    ``s_in[d]`` is the per-block list of ``[B_d, n_q, n_q]`` lesser inputs
    (None entries are zero blocks) and switches the lesser sweep on.
    """
    _lib.require_cuda()
    lib = _lib.load()
    dev = geom.device
    nd = len(geom.devs)
    outputs = set(outputs)
    lesser = s_in is not None
    if lesser:
        outputs |= {"gnd", "gnl", "gnu", "gin_left"}
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
    if lesser:
        flags |= _lib.LESSER

    blocks = geom.blocks.copy()
    devs = geom.devs.copy()
    out_cursor = 0
    layout = []  # per device: tag -> list of (offset, shape, B)
    se_pieces, sin_pieces = [], []
    se_cursor = 0
    sin_cursor = 0
    items = []
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
        for tag in ("grd", "grl", "gru", "gr_lc", "gr_left", "gnd", "gnl", "gnu", "gin_left"):
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
        # self-energies
        sl_off = sr_off = -1
        nsl = nsr = 0
        if se_l[d] is not None:
            t = se_l[d].to(device=dev, dtype=C128).contiguous()
            if t.ndim == 2:
                t = t.unsqueeze(0).expand(B, -1, -1)
            nsl = int(t.shape[-1])
            sl_off = se_cursor
            se_pieces.append(t.reshape(-1))
            se_cursor += B * nsl * nsl
        if se_r[d] is not None:
            t = se_r[d].to(device=dev, dtype=C128).contiguous()
            if t.ndim == 2:
                t = t.unsqueeze(0).expand(B, -1, -1)
            nsr = int(t.shape[-1])
            sr_off = se_cursor
            se_pieces.append(t.reshape(-1))
            se_cursor += B * nsr * nsr
        if lesser:
            for q in range(K):
                t = s_in[d][q]
                if t is None:
                    continue
                t = t.to(device=dev, dtype=C128)
                if t.ndim == 2:
                    t = t.unsqueeze(0).expand(B, -1, -1)
                blocks[b0 + q]["s_in"] = sin_cursor
                sin_pieces.append(t.reshape(-1))
                sin_cursor += B * dims[q] * dims[q]
        z = (E.to(torch.complex128).cpu().numpy() + complex(E_ref)) + 1j * float(eta)
        n_orb = int(devs[d]["n_orb"])
        for b in range(B):
            it = np.zeros((), dtype=_lib.ITEM_DTYPE)
            it["dev"] = d
            it["row"] = b
            it["z_re"] = z[b].real
            it["z_im"] = z[b].imag
            it["se_l"] = -1 if sl_off < 0 else sl_off + b * nsl * nsl
            it["se_r"] = -1 if sr_off < 0 else sr_off + b * nsr * nsr
            it["nse_l"] = nsl
            it["nse_r"] = nsr
            it["out"] = item_cursor
            it["orb"] = orb_cursor
            items.append((sum(n ** 3 for n in dims), it))
            item_cursor += 1
            orb_cursor += n_orb
    n_items = len(items)
    # largest work first (stable: equal costs keep energy order)
    order = sorted(range(n_items), key=lambda i: -items[i][0])
    item_arr = np.array([items[i][1] for i in order], dtype=_lib.ITEM_DTYPE)

    u8 = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).to(dev)
    blocks_t = u8(blocks)
    devs_t = u8(devs)
    items_t = u8(item_arr) if n_items else torch.zeros(1, dtype=torch.uint8, device=dev)
    se_t = torch.cat(se_pieces) if se_pieces else torch.zeros(1, dtype=C128, device=dev)
    sin_t = torch.cat(sin_pieces) if sin_pieces else torch.zeros(1, dtype=C128, device=dev)
    out_t = torch.empty(max(out_cursor, 1), dtype=C128, device=dev)
    trans_t = torch.empty(max(item_cursor, 1), dtype=torch.float64, device=dev) if trans else None
    orb_t = torch.empty(max(orb_cursor, 1), dtype=torch.float64, device=dev) if orb_dos else None
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
    prob.se = se_t.data_ptr()
    prob.s_in = sin_t.data_ptr()
    prob.out = out_t.data_ptr()
    prob.trans = trans_t.data_ptr() if trans else None
    prob.orb_dos = orb_t.data_ptr() if orb_dos else None
    prob.status = status_t.data_ptr()
    prob.flags = flags
    prob.n_slots = n_slots
    need = lib.negf_rgf_scratch_bytes(ctypes.byref(prob))
    scratch = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
    prob.scratch = scratch.data_ptr()
    prob.scratch_bytes = scratch.numel()
    # the staging tensors may be released on return: the caching allocator
    # only hands their memory to work ordered after this launch on the stream
    _lib.check(lib.negf_rgf_run(ctypes.byref(prob), _lib.stream_handle(stream)), "negf_rgf_run")

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
    if check and n_items:
        st = status_t[:n_items].cpu()
        if (st != 0).any():
            bad = int((st != 0).nonzero()[0, 0])
            code = int(st[bad])
            if code == _lib.NEGF_ERR_SINGULAR:
                raise torch.linalg.LinAlgError(
                    f"RGF: a left-connected block is singular (item {bad}); the matrix is not invertible")
            raise _lib.NegfError(f"RGF failed for item {bad} with status {code}")
    return RgfResult(trans=trans_t[:item_cursor] if trans else None,
                     orb_dos=orb_t[:orb_cursor] if orb_dos else None,
                     status=status_t[:item_cursor], blocks=res_blocks)
