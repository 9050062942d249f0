"""Drop-in ``recursive_gf`` running the batched RGF sweep on the B200.

Same signature, argument meaning, tensor layouts and 14-tuple return as the
reference wrapper (negf/recursive_green_cal.py:324-477, tuple order of
``_pack_ans`` :299-321, scalar squeeze rule :380-393 and :480-491).  The
whole sweep is one launch of the CUDA kernel ``negf_rgf_run``; inputs that
live on the CPU are copied to the current CUDA device and the results copied
back, so a caller that passes host tensors gets host tensors.
"""
import torch

from . import rgf_plan

TAGS = ("g_trans", "gr_lc", "grd", "grl", "gru", "gr_left",
        "gnd", "gnl", "gnu", "gin_left", "gpd", "gpl", "gpu", "gip_left")


def _is3(t):
    return torch.is_tensor(t) and t.ndim == 3


def _bsel(t, b):
    """Energy row ``b`` of a per-energy block, or the block itself if 2-D."""
    if t is None or not torch.is_tensor(t):
        return t
    return t[b] if t.ndim == 3 else t


def recursive_gf(energy, hl, hd, hu, sd, su, sl, left_se, right_se, seP=None, E_ref=0.0, s_in=0, s_out=0,
                 eta=1e-5, need_lesser=False, need_greater=False, need_gr_lc=False, keep_gr_left=True):
    """Batched RGF (Anantram, Lundstrom, Nikonov, Proc. IEEE 96, 1511 (2008)).

    ``energy`` is a 0-d/scalar or 1-D ``[B]`` tensor; ``hd``/``sd`` are lists of
    K square blocks, ``hu``/``su`` (``[n_q, n_{q+1}]``) and ``hl``/``sl``
    (``[n_{q+1}, n_q]``) lists of K-1 blocks, each 2-D (shared by all energies)
    or 3-D ``[B, ...]``.  ``left_se``/``right_se`` are ``[B, n, n]`` (2-D for a
    scalar energy) and are added to the top-left / bottom-right corner of the
    first / last diagonal block.  ``s_in`` (list of K ``[B, n_q, n_q]``) feeds
    the lesser sweep when ``need_lesser``; ``s_out`` (same layout) feeds the
    greater sweep when ``need_greater``.  Returns the 14-tuple
    ``(g_trans, gr_lc, grd, grl, gru, gr_left, gnd, gnl, gnu, gin_left,
    gpd, gpl, gpu, gip_left)``; the batch dim is squeezed for scalar callers
    (``left_se`` 2-D).
    """
    if need_lesser:
        assert isinstance(s_in, list), "Lesser Green's function calculation requires s_in to be a list of coupling matrices"
    if need_greater:
        assert isinstance(s_out, list), "Greater Green's function calculation requires s_out to be a list of coupling matrices"

    out_dev = hd[0].device if torch.is_tensor(hd[0]) else torch.device("cpu")
    dev = out_dev if out_dev.type == "cuda" else torch.device("cuda", torch.cuda.current_device()
                                                              if torch.cuda.is_available() else 0)

    shift = energy + E_ref
    if not torch.is_tensor(shift):
        shift = torch.as_tensor(shift, dtype=torch.complex128)
    se_probe = left_se if isinstance(left_se, torch.Tensor) else right_se
    squeezed = isinstance(se_probe, torch.Tensor) and se_probe.ndim == 2
    if shift.ndim == 0:
        shift = shift.reshape(1)
    shift = shift.to(torch.complex128)
    B = int(shift.shape[0])
    K = len(hd)

    if seP is not None:  # added to the diagonal blocks as the reference does, numbers included (:411-414)
        hd = [h if p is None else h + (p.to(h.device) if torch.is_tensor(p) else p) for h, p in zip(hd, seP)]

    per_energy = any(_is3(t) for lst in (hd, hu, hl, sd, su, sl) for t in lst)
    if per_energy:
        devices = [rgf_plan.DeviceBlocks([_bsel(t, b) for t in hd], [_bsel(t, b) for t in hu],
                                         [_bsel(t, b) for t in hl], [_bsel(t, b) for t in sd],
                                         [_bsel(t, b) for t in su], [_bsel(t, b) for t in sl])
                   for b in range(B)]
        energies = [shift[b:b + 1] for b in range(B)]
    else:
        devices = [rgf_plan.DeviceBlocks(hd, hu, hl, sd, su, sl)]
        energies = [shift]

    def se_for(se, d):
        if not torch.is_tensor(se):
            return None
        if se.ndim == 2:
            return se.unsqueeze(0).expand(energies[d].shape[0], -1, -1)
        return se[d:d + 1] if per_energy else se

    geom = rgf_plan.Geometry(devices, device=dev)
    outputs = ["g_trans", "grd", "grl", "gru"]
    if need_gr_lc:
        outputs.append("gr_lc")
    if keep_gr_left:
        outputs.append("gr_left")

    def per_device(src):
        """Per-device lists of per-block [B_d, n, n] inputs (None = zero block)."""
        res = []
        for d in range(len(devices)):
            lst = []
            for q in range(K):
                t = src[q]
                if not torch.is_tensor(t):
                    lst.append(None)
                    continue
                if t.ndim == 2:
                    t = t.unsqueeze(0).expand(energies[d].shape[0], -1, -1)
                elif per_energy:
                    t = t[d:d + 1]
                lst.append(t)
            res.append(lst)
        return res

    sin = per_device(s_in) if need_lesser else None
    sout = per_device(s_out) if need_greater else None
    res = rgf_plan.run(geom, energies, [se_for(left_se, d) for d in range(len(devices))],
                       [se_for(right_se, d) for d in range(len(devices))], eta=eta, E_ref=0.0,
                       outputs=outputs, s_in=sin, s_out=sout)

    def gather(tag):
        if tag not in res.blocks[0]:
            return None
        if not per_energy:
            return res.blocks[0][tag]
        if tag == "g_trans":
            return torch.cat([r[tag] for r in res.blocks], 0)
        return [torch.cat([r[tag][q] for r in res.blocks], 0) for q in range(len(res.blocks[0][tag]))]

    vals = {t: gather(t) for t in TAGS}
    ans = tuple(vals.get(t) for t in TAGS)
    if out_dev.type != "cuda":
        ans = _to(ans, out_dev)
    if squeezed:
        ans = _squeeze_ans(ans)
    return ans


def _to(ans, dev):
    def mv(x):
        if x is None:
            return None
        if torch.is_tensor(x):
            return x.to(dev)
        return [t.to(dev) for t in x]
    return tuple(mv(x) for x in ans)


def _squeeze_ans(ans):
    """Drop the leading batch dim of every output (reference :480-491)."""
    def sq(x):
        if x is None:
            return None
        if torch.is_tensor(x):
            return x.squeeze(0)
        if isinstance(x, list):
            return [t.squeeze(0) if torch.is_tensor(t) else t for t in x]
        return x
    return tuple(sq(x) for x in ans)
