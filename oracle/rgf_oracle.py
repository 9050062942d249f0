"""numpy restatement of the reference NEGF hot path (complex128).

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).  Every function cites
the reference file:line it follows; citations are relative to the dpnegf
source tree.

Conventions (same as the reference):
  * ``mat_d = H + Sigma - z S`` with ``z = E + E_ref + 1j*eta``
    (negf/recursive_green_cal.py:75-78, :175-182, :378, :411-428);
  * ``gr_left[q] = (-mat_d[q] - mat_l[q-1] gr_left[q-1] mat_u[q-1])^-1``
    (:88-94 / :198-207);
  * backward sweep (:98-114 / :209-238), lesser (:121-140 / :241-264),
    greater (:143-161 / :267-289).
"""
import numpy as np

TAGS = ("g_trans", "gr_lc", "grd", "grl", "gru", "gr_left",
        "gnd", "gnl", "gnu", "gin_left", "gpd", "gpl", "gpu", "gip_left")


def _bt(x, B):
    """Broadcast a 2-D k-block to [B, m, n] (recursive_green_cal.py:404-407)."""
    x = np.asarray(x, dtype=np.complex128)
    if x.ndim == 2:
        return np.broadcast_to(x, (B,) + x.shape)
    return x


def _mH(x):
    return np.conj(np.swapaxes(x, -1, -2))


def rgf(energy, hl, hd, hu, sd, su, sl, left_se, right_se, seP=None, E_ref=0.0,
        s_in=None, s_out=None, eta=1e-5, need_lesser=False, need_greater=False,
        need_gr_lc=False, keep_gr_left=True):
    """Batched RGF, returns a dict keyed by the 14 reference tags.

    Follows ``recursive_gf`` (negf/recursive_green_cal.py:324-477) and
    ``recursive_gf_cal`` (:4-296).  ``energy`` is a scalar or ``[B]`` array;
    the energy-independent blocks may be 2-D; ``left_se``/``right_se`` are
    ``[B, nL, nL]`` (or 2-D for a scalar energy) and are added into the
    top-left / bottom-right corner of the first / last diagonal block
    (:411-428).  Outputs always carry the leading batch dim.
    """
    z = np.atleast_1d(np.asarray(energy, dtype=np.complex128)) + E_ref
    B = z.shape[0]
    K = len(hd)
    zb = (z + 1j * eta).reshape(B, 1, 1)

    D = [(_bt(hd[q], B) - zb * _bt(sd[q], B)).copy() for q in range(K)]
    Lm = [_bt(hl[q], B) - zb * _bt(sl[q], B) for q in range(K - 1)]
    Um = [_bt(hu[q], B) - zb * _bt(su[q], B) for q in range(K - 1)]
    if seP is not None:
        for q in range(K):
            D[q] = D[q] + _bt(seP[q], B)
    if left_se is not None:
        se = _bt(left_se, B)
        a, b = min(D[0].shape[-2], se.shape[-2]), min(D[0].shape[-1], se.shape[-1])
        D[0][:, :a, :b] += se[:, :a, :b]
    if right_se is not None:
        se = _bt(right_se, B)
        a, b = min(D[-1].shape[-2], se.shape[-2]), min(D[-1].shape[-1], se.shape[-1])
        D[-1][:, D[-1].shape[-2] - a:, D[-1].shape[-1] - b:] += se[:, se.shape[-2] - a:, se.shape[-1] - b:]

    # forward sweep: left-connected blocks (:88-94)
    g = [None] * K
    g[0] = np.linalg.inv(-D[0])
    for q in range(K - 1):
        g[q + 1] = np.linalg.inv(-D[q + 1] - Lm[q] @ g[q] @ Um[q])

    # backward sweep (:98-114)
    grd = [None] * K
    grl = [None] * (K - 1)
    gru = [None] * (K - 1)
    grd[-1] = g[-1].copy()
    g_trans = g[-1].copy()
    gr_lc = [g_trans] if need_gr_lc else None
    for q in range(K - 2, -1, -1):
        gU = g[q] @ Um[q]
        grl[q] = grd[q + 1] @ Lm[q] @ g[q]
        gru[q] = gU @ grd[q + 1]
        grd[q] = g[q] + gU @ grl[q]
        g_trans = gU @ g_trans
        if need_gr_lc:
            gr_lc.append(g_trans)
    if need_gr_lc:
        gr_lc.reverse()

    out = dict.fromkeys(TAGS)
    out.update(g_trans=g_trans, gr_lc=gr_lc, grd=grd, grl=grl, gru=gru,
               gr_left=g if keep_gr_left else None)

    if need_lesser:
        sin = [_bt(s_in[q], B) for q in range(K)]
        gin = [None] * K
        gin[0] = g[0] @ sin[0] @ _mH(g[0])
        for q in range(K - 1):
            sla2 = Lm[q] @ gin[q] @ Um[q]
            gin[q + 1] = g[q + 1] @ (sin[q + 1] + sla2) @ _mH(g[q + 1])
        gnd = [None] * K
        gnl = [None] * (K - 1)
        gnu = [None] * (K - 1)
        gnd[-1] = gin[-1].copy()
        for q in range(K - 2, -1, -1):
            gLmH = Lm[q] @ _mH(g[q])
            gnl[q] = grd[q + 1] @ Lm[q] @ gin[q] + gnd[q + 1] @ gLmH
            gnd[q] = (gin[q] + g[q] @ Um[q] @ gnd[q + 1] @ gLmH
                      + gin[q] @ Um[q] @ _mH(gru[q]) + gru[q] @ Lm[q] @ gin[q])
            gnu[q] = _mH(gnl[q])
        out.update(gnd=gnd, gnl=gnl, gnu=gnu, gin_left=gin)

    if need_greater:
        sout = [_bt(s_out[q], B) for q in range(K)]
        gip = [None] * K
        gip[0] = g[0] @ sout[0] @ np.conj(g[0])
        for q in range(K - 1):
            sla2 = Lm[q] @ gip[q] @ np.conj(Um[q])
            gip[q + 1] = g[q + 1] @ (sout[q + 1] + sla2) @ np.conj(g[q + 1])
        gpd = [None] * K
        gpl = [None] * (K - 1)
        gpu = [None] * (K - 1)
        gpd[-1] = gip[-1].copy()
        for q in range(K - 2, -1, -1):
            lcgc = np.conj(Lm[q]) @ np.conj(g[q])
            gpl[q] = grd[q + 1] @ Lm[q] @ gip[q] + gpd[q + 1] @ lcgc
            gpd[q] = (gip[q] + g[q] @ Um[q] @ gpd[q + 1] @ lcgc
                      + gip[q] @ np.conj(Um[q]) @ np.conj(grl[q]) + gru[q] @ Lm[q] @ gip[q])
            gpu[q] = _mH(gpl[q])
        out.update(gpd=gpd, gpl=gpl, gpu=gpu, gip_left=gip)
    return out


def gamma_from_se(se):
    """Gamma = i (Sigma - Sigma^H) (negf/lead_property.py:437-460)."""
    return 1j * (se - _mH(se))


def transmission(g_trans, gammaL_full, gammaR_full):
    """T(E) = Re Tr[Gamma_L G_1N Gamma_R G_1N^H] with corner-embedded Gammas.

    Follows DeviceProperty._cal_tc_ (negf/device_property.py:374-406).
    ``g_trans`` is [B, n1, nN]; Gammas are [B, nL, nL] / [B, nR, nR].
    """
    B, tx, ty = g_trans.shape
    x0 = min(gammaL_full.shape[-2], tx)
    x1 = min(gammaR_full.shape[-2], ty)
    gL = np.zeros((B, tx, tx), np.complex128)
    gR = np.zeros((B, ty, ty), np.complex128)
    gL[:, :x0, :x0] += gammaL_full[:, :x0, :x0]
    gR[:, ty - x1:, ty - x1:] += gammaR_full[:, gammaR_full.shape[-2] - x1:, gammaR_full.shape[-1] - x1:]
    prod = gL @ g_trans @ gR @ _mH(g_trans)
    return np.real(np.einsum("bii->b", prod))


def _dos_blocks(grd, grl, gru, sd, su, sl):
    """Per-block ``G S`` diagonal (negf/device_property.py:428-437 / :451-463)."""
    K = len(grd)
    B = grd[0].shape[0]
    res = []
    for jj in range(K):
        t = grd[jj] @ _bt(sd[jj], B)
        if K > 1:
            if jj == 0:
                t = t + gru[jj] @ _bt(sl[jj], B)
            elif jj == K - 1:
                t = t + grl[jj - 1] @ _bt(su[jj - 1], B)
            else:
                t = t + grl[jj - 1] @ _bt(su[jj - 1], B) + gru[jj] @ _bt(sl[jj], B)
        res.append(np.imag(np.einsum("bii->bi", t)))
    return res


def dos(grd, grl, gru, sd, su, sl):
    """DOS = -(2/pi) sum_q Im Tr[...]  (negf/device_property.py:408-439)."""
    return -2.0 * sum(d.sum(-1) for d in _dos_blocks(grd, grl, gru, sd, su, sl)) / np.pi


def ldos(grd, grl, gru, sd, su, sl, norbs_per_atom):
    """Per-atom LDOS with spin factor 2 (negf/device_property.py:441-470)."""
    per_orb = -np.concatenate(_dos_blocks(grd, grl, gru, sd, su, sl), axis=-1) / np.pi
    acc = np.cumsum([0] + list(norbs_per_atom))
    return 2.0 * np.stack([per_orb[..., acc[i]:acc[i + 1]].sum(-1) for i in range(len(acc) - 1)], -1)


def fermi_dirac(x, mu, kBT):
    """1/(1+exp((x-mu)/kBT)) (negf/lead_property.py:455-456)."""
    return 1.0 / (1.0 + np.exp((np.asarray(x) - mu) / kBT))


def s_in_from_se(seL, seR, fL, fR, block_dims):
    """Sigma^in = i(Sigma - Sigma^H) f, corner-embedded per block.

    Follows negf/device_property.py:259-272 and ``_build_s_in_batched`` (:21-31).
    """
    B = seL.shape[0]
    s_in = [np.zeros((B, n, n), np.complex128) for n in block_dims]
    sinL = 1j * (seL - _mH(seL)) * np.reshape(fL, (B, 1, 1))
    sinR = 1j * (seR - _mH(seR)) * np.reshape(fR, (B, 1, 1))
    a = min(block_dims[0], seL.shape[-1])
    b = min(block_dims[-1], seR.shape[-1])
    s_in[0][:, :a, :a] += sinL[:, :a, :a]
    s_in[-1][:, block_dims[-1] - b:, block_dims[-1] - b:] += sinR[:, seR.shape[-1] - b:, seR.shape[-1] - b:]
    return s_in
