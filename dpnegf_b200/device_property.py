"""Device object with the GPU RGF sweep (mirror of negf/device_property.py).

Same constructor, attributes, ``greenfuncs`` tags and properties as the
reference ``DeviceProperty`` (:34-631).  ``cal_green_function`` runs one launch
of the batched RGF kernel that produces the requested Green's-function blocks
and, in the same sweep, T(E) and the per-orbital DOS diagonal; the ``tc``,
``dos`` and ``ldos`` properties return those fused results (identical, up to
rounding, to the reference's post-hoc products :374-470, evaluated with the
lead self-energies present at the time of ``cal_green_function``).
"""
import logging
import os
from typing import Union

import numpy as np
import torch
from scipy.constants import Boltzmann

from . import rgf_plan
from .negf_utils import simpson

log = logging.getLogger(__name__)
eV2J = 1.6021766208e-19
pi = np.pi

TAGS = ["g_trans", "gr_lc", "grd", "grl", "gru", "gr_left",
        "gnd", "gnl", "gnu", "gin_left", "gpd", "gpl", "gpu", "gip_left"]


def _build_s_in_batched(hd, seinL, seinR, idx0, idy0, idx1, idy1):
    """Per-block [B, n_q, n_q] zeros with the corner in-scattering injected (reference :21-31)."""
    B = seinL.shape[0]
    s_in = [torch.zeros((B,) + tuple(blk.shape), dtype=torch.complex128, device=seinL.device) for blk in hd]
    s_in[0][:, :idx0, :idy0] += seinL[:, :idx0, :idy0]
    s_in[-1][:, -idx1:, -idy1:] += seinR[:, -idx1:, -idy1:]
    return s_in


class DeviceProperty(object):
    def __init__(self, hamiltonian, structure, results_path, e_T=300,
                 efermi: dict = None, chemiPot: dict = None, E_ref: float = None,
                 rgf_device: Union[str, torch.device] = "cuda") -> None:
        self.greenfuncs = 0
        self.hamiltonian = hamiltonian
        self.structure = structure
        self.results_path = results_path
        self.cdtype = torch.complex128
        if isinstance(rgf_device, str):
            rgf_device = torch.device(rgf_device)
        self.rgf_device = rgf_device
        self.kBT = Boltzmann * e_T / eV2J
        self.e_T = e_T
        self.chemiPot = chemiPot
        self.E_ref = efermi if E_ref is None else E_ref
        self.kpoint = None
        self.newK_flag = None
        self.newV_flag = None
        self._geom = None
        self._fused = None

    def set_leadLR(self, lead_L, lead_R):
        self.lead_L = lead_L
        self.lead_R = lead_R

    # ----------------------------------------------------------------------
    def _compute_device(self):
        d = self.rgf_device if isinstance(self.rgf_device, torch.device) else torch.device(self.rgf_device)
        if d.type == "cuda":
            return d
        return torch.device("cuda", torch.cuda.current_device())

    def _refresh_hs(self, block_tridiagonal):
        self.hd, self.sd, self.hl, self.su, self.sl, self.hu = \
            self.hamiltonian.get_hs_device(self.kpoint, self.V, block_tridiagonal)
        dev = self._compute_device()
        mv = lambda xs: [torch.as_tensor(b).to(dev) for b in xs]
        self.hd, self.sd, self.hl = mv(self.hd), mv(self.sd), mv(self.hl)
        self.su, self.sl, self.hu = mv(self.su), mv(self.sl), mv(self.hu)
        self._geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(self.hd, self.hu, self.hl, self.sd, self.su,
                                                              self.sl)], device=dev)

    def _prepare(self, energy, kpoint, block_tridiagonal, Vbias):
        """Energy batch, potential and H/S refresh, self-energy checks of ``cal_green_function``
        (reference device_property.py:170-255)."""
        assert len(np.array(kpoint).reshape(-1)) == 3
        dev = self._compute_device()
        energy = torch.as_tensor(energy, dtype=torch.complex128, device=dev)
        if energy.ndim == 0:
            energy = energy.reshape(1)
        assert energy.ndim == 1, f"energy must be 0-d, scalar, or 1-D [B]; got shape {tuple(energy.shape)}"
        B = energy.shape[0]
        batched_mode = B > 1
        self.block_tridiagonal = block_tridiagonal
        if self.kpoint is None or abs(self.kpoint - torch.tensor(kpoint)).sum() > 1e-5:
            self.kpoint = torch.tensor(kpoint)
            self.newK_flag = True
        else:
            self.newK_flag = False
        self.oldV = self.V if hasattr(self, "V") else None
        if Vbias is None:
            if self.results_path and os.path.exists(os.path.join(self.results_path, "POTENTIAL.pth")):
                self.V = torch.load(os.path.join(self.results_path, "POTENTIAL.pth"))
            else:
                self.V = torch.tensor(0.)
        else:
            self.V = Vbias
        assert torch.is_tensor(self.V)
        self.V = self.V.to(dev)
        if self.oldV is not None:
            self.newV_flag = bool(torch.abs(self.V - self.oldV.to(dev)).sum() > 1e-5)
        else:
            self.newV_flag = True
        if (not (hasattr(self, "hd") and hasattr(self, "sd"))) or self.newK_flag or self.newV_flag \
                or self._geom is None:
            self._refresh_hs(block_tridiagonal)

        seL = torch.as_tensor(self.lead_L.se).to(dev)
        seR = torch.as_tensor(self.lead_R.se).to(dev)
        if batched_mode:
            assert seL.ndim == 3 and seR.ndim == 3, \
                f"In batched mode, the self-energy should have shape [B,n,n], but got {seL.shape} and {seR.shape}"
        else:
            assert seL.ndim == 2 and seR.ndim == 2, \
                f"In non-batched mode, the self-energy should have shape [n,n], but got {seL.shape} and {seR.shape}"
        s01, s02 = self.hd[0].shape
        se01, se02 = seL.shape[-2], seL.shape[-1]
        s11, s12 = self.hd[-1].shape
        se11, se12 = seR.shape[-2], seR.shape[-1]
        idx0, idy0 = min(s01, se01), min(s02, se02)
        idx1, idy1 = min(s11, se11), min(s12, se12)
        if block_tridiagonal:
            if se01 > s01 or se02 > s02:
                log.warning(f"The shape of left self-energy ({se01},{se02}) is larger than "
                            f"the first Hamiltonian block ({s01},{s02}).")
                raise ValueError("Left Lead Self Energy size is larger than the first Hamiltonian Block.")
            if se11 > s11 or se12 > s12:
                log.warning(f"The shape of right self-energy ({se11},{se12}) is larger than "
                            f"the last Hamiltonian block ({s11},{s12}).")
                raise ValueError("Right Lead Self Energy size is larger than the last Hamiltonian Block.")
        seLb = seL if seL.ndim == 3 else seL.unsqueeze(0)
        seRb = seR if seR.ndim == 3 else seR.unsqueeze(0)
        return energy, B, batched_mode, seLb, seRb, (idx0, idy0, idx1, idy1)

    def orbital_spectra(self, energy, kpoint, eta_device=0., block_tridiagonal=True, Vbias=None):
        """Per-orbital diag(G_qq) and diag(G_qN Gamma_R G_qN^H) over every block at ``energy``
        (scalar or [B]), reduced inside one sweep without materialising Green's-function blocks:
        ``([B, n_orb] complex, [B, n_orb] float64)``.  The self-energies are the leads' current
        ``se`` as in ``cal_green_function``; Gamma_R = i(Sigma_R - Sigma_R^H) in the last block's
        bottom-right corner."""
        energy, B, _, seLb, seRb, _ = self._prepare(energy, kpoint, block_tridiagonal, Vbias)
        res = rgf_plan.run(self._geom, [energy], [seLb], [seRb], eta=eta_device, E_ref=self.E_ref,
                           outputs=(), orb_g=True, orb_ar=True)
        n_orb = int(self._geom.n_orb[0])
        return res.orb_g.view(B, n_orb), res.orb_ar.view(B, n_orb)

    def cal_green_function(self, energy, kpoint, eta_device=0., block_tridiagonal=True, Vbias=None,
                           HS_inmem: bool = True, need_lesser: bool = False, need_greater: bool = False,
                           need_gr_lc: bool = False):
        """Green's functions (and fused T, DOS, LDOS) at ``energy`` (scalar or [B]) for ``kpoint``."""
        # the reference passes s_out=None to recursive_gf here (device_property.py:283), whose greater
        # branch then fails its list check (recursive_green_cal.py:67 / :268): same error
        assert not need_greater, \
            "Greater Green's function calculation requires s_out to be a list of coupling matrices"
        energy, B, batched_mode, seLb, seRb, corners = self._prepare(energy, kpoint, block_tridiagonal, Vbias)
        idx0, idy0, idx1, idy1 = corners

        s_in = None
        if need_lesser:
            Eabs = energy + self.E_ref
            fL = self.lead_L.fermi_dirac(Eabs).reshape(B, 1, 1)
            fR = self.lead_R.fermi_dirac(Eabs).reshape(B, 1, 1)
            seinL = 1j * (seLb - seLb.mH) * fL
            seinR = 1j * (seRb - seRb.mH) * fR
            s_in = [_build_s_in_batched(self.hd, seinL, seinR, idx0, idy0, idx1, idy1)]

        outputs = ["g_trans", "grd", "grl", "gru"]
        if need_gr_lc:
            outputs.append("gr_lc")
        if need_lesser:
            outputs.append("gr_left")  # keep_gr_left = need_lesser or need_greater (:278)
        res = rgf_plan.run(self._geom, [energy], [seLb], [seRb], eta=eta_device, E_ref=self.E_ref,
                           outputs=outputs, s_in=s_in, trans=True, orb_dos=True, dos=True)
        blocks = res.blocks[0]
        green = {t: blocks.get(t) for t in TAGS}
        if not batched_mode:
            sq = lambda x: x if x is None else (x.squeeze(0) if torch.is_tensor(x) else [t.squeeze(0) for t in x])
            green = {t: sq(v) for t, v in green.items()}
        out_dev = self.rgf_device if isinstance(self.rgf_device, torch.device) else torch.device(self.rgf_device)
        if out_dev.type != "cuda":
            mvv = lambda x: x if x is None else (x.to(out_dev) if torch.is_tensor(x) else [t.to(out_dev) for t in x])
            green = {t: mvv(v) for t, v in green.items()}
        self.greenfuncs = green
        n_orb = int(self._geom.n_orb[0])
        T, D, orb = res.trans, res.dos, res.orb_dos.view(B, n_orb)
        if not batched_mode:
            T, D, orb = T[0], D[0], orb[0]
        if out_dev.type != "cuda":
            T, D, orb = T.to(out_dev), D.to(out_dev), orb.to(out_dev)
        self._fused = {"tc": T, "dos": D, "orb": orb}
        if not HS_inmem:
            del self.hd, self.sd, self.hl, self.su, self.sl, self.hu
            self._geom = None

    def release_greenfuncs(self):
        self.greenfuncs = 0
        self._fused = None
        if isinstance(self.rgf_device, torch.device) and self.rgf_device.type == "cuda":
            torch.cuda.empty_cache()

    # ------------------------------------------------------------ observables
    def _cal_tc_(self):
        """T(E) = Re Tr[Gamma_L G_1N Gamma_R G_1N^H] (reduced inside the sweep)."""
        return self._fused["tc"]

    def _cal_dos_(self):
        """DOS with spin multiplicity (reduced inside the sweep)."""
        return self._fused["dos"]

    def _cal_ldos_(self):
        """Per-atom LDOS with spin multiplicity (reference :441-470)."""
        orb = self._fused["orb"]
        acc = np.cumsum([0] + list(self.norbs_per_atom))
        return 2 * torch.stack([orb[..., acc[i]:acc[i + 1]].sum(-1) for i in range(len(acc) - 1)], dim=-1)

    def _cal_current_nscf_(self, energy_grid, tc):
        """Non-self-consistent I-V sweep by Simpson integration (reference :333-371), FP64 on tc's device."""
        if abs(self.lead_L.efermi - self.lead_R.efermi) < 5e-4:
            log.warning(msg="The Fermi energy of the left and right leads should be equal in nscf current calculation.")
        efermi = self.lead_L.efermi
        tc = torch.as_tensor(tc)
        energy_grid = torch.as_tensor(energy_grid, dtype=torch.float64, device=tc.device)
        f = lambda x, mu: 1 / (1 + torch.exp((x - mu) / self.kBT))
        emin, emax = energy_grid.min(), energy_grid.max()
        vmin, vmax = emin + 4 * self.kBT, emax - 4 * self.kBT
        vm = 0.5 * (vmin + vmax)
        vmid = vm - vmin
        # the default dtype (float32), as the reference's torch.linspace (device_property.py:362)
        vv = torch.linspace(start=0., end=float(vmid), steps=int(vmid / 0.1) + 1) * 2
        cc = []
        for dv in vv * 0.5:
            y = (f(energy_grid + efermi, efermi - vm + dv) - f(energy_grid + efermi, efermi - vm - dv)) * tc
            cc.append(simpson(y, energy_grid))
        return vv, cc

    def _cal_local_current_(self):
        """Bond currents between atoms from G^< (non-block-tridiagonal, reference :472-503)."""
        na = len(self.norbs_per_atom)
        hd = torch.as_tensor(self.hamiltonian.get_hs_device(kpoint=self.kpoint, V=self.V,
                                                            block_tridiagonal=self.block_tridiagonal)[0][0])
        gnd = self.gnd[0]
        hd = hd.to(gnd.device)
        # K[I,J] = Re Tr[H_IJ (i G^<_JI)] by orbital-block sums of H * (i G^<)^T
        M = (hd * (1j * gnd).transpose(-1, -2)).real
        acc = np.cumsum([0] + list(self.norbs_per_atom))
        rows = torch.stack([M[acc[i]:acc[i + 1]].sum(0) for i in range(na)])
        K = torch.stack([rows[:, acc[j]:acc[j + 1]].sum(1) for j in range(na)], dim=1)
        lc = K - K.T
        lc.fill_diagonal_(0.0)
        return lc.contiguous()

    def _cal_density_(self, dm_options):
        from .density import Ozaki
        dm = Ozaki(**dm_options)
        return dm.integrate(deviceprop=self, kpoint=self.kpoint)

    @property
    def dos(self):
        return self._cal_dos_()

    @property
    def ldos(self):
        return self._cal_ldos_()

    @property
    def tc(self):
        return self._cal_tc_()

    @property
    def lcurrent(self):
        return self._cal_local_current_()

    @property
    def g_trans(self):
        return self.greenfuncs["g_trans"]

    @property
    def gr_lc(self):
        return self.greenfuncs["gr_lc"]

    @property
    def grd(self):
        return self.greenfuncs["grd"]

    @property
    def grl(self):
        return self.greenfuncs["grl"]

    @property
    def gru(self):
        return self.greenfuncs["gru"]

    @property
    def gr_left(self):
        return self.greenfuncs["gr_left"]

    @property
    def gnd(self):
        return self.greenfuncs["gnd"]

    @property
    def gnl(self):
        return self.greenfuncs["gnl"]

    @property
    def gnu(self):
        return self.greenfuncs["gnu"]

    @property
    def gin_left(self):
        return self.greenfuncs["gin_left"]

    @property
    def gpd(self):
        return self.greenfuncs["gpd"]

    @property
    def gpl(self):
        return self.greenfuncs["gpl"]

    @property
    def gpu(self):
        return self.greenfuncs["gpu"]

    @property
    def gip_left(self):
        return self.greenfuncs["gip_left"]

    @property
    def norbs_per_atom(self):
        return self.hamiltonian.device_norbs

    @property
    def positions(self):
        return self.structure.positions

    def get_index(self, iatom):
        start = sum(self.norbs_per_atom[:iatom])
        return [start, start + self.norbs_per_atom[iatom]]
