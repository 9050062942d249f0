"""Ozaki pole-sum density on the B200 (mirror of negf/density.py:107-230).

``Ozaki(R, M_cut, n_gauss).integrate`` evaluates

  DM_eq  = Re[ iR G(iR - mu_D) - sum_p Im(-4i kT G(z_p) r_p) ],
           z_p = i pole_p kT + mu_L - mu_D                    (density.py:164-181)
  DM_neq = sum_i w_i Re[G Gamma_R G^H] (f_R - f_L)            (density.py:183-195)

with G the first diagonal block ``grd[0]`` as in the reference.  The
reference reads ``deviceprop.mu`` and ``deviceprop.lead_L.mu``, which its
classes never define; here they are the arguments ``mu`` / ``mu_lead`` and
default to the device ``E_ref`` offset 0 (energies are relative to E_ref) and
the left lead's chemical potential relative to E_ref.  All poles go through
one batched Lopez-Sancho launch per lead and one batched RGF launch instead of
M_cut + 1 scalar round trips.

``integrate_orbitals`` is the block-tridiagonal generalisation: the
per-orbital density over every block from the in-sweep reductions diag(G_qq)
and diag(G_qN Gamma_R G_qN^H), without materialising Green's-function blocks.
``uneven_batch`` does the same, plus T(E) in the bias window, for many devices
of uneven block size and length: one Lopez-Sancho launch for every lead at
every energy and one persistent RGF launch for every (device, energy) item.
"""
import logging

import numpy as np
import torch

from .negf_utils import gauss_xw
from .ozaki_res_cal import ozaki_residues

log = logging.getLogger(__name__)


class Density(object):
    def __init__(self) -> None:
        pass

    def integrate(self, deviceprop):
        pass


class Ozaki(Density):
    def __init__(self, R, M_cut, n_gauss):
        super().__init__()
        self.poles, self.residues = ozaki_residues(M_cut)
        self.R = R
        self.n_gauss = n_gauss

    def _mus(self, deviceprop, mu, mu_lead):
        mu_D = 0.0 if mu is None else float(mu)
        if mu_lead is None:
            mu_lead = float(deviceprop.lead_L.chemiPot_lead) - float(deviceprop.E_ref)
        return mu_D, float(mu_lead)

    def _green_first_block(self, deviceprop, kpoint, energies, eta_lead, eta_device, Vbias, block_tridiagonal):
        """grd[0] at every energy of ``energies`` ([B] complex) in one lead launch + one RGF launch; [B, n0, n0]."""
        E = torch.as_tensor(np.asarray(energies), dtype=torch.complex128).reshape(-1)
        if E.shape[0] == 1:
            E = E[0]  # scalar call: self-energies and blocks stay 2-D as in the reference
        deviceprop.lead_L.self_energy(kpoint=kpoint, energy=E, eta_lead=eta_lead)
        deviceprop.lead_R.self_energy(kpoint=kpoint, energy=E, eta_lead=eta_lead)
        deviceprop.cal_green_function(energy=E, kpoint=kpoint, block_tridiagonal=block_tridiagonal,
                                      eta_device=eta_device, Vbias=Vbias)
        g = deviceprop.grd[0]
        return g.unsqueeze(0) if g.ndim == 2 else g

    def integrate(self, deviceprop, kpoint, eta_lead=1e-5, eta_device=0., Vbias=None, block_tridiagonal=False,
                  mu=None, mu_lead=None):
        kBT = deviceprop.kBT
        mu_D, mu_L = self._mus(deviceprop, mu, mu_lead)
        zp = 1j * self.poles.numpy() * kBT + mu_L - mu_D
        # far pole iR (the reference evaluates it with the default eta_lead and eta_device = 0)
        gR = self._green_first_block(deviceprop, kpoint, np.array([1j * self.R - mu_D]),
                                     1e-5, 0.0, Vbias, block_tridiagonal)[0]
        DM_eq = 1.0j * self.R * gR
        G = self._green_first_block(deviceprop, kpoint, zp, eta_lead, eta_device, Vbias, block_tridiagonal)
        r = self.residues.to(G.device).reshape(-1, 1, 1)
        DM_eq = DM_eq - ((-4j * kBT) * G * r).imag.sum(0)
        DM_eq = DM_eq.real

        vL, vR = float(deviceprop.lead_L.voltage), float(deviceprop.lead_R.voltage)
        if abs(vL - vR) > 1e-14:
            xl, xu = min(vL, vR) - 8 * kBT, max(vL, vR) + 8 * kBT
            xs, wlg = gauss_xw(xl=torch.scalar_tensor(xl, dtype=torch.float64),
                               xu=torch.scalar_tensor(xu, dtype=torch.float64), n=self.n_gauss)
            Gr = self._green_first_block(deviceprop, kpoint, xs.to(torch.complex128), eta_lead, eta_device,
                                         None, block_tridiagonal)
            gam = deviceprop.lead_R.gamma.to(Gr.device)
            n0 = Gr.shape[-1]
            cr = min(n0, gam.shape[-1])
            GR = torch.zeros(gam.shape[0], n0, n0, dtype=torch.complex128, device=Gr.device)
            GR[:, n0 - cr:, n0 - cr:] = gam[:, gam.shape[-2] - cr:, gam.shape[-1] - cr:]
            A = (Gr @ GR @ Gr.mH).real
            e = xs.to(Gr.device)
            df = (deviceprop.lead_R.fermi_dirac(e + mu_D) - deviceprop.lead_L.fermi_dirac(e + mu_D)).real
            DM_neq = (wlg.to(Gr.device).reshape(-1, 1, 1) * A * df.reshape(-1, 1, 1)).sum(0)
        else:
            DM_neq = 0.
        return DM_eq, DM_neq

    def get_density_onsite(self, deviceprop, DM):
        """Per-atom density with positions, [n_atoms, 4] (reference :201-230)."""
        if len(DM.shape) == 2:
            DM = DM.diagonal()
        elif not len(DM.shape) == 1:
            log.error("The DM must be the of shape [norbs] or [norbs, norbs]")
        acc = np.cumsum([0] + list(deviceprop.norbs_per_atom))
        onsite = torch.stack([DM[acc[i]:acc[i + 1]].sum() for i in range(len(acc) - 1)])
        pos = torch.as_tensor(np.asarray(deviceprop.structure.positions), dtype=onsite.dtype, device=onsite.device)
        return torch.cat([pos, onsite.unsqueeze(-1)], dim=-1)

    def integrate_orbitals(self, geometry, se_left, se_right, kBT, mu_L, mu_D=0.0, vL=0.0, vR=0.0,
                           fermi_L=None, fermi_R=None, eta_device=0.0, E_ref=0.0, se_real=None):
        """Per-orbital equilibrium and non-equilibrium density of a BTD device.

        ``se_left(E)`` / ``se_right(E)`` return [B, n, n] lead self-energies for
        a [B] complex energy array.  Uses one RGF launch for the iR point and
        all poles (diag(G_qq)), and one for the Gauss-Legendre points
        (diag(G_qN Gamma_R G_qN^H)).  Returns ``(n_eq, n_neq)`` of length n_orb.
        """
        from . import rgf_plan
        zs = np.concatenate([[1j * self.R - mu_D], 1j * self.poles.numpy() * kBT + mu_L - mu_D])
        E = torch.as_tensor(zs, dtype=torch.complex128)
        res = rgf_plan.run(geometry, [E.to(geometry.device)], [se_left(zs)], [se_right(zs)], eta=eta_device,
                           E_ref=E_ref, outputs=(), orb_g=True)
        n_orb = geometry.n_orb[0]
        g = res.orb_g.view(len(zs), n_orb)
        r = self.residues.to(g.device).reshape(-1, 1)
        n_eq = (1j * self.R * g[0] - ((-4j * kBT) * g[1:] * r).imag.sum(0)).real
        if abs(vL - vR) > 1e-14:
            xl, xu = min(vL, vR) - 8 * kBT, max(vL, vR) + 8 * kBT
            xs, wlg = gauss_xw(xl=torch.scalar_tensor(xl, dtype=torch.float64),
                               xu=torch.scalar_tensor(xu, dtype=torch.float64), n=self.n_gauss)
            xr = xs.numpy().astype(np.complex128)
            res2 = rgf_plan.run(geometry, [torch.as_tensor(xr).to(geometry.device)], [se_left(xr)], [se_right(xr)],
                                eta=eta_device, E_ref=E_ref, outputs=(), orb_ar=True)
            a = res2.orb_ar.view(len(xr), n_orb)
            e = xs.to(a.device)
            df = (fermi_R(e + mu_D) - fermi_L(e + mu_D)).real.reshape(-1, 1)
            n_neq = (wlg.to(a.device).reshape(-1, 1) * a * df).sum(0)
        else:
            n_neq = torch.zeros(n_orb, dtype=torch.float64, device=g.device)
        return n_eq, n_neq

    def uneven_batch(self, devices, leads, kBT, mu_L, mu_D=0.0, vL=0.0, vR=0.0, fermi_L=None, fermi_R=None,
                     eta_lead=1e-5, eta_device=0.0, E_ref=0.0, precision="fp64", refine=False, refine_steps=3,
                     device="cuda"):
        """Per-orbital density and T(E) of many BTD devices in one lead launch + one RGF launch.

        ``devices`` are ``rgf_plan.DeviceBlocks``; ``leads[d] = (left, right)`` are
        ``surface_green.LeadBlocks`` whose ``hDL`` couples the lead to the first /
        last block.  Energies (relative to ``E_ref``): the far pole ``iR - mu_D``,
        the Ozaki poles ``i pole kT + mu_L - mu_D`` and, when ``vL != vR``, the
        ``n_gauss`` Gauss-Legendre points of ``[min V - 8kT, max V + 8kT]``; every
        energy uses ``eta_lead`` for the leads and ``eta_device`` for the device.
        Items are ordered largest first by the planner, so devices of very
        different size balance over the persistent CTAs.  Returns one dict per
        device: ``n_eq`` and ``n_neq`` [n_orb] (formulas of ``integrate_orbitals``),
        and ``energy`` / ``trans`` on the real-axis points (empty without bias).
        """
        from . import rgf_plan
        from .surface_green import LeadArena, self_energies
        nd = len(devices)
        if len(leads) != nd:
            raise ValueError("one (left, right) lead pair per device")
        P = len(self.poles)
        zs = np.concatenate([[1j * self.R - mu_D], 1j * self.poles.numpy() * kBT + mu_L - mu_D]).astype(np.complex128)
        bias = abs(vL - vR) > 1e-14
        if bias:
            xl, xu = min(vL, vR) - 8 * kBT, max(vL, vR) + 8 * kBT
            xs, wlg = gauss_xw(xl=torch.scalar_tensor(xl, dtype=torch.float64),
                               xu=torch.scalar_tensor(xu, dtype=torch.float64), n=self.n_gauss)
            zs = np.concatenate([zs, xs.numpy().astype(np.complex128)])
        nE = len(zs)
        arena = LeadArena([ld for pair in leads for ld in pair], device=device)
        idx = np.repeat(np.arange(2 * nd), nE)
        ls = self_energies(arena, idx, np.tile(zs, 2 * nd), eta_lead, E_ref=E_ref)
        se = [torch.stack(ls.sigma[i * nE:(i + 1) * nE]) for i in range(2 * nd)]
        geom = rgf_plan.Geometry(list(devices), device=device)
        E = torch.as_tensor(zs).to(geom.device)
        res = rgf_plan.run(geom, [E] * nd, se[0::2], se[1::2], eta=eta_device, E_ref=E_ref, outputs=(),
                           trans=True, orb_g=True, orb_ar=bias, precision=precision, refine=refine and bias,
                           refine_steps=refine_steps)
        r = self.residues.to(geom.device).reshape(-1, 1)
        out, orb0 = [], 0
        for d in range(nd):
            n_orb = int(geom.devs[d]["n_orb"])
            g = res.orb_g[orb0:orb0 + nE * n_orb].view(nE, n_orb)
            n_eq = (1j * self.R * g[0] - ((-4j * kBT) * g[1:1 + P] * r).imag.sum(0)).real
            rec = {"n_eq": n_eq, "energy": torch.zeros(0, dtype=torch.float64),
                   "trans": torch.zeros(0, dtype=torch.float64, device=geom.device)}
            if bias:
                a = res.orb_ar[orb0:orb0 + nE * n_orb].view(nE, n_orb)[1 + P:]
                e = xs.to(a.device)
                df = (fermi_R(e + mu_D) - fermi_L(e + mu_D)).real.reshape(-1, 1)
                rec["n_neq"] = (wlg.to(a.device).reshape(-1, 1) * a * df).sum(0)
                rec["energy"] = xs
                rec["trans"] = res.trans[d * nE + 1 + P:(d + 1) * nE]
            else:
                rec["n_neq"] = torch.zeros(n_orb, dtype=torch.float64, device=g.device)
            out.append(rec)
            orb0 += nE * n_orb
        return out
