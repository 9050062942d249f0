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
from .products import gamma_sum
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
            # as the reference (density.py:186): limits from torch.scalar_tensor (the default dtype,
            # float32), so the nodes, weights and Fermi factors are float32
            xs, wlg = gauss_xw(xl=torch.scalar_tensor(xl), xu=torch.scalar_tensor(xu), n=self.n_gauss)
            Gr = self._green_first_block(deviceprop, kpoint, xs.to(torch.complex128), eta_lead, eta_device,
                                         None, block_tridiagonal)
            gam = deviceprop.lead_R.gamma.to(Gr.device)
            if gam.ndim == 2:
                gam = gam.unsqueeze(0)
            n0 = Gr.shape[-1]
            cr = min(n0, gam.shape[-1])
            # f_R - f_L per node on 0-d host tensors, the reference's arithmetic (density.py:192)
            df = torch.stack([torch.as_tensor(deviceprop.lead_R.fermi_dirac(x + mu_D)
                                              - deviceprop.lead_L.fermi_dirac(x + mu_D)).real.cpu() for x in xs])
            # sum_i wlg_i df_i Re(G_i Gamma_R G_i^H) with Gamma_R in the last cr x cr corner: one CUDA
            # call (per-node products, then one GEMM over every node)
            w = wlg.to(torch.float64) * df.to(torch.float64)
            DM_neq = gamma_sum(Gr, gam[:, gam.shape[-2] - cr:, gam.shape[-1] - cr:], n0 - cr, w)
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


class Fiori(Density):
    """Free charge per atom on a real energy grid (mirror of negf/density.py:234-395).

    The reference walks ``integrate_range`` one energy at a time: both lead
    self-energies, a full ``cal_green_function``, then for every diagonal block
    A_R = G_qN Gamma_R G_qN^H, A_L = i(G_qq - G_qq^H) - A_R,
    G^n = A_L f_L(E + E_ref) + A_R f_R(E + E_ref) and G^p = A_L + A_R - G^n, and
    per atom adds  w_E * (-1/pi) Tr_atom G^n  when E >= -potential_at_atom
    (electrons) or  w_E * (1/pi) Tr_atom G^p  otherwise (holes)
    (density.py:268-360).  Only diagonals of those blocks enter the traces, so
    here every energy of the grid goes through one Lopez-Sancho launch per lead
    and one RGF launch that reduces diag(G_qq) and diag(G_qN Gamma_R G_qN^H)
    inside the sweep (``DeviceProperty.orbital_spectra``); the per-atom sums
    and the electron/hole selection are tensor ops on the GPU.

    The weights and nodes follow the reference's dtypes: ``dE * torch.ones``
    and ``gauss_xw`` of ``torch.scalar_tensor`` limits are float32, as there.
    Two reference branches cannot run as written, and run here as intended:
    with ``block_tridiagonal=True`` the reference reads ``gr_lc``, which its
    ``cal_green_function`` call never requests (density.py:293-294, 304), and
    without Dirichlet leads it passes ``save=False``, which
    ``LeadProperty.self_energy`` does not accept (density.py:278-279); here the
    last block column enters through the sweep's reduction and the lead
    self-energies are recomputed, never loaded, without Dirichlet leads.
    """

    def __init__(self, n_gauss=None, integrate_way: str = "direct", e_grid=None):
        super().__init__()
        self.n_gauss = n_gauss
        self.e_grid = e_grid
        self.integrate_way = integrate_way
        self.xs = None
        self.wlg = None
        self.e_grid_Fiori = None
        if integrate_way == "gauss":
            assert self.n_gauss is not None, "n_gauss must be set in the Fiori class with gauss integration"
            self.xs, self.wlg = gauss_xw(xl=torch.scalar_tensor(e_grid[0]), xu=torch.scalar_tensor(e_grid[-1]),
                                         n=self.n_gauss)
            self.e_grid_Fiori = e_grid
            integrate_range, pre_factor = self.xs, self.wlg
        elif integrate_way == "direct":
            dE = e_grid[1] - e_grid[0]
            integrate_range = e_grid
            pre_factor = dE * torch.ones(len(e_grid))
        else:
            raise ValueError("integrate_way only supports 'gauss' and 'direct' in this version")
        self.integrate_range = integrate_range
        self.pre_factor = pre_factor

    def density_integrate_Fiori(self, e_grid, kpoint, Vbias, block_tridiagonal, subblocks, integrate_way, deviceprop,
                                device_atom_norbs, potential_at_atom, with_Dirichlet_leads, free_charge, E_ref,
                                eta_lead=1e-5, eta_device=1e-5, self_energy_save_path=None):
        """Add this k-point's free charge per atom into ``free_charge[str(kpoint)]`` (in place).

        ``e_grid`` and ``integrate_way`` are accepted for the reference's signature; the grid
        and weights are the ones built in ``__init__``, as in the reference.  ``subblocks`` is
        implied by the device blocks: orbitals are numbered through the blocks in order."""
        E = torch.as_tensor(self.integrate_range)
        B = E.shape[0]
        e_arg = E if B > 1 else E[0]  # one energy: the scalar contract ([n, n] self-energies)
        for lead in (deviceprop.lead_L, deviceprop.lead_R):
            if with_Dirichlet_leads:
                lead.self_energy(kpoint=kpoint, energy=e_arg, eta_lead=eta_lead, save_path=self_energy_save_path)
            else:
                lead.se = lead.self_energy_cal(kpoint, e_arg, eta_lead=eta_lead)
        g, a_R = deviceprop.orbital_spectra(energy=e_arg, kpoint=kpoint, eta_device=eta_device,
                                            block_tridiagonal=block_tridiagonal, Vbias=Vbias)
        dev = g.device
        a_L = -2.0 * g.imag - a_R  # diag of i(G - G^H) - A_R
        e = E.to(dev)
        fL = torch.as_tensor(deviceprop.lead_L.fermi_dirac(e + E_ref)).to(dev).reshape(B, 1)
        fR = torch.as_tensor(deviceprop.lead_R.fermi_dirac(e + E_ref)).to(dev).reshape(B, 1)
        gn = a_L * fL + a_R * fR
        gp = a_L + a_R - gn
        norbs = [int(x) for x in device_atom_norbs]
        if sum(norbs) != g.shape[1]:
            raise ValueError(f"device_atom_norbs covers {sum(norbs)} orbitals, the device has {g.shape[1]}")
        atom_of_orb = torch.as_tensor(np.repeat(np.arange(len(norbs)), norbs), device=dev)
        gn_atom = torch.zeros(B, len(norbs), dtype=gn.dtype, device=dev).index_add_(1, atom_of_orb, gn)
        gp_atom = torch.zeros(B, len(norbs), dtype=gp.dtype, device=dev).index_add_(1, atom_of_orb, gp)
        # -potential per atom (a list is taken as values, not repeated as -1 * list would)
        Ei = -torch.as_tensor(potential_at_atom, dtype=torch.float64).to(dev).reshape(1, -1)
        pre = torch.as_tensor(self.pre_factor).to(dev)
        c_e = (pre * 2 * (-1) / 2 / torch.pi).reshape(B, 1)
        c_h = (pre * 2 * 1 / 2 / torch.pi).reshape(B, 1)
        charge = torch.where(e.reshape(B, 1) >= Ei, c_e * gn_atom, c_h * gp_atom).sum(0)
        fc = free_charge[str(kpoint)]
        fc += charge.to(device=fc.device, dtype=fc.dtype)

    def get_subblock_index(self, subblocks, atom_index, device_atom_norbs):
        """Blocks holding atom ``atom_index``'s orbitals, with the first orbital's offset in the
        first of them and the end offset in the last (density.py:362-395)."""
        edges = np.concatenate([[0], np.cumsum(subblocks)])
        first = int(sum(device_atom_norbs[:atom_index]))
        last = first + int(device_atom_norbs[atom_index])
        i = int(np.searchsorted(edges, first, side="right")) - 1
        blocks = [i]
        while last > edges[blocks[-1] + 1]:
            blocks.append(blocks[-1] + 1)
        return blocks, first - int(edges[i]), last - int(edges[blocks[-1]])
