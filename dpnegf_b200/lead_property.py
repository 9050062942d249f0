"""Lead object with GPU self-energies (mirror of negf/lead_property.py).

Same constructor, attributes and methods as the reference ``LeadProperty``
(:30-460): ``self_energy`` sets ``self.se``, ``gamma`` is i(Sigma - Sigma^H),
``fermi_dirac`` uses ``chemiPot_lead = efermi - voltage``.  The self-energy is
computed by the batched Lopez-Sancho kernel; ``energy`` may also be a 1-D
tensor of energies, in which case ``self.se`` is ``[B, n, n]`` from a single
launch (the reference computes one energy per call and stacks them in the
runner, runner/NEGF.py:762-778).  Saved self-energies are found and read as
the reference does (``_get_save_path`` / ``_load_self_energy``: per-(k, E)
``pth`` files, or the per-lead HDF5 files with groups ``E_{e:.8f}`` and
datasets ``k_{k0}_{k1}_{k2}``, the HDF5 form when h5py is importable).
``compute_all_self_energy`` replaces the reference's joblib pool over (k, E)
(negf/lead_property.py:599-683) with one decimation launch per (lead, k) over
the whole energy grid; it returns the self-energies in memory for the sweep
and writes the same files.
"""
import logging
import os
from typing import List

import numpy as np
import torch
from scipy.constants import Boltzmann

from .bloch import Bloch
from .surface_green import LeadArena, LeadBlocks, self_energies
from .products import coupling_sigma

log = logging.getLogger(__name__)
eV2J = 1.6021766208e-19  # J per eV, as in dpnegf/utils/constants.py


class LeadProperty(object):
    def __init__(self, tab, hamiltonian, structure, results_path, voltage,
                 structure_leads_fold=None, bloch_sorted_indice=None, useBloch: bool = False,
                 bloch_factor: List[int] = [1, 1, 1], bloch_R_list=None,
                 e_T=300, efermi: float = 0.0, E_ref: float = None) -> None:
        self.hamiltonian = hamiltonian
        self.structure = structure
        self.tab = tab
        self.voltage = voltage
        self.results_path = results_path
        self.kBT = Boltzmann * e_T / eV2J
        self.e_T = e_T
        self.efermi = efermi
        self.E_ref = efermi if E_ref is None else E_ref
        self.chemiPot_lead = efermi - voltage
        self.kpoint = None
        self.voltage_old = None
        self.useBloch = useBloch
        self.bloch_factor = bloch_factor
        self.bloch_sorted_indice = bloch_sorted_indice
        self.bloch_R_list = bloch_R_list
        self.structure_leads_fold = structure_leads_fold
        self._arena = None
        self._arena_key = None
        if self.useBloch:
            assert self.bloch_sorted_indice is not None
            assert self.bloch_R_list is not None
            assert self.bloch_factor is not None
            assert self.structure_leads_fold is not None

    # ------------------------------------------------------------------ API
    def self_energy(self, kpoint, energy, eta_lead: float = 1e-5, method: str = "Lopez-Sancho",
                    save_path: str = None, save_format: str = "h5", se_info_display: bool = False,
                    HS_inmem: bool = True):
        """Set ``self.se`` for ``kpoint`` at ``energy`` (scalar or [B], relative to E_ref): loaded
        from a saved file when one exists at the reference's path (lead_property.py:105-158, a
        scalar energy), else computed on the GPU."""
        assert len(np.array(kpoint).reshape(-1)) == 3
        if not isinstance(energy, torch.Tensor):
            energy = torch.tensor(energy)
        if energy.ndim == 0:
            path = self._get_save_path(kpoint, energy, save_format, save_path)
            if os.path.isfile(path):
                if se_info_display:
                    log.info(f"Loading {self.tab} self-energy from {path}")
                self.se = self._load_self_energy(path, kpoint, energy, save_format)
                return
        self.se = self.self_energy_cal(kpoint, energy, eta_lead=eta_lead, method=method, HS_inmem=HS_inmem)

    def _get_save_path(self, kpoint, energy, save_format: str, save_path: str = None):
        """File of a saved self-energy, named as the reference names it (lead_property.py:160-218)."""
        kx, ky, kz = np.asarray(kpoint, dtype=float).reshape(3)
        ev = energy.item() if hasattr(energy, "item") else float(energy)
        if save_format not in ("pth", "h5"):
            raise ValueError(f"Unsupported save_format {save_format}, only 'pth' and 'h5' are supported.")
        if save_path is not None and not os.path.isdir(save_path):
            return save_path
        parent = save_path if save_path is not None else os.path.join(self.results_path or "", "self_energy")
        if save_format == "pth":
            return os.path.join(parent, f"se_{self.tab}_k{kx:.4f}_{ky:.4f}_{kz:.4f}_E{ev:.6f}.pth")
        if self.tab not in ("lead_L", "lead_R"):
            raise ValueError(f"Unsupported tab {self.tab} for h5 save.")
        return os.path.join(parent, "self_energy_leadL.h5" if self.tab == "lead_L" else "self_energy_leadR.h5")

    @staticmethod
    def _load_self_energy(save_path: str, kpoint, energy, save_format: str):
        """Read a saved self-energy (lead_property.py:220-264)."""
        if save_format == "pth":
            try:
                return torch.load(save_path, weights_only=False)
            except Exception as e:
                raise IOError(f"Failed to load self-energy from {save_path} (pth format).") from e
        if save_format == "h5":
            ev = energy.item() if hasattr(energy, "item") else float(energy)
            try:
                return torch.as_tensor(read_from_hdf5(save_path, kpoint, ev), dtype=torch.complex128)
            except KeyError as e:
                kx, ky, kz = np.asarray(kpoint, dtype=float).reshape(3)
                raise KeyError(f"Cannot find self-energy in {save_path} for k=({kx:.4f},{ky:.4f},{kz:.4f}), "
                               f"E={ev:.6f}") from e
        raise ValueError(f"Unsupported save_format {save_format}, only 'pth' and 'h5' are supported.")

    def self_energy_cal(self, kpoint, energy, eta_lead: float = 1e-5, method: str = "Lopez-Sancho",
                        se_numba_jit=None, HS_inmem: bool = True):
        if method not in ("Lopez-Sancho",):
            log.warning(f"sgf_solver {method} is not provided; using Lopez-Sancho")
        E = torch.as_tensor(energy).to(torch.complex128).reshape(-1).cpu().numpy()
        scalar = torch.as_tensor(energy).ndim == 0
        subblocks = self.hamiltonian.get_hs_device(kpoint, only_subblocks=True)
        if not self.useBloch:
            key = (tuple(np.asarray(kpoint, dtype=float).reshape(3)), float(self.voltage))
            if self._arena is None or self._arena_key != key:
                self.HLk, self.HLLk, self.HDLk, self.SLk, self.SLLk, self.SDLk = \
                    self.hamiltonian.get_hs_lead(kpoint, tab=self.tab, v=self.voltage)
                self.voltage_old = self.voltage
                self.kpoint = torch.tensor(kpoint)
                hdl, sdl = self.HDL_reduced(torch.as_tensor(self.HDLk), torch.as_tensor(self.SDLk), subblocks)
                self._arena = LeadArena([LeadBlocks(torch.as_tensor(self.HLk), torch.as_tensor(self.HLLk),
                                                    torch.as_tensor(self.SLk), torch.as_tensor(self.SLLk),
                                                    hdl, sdl)])
                self._arena_key = key
            res = self_energies(self._arena, [0] * len(E), E, eta_lead, E_ref=self.E_ref)
            se = torch.stack(res.sigma) if not scalar else res.sigma[0]
        else:
            se = self._bloch_self_energy(kpoint, E, eta_lead, subblocks)
            if scalar:
                se = se[0]
        if not HS_inmem:
            for a in ("HLk", "HLLk", "HDLk", "SLk", "SLLk", "SDLk"):
                if hasattr(self, a):
                    delattr(self, a)
            self._arena = None
        return se

    def _bloch_self_energy(self, kpoint, E, eta_lead, subblocks):
        """Bloch-unfolded lead (reference :330-379): decimate every unfolded k on the
        GPU in one launch, phase-kron and average the surface Green's functions."""
        self.kpoint = torch.tensor(kpoint)
        self.voltage_old = self.voltage
        unfolder = Bloch(self.bloch_factor)
        kps = unfolder.unfold_points(self.kpoint.tolist())
        m_size = int(self.bloch_factor[1] * self.bloch_factor[0])
        leads = []
        for kb in kps:
            hL, hLL, hDL, sL, sLL, sDL = self.hamiltonian.get_hs_lead(torch.tensor(kb), tab=self.tab, v=self.voltage)
            leads.append(LeadBlocks(torch.as_tensor(hL), torch.as_tensor(hLL), torch.as_tensor(sL),
                                    torch.as_tensor(sLL)))
            self.HLk, self.HLLk, self.HDLk, self.SLk, self.SLLk, self.SDLk = hL, hLL, hDL, sL, sLL, sDL
        arena = LeadArena(leads)
        nk, nE = len(kps), len(E)
        idx = [ik for ik in range(nk) for _ in range(nE)]
        res = self_energies(arena, idx, np.tile(E, nk), eta_lead, E_ref=self.E_ref, want_gs=True, want_sigma=False)
        dev = res.gs[0].device
        R = [torch.as_tensor(r, dtype=torch.float64) for r in self.bloch_R_list]
        sgf = None
        for ik, kb in enumerate(kps):
            kbt = torch.tensor(kb, dtype=torch.float64)
            ph = torch.ones(m_size, m_size, dtype=torch.complex128)
            for i in range(m_size):
                for j in range(m_size):
                    if i != j:
                        ph[i, j] = torch.exp(1j * 2 * torch.pi * torch.dot(R[j] - R[i], kbt))
            g = torch.stack(res.gs[ik * nE:(ik + 1) * nE])  # [nE, n, n]
            n1 = g.shape[-1]
            # kron(ph, g[e]) for every energy at once: [e, i n1 + a, j n1 + c] = ph[i, j] g[e, a, c]
            term = (ph.to(dev).view(1, m_size, 1, m_size, 1) * g.view(nE, 1, n1, 1, n1)).reshape(
                nE, m_size * n1, m_size * n1)
            sgf = term if sgf is None else sgf + term
        sgf = sgf / nk
        idxs = torch.as_tensor(self.bloch_sorted_indice, device=dev)
        sgf = sgf[:, idxs, :][:, :, idxs]
        hdl, sdl = self.HDL_reduced(torch.as_tensor(self.HDLk), torch.as_tensor(self.SDLk), subblocks)
        # (E S_DL - H_DL) sgf[:b,:b] (E S_DL^H - H_DL^H) for every energy: the decimation kernel's
        # coupling product on the unfolded surface Green's functions (one launch)
        return coupling_sigma(sgf, hdl, sdl, E, E_ref=self.E_ref)

    @staticmethod
    def HDL_reduced(HDL: torch.Tensor, SDL: torch.Tensor, subblocks) -> torch.Tensor:
        """Trim the lead-device coupling to the coupled device rows (reference :386-434)."""
        assert len(HDL.shape) == 2, "The shape of HDL should be 2."
        assert len(SDL.shape) == 2, "The shape of SDL should be 2."
        assert HDL.shape == SDL.shape, "The shape of HDL and SDL should be the same."
        nz = HDL.nonzero()
        row_min, row_max = nz.min(dim=0).values[0], nz.max(dim=0).values[0]
        if HDL.shape[0] == 1:
            return HDL, SDL
        if row_min > 0:  # right lead: coupled rows sit at the bottom
            cut = row_min if subblocks is None else -1 * subblocks[-1]
            return HDL[cut:, :], SDL[cut:, :]
        cut = row_max + 1 if subblocks is None else subblocks[0]  # left lead
        return HDL[:cut, :], SDL[:cut, :]

    def sigmaLR2Gamma(self, se):
        """Gamma = i (Sigma - Sigma^H)."""
        return 1j * (se - se.mH)

    def fermi_dirac(self, x) -> torch.Tensor:
        return 1 / (1 + torch.exp((x - self.chemiPot_lead) / self.kBT))

    @property
    def gamma(self):
        return self.sigmaLR2Gamma(self.se)


def _h5py():
    try:
        import h5py
    except ImportError as e:
        raise ImportError("the HDF5 self-energy files need h5py (not installed); use save_format='pth'") from e
    return h5py


def hdf5_keys(k, e):
    """Group and dataset name of the self-energy at (k, e) in the per-lead HDF5 files
    (negf/lead_property.py:932-952)."""
    return f"E_{e:.8f}", f"k_{k[0]}_{k[1]}_{k[2]}"


def write_to_hdf5(h5_path, k, e, se):
    h5py = _h5py()
    g, d = hdf5_keys(k, e)
    with h5py.File(h5_path, "a") as f:
        grp = f.require_group(g)
        if d not in grp:
            grp.create_dataset(d, data=torch.as_tensor(se).cpu().numpy(), compression="gzip")


def read_from_hdf5(h5_path, k, e):
    h5py = _h5py()
    g, d = hdf5_keys(k, e)
    with h5py.File(h5_path, "r") as f:
        if g in f and d in f[g]:
            return f[g][d][:]
    raise KeyError(f"Data for kpoint {k} and energy {e} not found.")


def compute_all_self_energy(eta, lead_L, lead_R, kpoints_grid, energy_grid, self_energy_save_path=None,
                            n_jobs=-1, batch_size=200, n_cpus=None, se_numba_jit=None, save_format="h5"):
    """Self-energies of both leads at every (k, E) (negf/lead_property.py:599-683).

    The reference spreads the (k, E) pairs over a joblib process pool and merges
    per-task HDF5 files; here every (lead, k) is one Lopez-Sancho launch over the
    whole energy grid on the GPU (Bloch-unfolded leads included), and the results
    come back in memory as ``{"lead_L": {k: [B, n, n]}, "lead_R": {...}}`` (k as a
    tuple of floats, rows in ``energy_grid`` order) for the sweep to use directly.
    They are also written where the reference writes them: ``save_format="h5"``
    (default, needs h5py) gives ``self_energy_leadL.h5`` / ``self_energy_leadR.h5``
    with groups ``E_{e:.8f}`` and datasets ``k_{k0}_{k1}_{k2}``; ``"pth"`` gives the
    per-(k, E) files ``LeadProperty.self_energy(save_format="pth")`` reads;
    ``None`` writes nothing.  ``n_jobs``, ``batch_size``, ``n_cpus`` and
    ``se_numba_jit`` size the reference's process pool and are accepted for
    compatibility only.
    """
    if self_energy_save_path is None:
        if lead_L.results_path != lead_R.results_path:
            log.warning("The results_path of lead_L and lead_R are different. "
                        "Self energy files will be saved in lead_L's results_path.")
        self_energy_save_path = os.path.join(lead_L.results_path, "self_energy")
    if save_format is not None:
        if save_format == "h5":
            _h5py()
        os.makedirs(self_energy_save_path, exist_ok=True)
    energies = [float(e) for e in np.asarray(energy_grid, dtype=float).reshape(-1)]
    E = torch.tensor(energies, dtype=torch.float64)
    out = {"lead_L": {}, "lead_R": {}}
    seen = []
    for k in kpoints_grid:
        key = tuple(float(x) for x in np.asarray(k, dtype=float).reshape(3))
        if key in seen:
            continue
        seen.append(key)
        for lead in (lead_L, lead_R):
            se = lead.self_energy_cal(kpoint=k, energy=E, eta_lead=eta)
            out[lead.tab][key] = se
            if save_format == "h5":
                path = os.path.join(self_energy_save_path,
                                    "self_energy_leadL.h5" if lead.tab == "lead_L" else "self_energy_leadR.h5")
                for i, e in enumerate(energies):
                    write_to_hdf5(path, k, e, se[i])
            elif save_format == "pth":
                for i, e in enumerate(energies):
                    torch.save(se[i].detach().cpu().clone(),
                               lead._get_save_path(k, torch.tensor(e), "pth", self_energy_save_path))
    return out
