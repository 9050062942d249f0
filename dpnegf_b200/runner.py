"""The non-self-consistent transport loop of the NEGF runner on the batched GPU path.

``NEGF.negf_compute`` (runner/NEGF.py:751-816, 904-906) walks the k-points, and
for every chunk of ``e_batch_size`` energies computes each lead's self-energy
one energy at a time (a joblib/numba call per (lead, k, E)), stacks them and
runs one batched ``recursive_gf``; after the loop it forms the k-weighted
``T_avg`` and the non-SCF current.  ``negf_compute_nscf`` is that loop with the
energies of a k-point taken all at once: one Lopez-Sancho launch per lead and
one fused sweep launch (blocks are not materialised; T, DOS and the per-orbital
LDOS are reduced inside the sweep).  It fills the same output keys as the
runner's ``self.out``.  Building the Hamiltonian (DeePTB), SCF with Poisson and
file output stay with the runner.
"""
from typing import Sequence

import numpy as np
import torch


def negf_compute_nscf(deviceprop, kpoints: Sequence, wk: Sequence[float], energies, eta_lead: float = 1e-5,
                      eta_device: float = 0.0, Vbias=None, block_tridiagonal: bool = True, out_tc: bool = True,
                      out_dos: bool = False, out_ldos: bool = False, out_current_nscf: bool = False,
                      self_energy_save_path: str = None, sgf_solver: str = "Lopez-Sancho",
                      e_batch_size: int = None) -> dict:
    """k-resolved T(E), DOS(E), LDOS(E) and their k-average for ``deviceprop`` (a
    ``dpnegf_b200.device_property.DeviceProperty`` with ``lead_L`` / ``lead_R`` set).

    ``energies`` [E] are relative to the reference energy, as the runner's
    ``uni_grid``; ``e_batch_size`` splits them into chunks (default: all at once,
    the GPU path's natural batch).  Returns ``{"k", "wk", "T_k", "DOS", "LDOS",
    "T_avg", "BIAS_POTENTIAL_NSCF", "CURRENT_NSCF"}`` as the runner does (per-k
    entries keyed by ``str(k)``, [E] tensors, LDOS [E, n_atoms])."""
    E = torch.as_tensor(energies, dtype=torch.float64).reshape(-1)
    chunk = e_batch_size or E.shape[0]
    out = {"k": [], "wk": list(wk)}
    need_t = out_tc or out_current_nscf
    for k in kpoints:
        out["k"].append(k)
        for e_chunk in torch.split(E, chunk):
            batched = e_chunk.shape[0] > 1
            e_arg = e_chunk if batched else e_chunk[0]  # one energy: the scalar contract ([n, n] self-energies)
            for lead in (deviceprop.lead_L, deviceprop.lead_R):
                lead.self_energy(kpoint=k, energy=e_arg, eta_lead=eta_lead, method=sgf_solver,
                                 save_path=self_energy_save_path)
            deviceprop.cal_green_function(energy=e_arg, kpoint=k, eta_device=eta_device,
                                          block_tridiagonal=block_tridiagonal, Vbias=Vbias)
            if out_dos:
                d = deviceprop.dos
                out.setdefault("DOS", {}).setdefault(str(k), []).append(d.reshape(-1).cpu())
            if need_t:
                t = deviceprop.tc
                out.setdefault("T_k", {}).setdefault(str(k), []).append(t.reshape(-1).cpu())
            if out_ldos:
                ld = deviceprop.ldos
                out.setdefault("LDOS", {}).setdefault(str(k), []).append((ld if batched else ld.unsqueeze(0)).cpu())
            deviceprop.release_greenfuncs()
        for tag in ("DOS", "T_k", "LDOS"):
            if tag in out:
                out[tag][str(k)] = torch.cat(out[tag][str(k)])
    out["k"] = np.array(out["k"])
    if need_t:
        out["T_avg"] = torch.tensor(out["wk"], dtype=torch.float64) @ torch.stack(list(out["T_k"].values()))
    if out_current_nscf:
        out["BIAS_POTENTIAL_NSCF"], out["CURRENT_NSCF"] = deviceprop._cal_current_nscf_(E, out["T_avg"])
    return out
