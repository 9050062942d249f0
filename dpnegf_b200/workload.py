"""Seeded synthetic block-tridiagonal devices and their leads.

These stand in for the Hamiltonians the dpnegf runner reads from DeePTB models
(negf/negf_hamiltonian_init.py:745-974), which cannot be built offline.  The
tensors come out in the exact layout ``get_hs_device`` / ``get_hs_lead`` hand to
the hot path: per-block 2-D complex128 tensors in lists.

Random Hermitian tight-binding device (block size ``b``, ``L`` blocks):
  * onsite block: real diagonal U[-2, 2] eV plus a Hermitian complex Gaussian
    with sigma = 0.3/sqrt(b);
  * coupling ``hu[q]``: complex Gaussian, sigma = 1.0/sqrt(b); ``hl[q] = hu[q]^H``;
  * overlap: ``sd[q] = I + `` Hermitian complex Gaussian, sigma = 0.01/sqrt(b);
    ``su[q]`` complex Gaussian with the same sigma (non-zero, so the
    energy-dependent off-diagonal path is exercised) and ``sl[q] = su[q]^H``.
Leads repeat the first / last block pair periodically: the left lead's
principal layer is ``(hd[0], sd[0])`` with inter-layer coupling ``hu[0]^H`` and
device coupling ``hDL = hu[0]^H``; the right lead uses ``(hd[-1], sd[-1])``
with ``hu[-1]`` for both couplings.
"""
from dataclasses import dataclass, field
from typing import List, Optional

import math
import torch

C128 = torch.complex128


def _cgauss(gen, shape, sigma):
    re = torch.randn(*shape, generator=gen, dtype=torch.float64)
    im = torch.randn(*shape, generator=gen, dtype=torch.float64)
    return (sigma / math.sqrt(2.0)) * torch.complex(re, im)


def _herm(x):
    return 0.5 * (x + x.mH)


@dataclass
class Lead:
    hL: torch.Tensor
    hLL: torch.Tensor
    sL: torch.Tensor
    sLL: torch.Tensor
    hDL: torch.Tensor
    sDL: torch.Tensor


@dataclass
class BTDDevice:
    hd: List[torch.Tensor]
    hu: List[torch.Tensor]
    hl: List[torch.Tensor]
    sd: List[torch.Tensor]
    su: List[torch.Tensor]
    sl: List[torch.Tensor]
    lead_L: Optional[Lead] = None
    lead_R: Optional[Lead] = None
    norbs_per_atom: List[int] = field(default_factory=list)

    @property
    def block_dims(self):
        return [int(h.shape[0]) for h in self.hd]

    def to(self, device):
        mv = lambda xs: [x.to(device) for x in xs]
        return BTDDevice(mv(self.hd), mv(self.hu), mv(self.hl), mv(self.sd), mv(self.su),
                         mv(self.sl), self.lead_L, self.lead_R, list(self.norbs_per_atom))


def _leads_from_edges(hd, hu, sd, su):
    left = Lead(hL=hd[0], hLL=hu[0].mH.contiguous(), sL=sd[0], sLL=su[0].mH.contiguous(),
                hDL=hu[0].mH.contiguous(), sDL=su[0].mH.contiguous())
    right = Lead(hL=hd[-1], hLL=hu[-1].contiguous(), sL=sd[-1], sLL=su[-1].contiguous(),
                 hDL=hu[-1].contiguous(), sDL=su[-1].contiguous())
    return left, right


def random_device(b, L, seed=0, overlap=True, block_dims=None):
    """Random Hermitian tight-binding BTD device (see module docstring)."""
    gen = torch.Generator().manual_seed(int(seed))
    dims = list(block_dims) if block_dims is not None else [int(b)] * int(L)
    hd, sd, hu, su = [], [], [], []
    for n in dims:
        diag = torch.rand(n, generator=gen, dtype=torch.float64) * 4.0 - 2.0
        h = _herm(_cgauss(gen, (n, n), 0.3 / math.sqrt(n)))
        h = h - torch.diag(torch.diagonal(h)) + torch.diag(diag.to(C128))
        hd.append(h.contiguous())
        s = torch.eye(n, dtype=C128)
        if overlap:
            s = s + _herm(_cgauss(gen, (n, n), 0.01 / math.sqrt(n)))
        sd.append(s.contiguous())
    for q in range(len(dims) - 1):
        n0, n1 = dims[q], dims[q + 1]
        hu.append(_cgauss(gen, (n0, n1), 1.0 / math.sqrt(max(n0, n1))).contiguous())
        if overlap:
            su.append(_cgauss(gen, (n0, n1), 0.01 / math.sqrt(max(n0, n1))).contiguous())
        else:
            su.append(torch.zeros(n0, n1, dtype=C128))
    hl = [u.mH.contiguous() for u in hu]
    sl = [u.mH.contiguous() for u in su]
    dev = BTDDevice(hd, hu, hl, sd, su, sl, norbs_per_atom=[1] * sum(dims))
    if len(dims) >= 2 and dims[0] == dims[1] and dims[-1] == dims[-2]:
        dev.lead_L, dev.lead_R = _leads_from_edges(hd, hu, sd, su)
    return dev


def chain_device(L=10, onsite=0.0, hopping=-1.0, defect=None):
    """Single-orbital 1-D chain with a 2-site principal layer.

    Blocks are 2x2: ``hd = [[e, t], [t, e]]`` and ``hu = [[0, 0], [t, 0]]`` (site 1
    of a layer couples to site 0 of the next).  ``defect`` adds an onsite
    shift to the centre site.  S = I.  Both leads are identical copies.
    """
    e, t = complex(onsite), complex(hopping)
    hd0 = torch.tensor([[e, t], [t, e]], dtype=C128)
    hu0 = torch.tensor([[0, 0], [t, 0]], dtype=C128)
    hd = [hd0.clone() for _ in range(L)]
    if defect is not None:
        site = L  # centre site index among 2L sites
        hd[site // 2][site % 2, site % 2] += complex(defect)
    hu = [hu0.clone() for _ in range(L - 1)]
    hl = [u.mH.contiguous() for u in hu]
    sd = [torch.eye(2, dtype=C128) for _ in range(L)]
    su = [torch.zeros(2, 2, dtype=C128) for _ in range(L - 1)]
    sl = [torch.zeros(2, 2, dtype=C128) for _ in range(L - 1)]
    dev = BTDDevice(hd, hu, hl, sd, su, sl, norbs_per_atom=[1] * (2 * L))
    dev.lead_L = Lead(hL=hd0, hLL=hu0.mH.contiguous(), sL=torch.eye(2, dtype=C128),
                      sLL=torch.zeros(2, 2, dtype=C128), hDL=hu0.mH.contiguous(),
                      sDL=torch.zeros(2, 2, dtype=C128))
    dev.lead_R = Lead(hL=hd0, hLL=hu0.clone(), sL=torch.eye(2, dtype=C128),
                      sLL=torch.zeros(2, 2, dtype=C128), hDL=hu0.clone(),
                      sDL=torch.zeros(2, 2, dtype=C128))
    return dev


def random_self_energy(B, n, seed=0, scale=0.5):
    """Retarded-like self-energies: Hermitian part plus -i * (positive matrix)."""
    gen = torch.Generator().manual_seed(int(seed))
    a = _cgauss(gen, (B, n, n), scale / math.sqrt(n))
    c = _cgauss(gen, (B, n, n), scale / math.sqrt(n))
    return (_herm(a) - 1j * (c @ c.mH + 0.05 * torch.eye(n, dtype=C128))).contiguous()


def energy_grid(n, emin=-3.0, emax=3.0):
    return torch.linspace(emin, emax, n, dtype=torch.float64)
