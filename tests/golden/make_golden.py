"""Generate the golden fixtures in this directory by running the REFERENCE code.

Run from the repository root in a container that has the dpnegf sources:

    python tests/golden/make_golden.py --ref-root PATH   (or DPNEGF_REF_ROOT=PATH)

It imports the reference hot path through ``oracle/ref_import.py`` and records
seeded inputs together with the reference's own outputs:

  rgf_*.npz       ``recursive_gf`` (negf/recursive_green_cal.py:324) retarded,
                  lesser and greater cases, uniform and non-uniform blocks,
                  batched and scalar energies, per-block self-energies ``seP``;
  devprop_*.npz   ``DeviceProperty.cal_green_function`` + ``_cal_tc_`` /
                  ``_cal_dos_`` / ``_cal_ldos_`` (negf/device_property.py)
                  driven through the same fakes the reference tests use;
  lopez_*.npz     ``surface_green`` / ``selfEnergy`` (negf/surface_green.py)
                  for the 1-D chain lead and a random non-orthogonal lead, and
                  without H_DL (the bulk forms, ``Bulk`` off and on);
  ozaki.npz       ``ozaki_residues`` (negf/ozaki_res_cal.py) and ``gauss_xw``
                  (negf/negf_utils.py:136);
  adjoint_*.npz   gradients of sum_E w_E T(E) w.r.t. every H/S block and both
                  self-energies by torch autograd through the reference
                  ``recursive_gf`` (T as in ``_cal_tc_``, device_property.py:374-406);
  adjoint_dos_*.npz  the same for sum_E (wT_E T(E) + wD_E DOS(E)), the DOS formed
                  from the reference's blocks as ``_cal_dos_`` does
                  (device_property.py:408-439): the summed onsite density over
                  an energy window when wD carries occupation x quadrature weights;
  fiori_*.npz     ``Fiori.density_integrate_Fiori`` (negf/density.py:268-360):
                  per-atom free charge on a direct and a Gauss grid, dense
                  device (``block_tridiagonal=False``) and BTD device.  The
                  reference's BTD branch reads ``gr_lc`` without requesting it,
                  so for that case the fake device property asks
                  ``cal_green_function`` for it (``need_gr_lc=True``); the
                  leads serve seeded self-energies per grid energy.  Also the
                  reference's ``get_subblock_index`` for every atom;
  ozaki_integrate.npz  ``Ozaki.integrate`` (negf/density.py:143-199) on a
                  single-block device under bias: the reference reads
                  ``deviceprop.mu`` and ``lead_L.mu``, which its classes never
                  set, so the fake device property carries them; the leads
                  compute their self-energies with the reference's own
                  ``selfEnergy`` (as ``LeadProperty.self_energy_cal`` does);
  current_nscf.npz  ``DeviceProperty._cal_current_nscf_`` (negf/device_property.py:333-371):
                  the bias grid and Simpson currents for a smooth T(E);
  lead_property.npz  ``LeadProperty.self_energy`` (negf/lead_property.py:105-158, 266-328):
                  both leads of a two-block device under a lead voltage, H_DL
                  trimmed to the edge block by ``HDL_reduced``, Python-float and
                  complex-tensor energies (a file path that does not exist is
                  given as ``save_path``, so nothing is read or written).
The fixtures are small (tens of KB) and are committed; the GPU box never needs
the reference sources.
"""
import argparse
import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_import  # noqa: E402
from dpnegf_b200 import workload  # noqa: E402


def _put(d, key, val):
    if val is None:
        return
    if isinstance(val, (list, tuple)):
        d[f"{key}#len"] = np.array(len(val))
        for i, v in enumerate(val):
            _put(d, f"{key}/{i}", v)
    else:
        d[key] = val.detach().resolve_conj().cpu().numpy() if torch.is_tensor(val) else np.asarray(val)


def _rgf_case(rgf_mod, name, dims, B, seed, lesser=False, greater=False, scalar=False,
              gr_lc=True, eta=1e-5, E_ref=0.0, sep=False):
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    seL = workload.random_self_energy(B, dims[0], seed=seed + 100)
    seR = workload.random_self_energy(B, dims[-1], seed=seed + 200)
    E = torch.linspace(-1.5, 1.5, B, dtype=torch.float64).to(torch.complex128)
    s_in = s_out = 0
    gen = torch.Generator().manual_seed(seed + 300)
    if lesser:
        s_in = []
        for n in dims:
            x = torch.complex(torch.randn(B, n, n, generator=gen, dtype=torch.float64),
                              torch.randn(B, n, n, generator=gen, dtype=torch.float64))
            s_in.append(0.5 * (x + x.mH))
    if greater:
        s_out = []
        for n in dims:
            x = torch.complex(torch.randn(B, n, n, generator=gen, dtype=torch.float64),
                              torch.randn(B, n, n, generator=gen, dtype=torch.float64))
            s_out.append(0.5 * (x + x.mH))
    seP = None
    if sep:  # per-block self-energy: energy independent (2-D), a 0 placeholder, per energy (3-D)
        c = lambda *sh: torch.complex(torch.randn(*sh, generator=gen, dtype=torch.float64),
                                      -torch.rand(*sh, generator=gen, dtype=torch.float64)) * 0.05
        seP = [c(n, n) if q % 3 == 0 else (0 if q % 3 == 1 else c(B, n, n)) for q, n in enumerate(dims)]
    kw = dict(hl=dev.hl, hd=dev.hd, hu=dev.hu, sd=dev.sd, su=dev.su, sl=dev.sl, eta=eta,
              E_ref=E_ref, need_lesser=lesser, need_greater=greater, need_gr_lc=gr_lc, seP=seP)
    if scalar:
        assert B == 1
        ans = rgf_mod.recursive_gf(E[0], left_se=seL[0], right_se=seR[0],
                                   s_in=[s[0] for s in s_in] if lesser else 0,
                                   s_out=[s[0] for s in s_out] if greater else 0, **kw)
    else:
        ans = rgf_mod.recursive_gf(E, left_se=seL, right_se=seR, s_in=s_in, s_out=s_out, **kw)
    d = {}
    _put(d, "dims", np.array(dims))
    _put(d, "energy", E)
    _put(d, "eta", np.array(eta))
    _put(d, "E_ref", np.array(E_ref))
    _put(d, "scalar", np.array(scalar))
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        _put(d, k, getattr(dev, k))
    _put(d, "left_se", seL)
    _put(d, "right_se", seR)
    if sep:
        _put(d, "seP", seP)
    if lesser:
        _put(d, "s_in", s_in)
    if greater:
        _put(d, "s_out", s_out)
    tags = ("g_trans", "gr_lc", "grd", "grl", "gru", "gr_left",
            "gnd", "gnl", "gnu", "gin_left", "gpd", "gpl", "gpu", "gip_left")
    for t, v in zip(tags, ans):
        _put(d, "out/" + t, v)
    np.savez_compressed(os.path.join(HERE, f"rgf_{name}.npz"), **d)


class _FakeHamiltonian:
    def __init__(self, dev):
        self._packed = (dev.hd, dev.sd, dev.hl, dev.su, dev.sl, dev.hu)
        self.device_norbs = dev.norbs_per_atom

    def get_hs_device(self, kpoint, V, block_tridiagonal):
        return self._packed


class _FakeLead:
    def __init__(self, mu, kBT=0.025):
        self.se = None
        self.chemiPot_lead = mu
        self.kBT = kBT

    def fermi_dirac(self, x):
        return 1.0 / (1.0 + torch.exp((x - self.chemiPot_lead) / self.kBT))

    @property
    def gamma(self):
        return 1j * (self.se - self.se.mH)


def _devprop_case(dp_mod, name, dims, B, seed, norbs, need_lesser=True, block_tridiagonal=True):
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    dev.norbs_per_atom = norbs
    seL = workload.random_self_energy(B, dims[0], seed=seed + 1)
    seR = workload.random_self_energy(B, dims[-1], seed=seed + 2)
    E = torch.linspace(-0.3, 0.4, B, dtype=torch.float64).to(torch.complex128)
    dp = dp_mod.DeviceProperty.__new__(dp_mod.DeviceProperty)
    dp.greenfuncs = 0
    dp.hamiltonian = _FakeHamiltonian(dev)
    dp.structure = None
    dp.results_path = "/nonexistent-negf-results"
    dp.cdtype = torch.complex128
    dp.rgf_device = "cpu"
    dp.kBT = 0.025
    dp.e_T = 300.0
    dp.chemiPot = None
    dp.E_ref = 0.05
    dp.kpoint = None
    dp.newK_flag = None
    dp.newV_flag = None
    dp.lead_L = _FakeLead(0.1)
    dp.lead_R = _FakeLead(-0.1)
    dp.lead_L.se = seL
    dp.lead_R.se = seR
    dp.cal_green_function(energy=E, kpoint=[0.0, 0.0, 0.0], eta_device=1e-6,
                          block_tridiagonal=block_tridiagonal, need_lesser=need_lesser)
    d = {}
    _put(d, "dims", np.array(dims))
    _put(d, "norbs", np.array(norbs))
    _put(d, "energy", E)
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        _put(d, k, getattr(dev, k))
    _put(d, "left_se", seL)
    _put(d, "right_se", seR)
    _put(d, "E_ref", np.array(0.05))
    _put(d, "block_tridiagonal", np.array(block_tridiagonal))
    _put(d, "eta_device", np.array(1e-6))
    _put(d, "muL", np.array(0.1))
    _put(d, "muR", np.array(-0.1))
    _put(d, "kBT", np.array(0.025))
    _put(d, "out/tc", dp._cal_tc_())
    _put(d, "out/dos", dp._cal_dos_())
    _put(d, "out/ldos", dp._cal_ldos_())
    if need_lesser:
        _put(d, "out/gnd", dp.greenfuncs["gnd"])
    np.savez_compressed(os.path.join(HERE, f"devprop_{name}.npz"), **d)


class _TableLead(_FakeLead):
    """Lead whose ``self_energy`` serves a seeded table, one matrix per grid energy."""

    def __init__(self, mu, energies, table):
        super().__init__(mu)
        self._keys = [float(x) for x in energies]
        self._table = table

    def self_energy(self, kpoint, energy, eta_lead=1e-5, save_path=None, **kw):
        self.se = self._table[self._keys.index(float(energy))]


def _fiori_case(dp_mod, dens_mod, name, dims, norbs, block_tridiagonal, integrate_way, seed, nL, nR):
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    e_grid = torch.linspace(-0.4, 0.4, 9, dtype=torch.float64)
    fi = dens_mod.Fiori(n_gauss=6 if integrate_way == "gauss" else None, integrate_way=integrate_way, e_grid=e_grid)
    E = fi.integrate_range
    B = len(E)
    seL = workload.random_self_energy(B, nL, seed=seed + 1)
    seR = workload.random_self_energy(B, nR, seed=seed + 2)
    dp = dp_mod.DeviceProperty.__new__(dp_mod.DeviceProperty)
    dp.greenfuncs = 0
    dp.hamiltonian = _FakeHamiltonian(dev)
    dp.structure = None
    dp.results_path = "/nonexistent-negf-results"
    dp.cdtype = torch.complex128
    dp.rgf_device = "cpu"
    dp.kBT = 0.025
    dp.e_T = 300.0
    dp.chemiPot = None
    dp.E_ref = 0.05
    dp.kpoint = None
    dp.newK_flag = None
    dp.newV_flag = None
    dp.lead_L = _TableLead(0.1, E, seL)
    dp.lead_R = _TableLead(-0.1, E, seR)
    if block_tridiagonal:
        plain = dp.cal_green_function
        dp.cal_green_function = lambda **kw: plain(need_gr_lc=True, **kw)
    gen = torch.Generator().manual_seed(seed + 3)
    pot = torch.rand(len(norbs), generator=gen, dtype=torch.float64) * 0.6 - 0.3
    k = [0.0, 0.0, 0.0]
    fc = {str(k): torch.zeros(len(norbs), dtype=torch.complex128)}
    fi.density_integrate_Fiori(e_grid=e_grid, kpoint=k, Vbias=None, block_tridiagonal=block_tridiagonal,
                               subblocks=dims, integrate_way=integrate_way, deviceprop=dp,
                               device_atom_norbs=norbs, potential_at_atom=pot, with_Dirichlet_leads=True,
                               free_charge=fc, E_ref=0.05, eta_lead=1e-5, eta_device=1e-6)
    d = {}
    _put(d, "dims", np.array(dims))
    _put(d, "norbs", np.array(norbs))
    _put(d, "block_tridiagonal", np.array(block_tridiagonal))
    _put(d, "integrate_way", np.array(integrate_way))
    _put(d, "e_grid", e_grid)
    _put(d, "integrate_range", E)
    _put(d, "pre_factor", fi.pre_factor)
    for key in ("hd", "hu", "hl", "sd", "su", "sl"):
        _put(d, key, getattr(dev, key))
    _put(d, "left_se", seL)
    _put(d, "right_se", seR)
    _put(d, "potential_at_atom", pot)
    _put(d, "E_ref", np.array(0.05))
    _put(d, "eta_device", np.array(1e-6))
    _put(d, "muL", np.array(0.1))
    _put(d, "muR", np.array(-0.1))
    _put(d, "kBT", np.array(0.025))
    _put(d, "out/free_charge", fc[str(k)])
    for a in range(len(norbs)):
        blk, s0, s1 = fi.get_subblock_index(dims, a, norbs)
        _put(d, f"out/subblock/{a}", np.array(list(blk) + [s0, s1]))
    np.savez_compressed(os.path.join(HERE, f"fiori_{name}.npz"), **d)


class _SelfEnergyLead(_FakeLead):
    """Lead whose ``self_energy`` runs the reference's ``selfEnergy`` on fixed lead blocks, as
    ``LeadProperty.self_energy_cal`` does for a non-Bloch lead (lead_property.py:305-328)."""

    def __init__(self, sg_mod, blocks, voltage, efermi, kBT):
        super().__init__(efermi - voltage, kBT)
        self._sg, self._blocks = sg_mod, blocks
        self.voltage, self.efermi = voltage, efermi

    def self_energy(self, kpoint, energy, eta_lead=1e-5, save_path=None, **kw):
        hL, hLL, sL, sLL, hDL, sDL = self._blocks
        if not isinstance(energy, torch.Tensor):  # as LeadProperty.self_energy (lead_property.py:135-136)
            energy = torch.tensor(energy)
        self.se, _ = self._sg.selfEnergy(hL=hL, hLL=hLL, sL=sL, sLL=sLL, ee=energy, hDL=hDL, sDL=sDL,
                                         etaLead=eta_lead, E_ref=0.0)


def _ozaki_integrate_case(dp_mod, dens_mod, sg_mod):
    from scipy.constants import Boltzmann
    kBT = Boltzmann * 300 / 1.6021766208e-19
    dev = workload.random_device(12, 3, seed=3)
    one = workload.BTDDevice([dev.hd[1]], [], [], [dev.sd[1]], [], [])
    lead_blocks = {}
    for tab, ld in (("lead_L", dev.lead_L), ("lead_R", dev.lead_R)):
        lead_blocks[tab] = (ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
    dp = dp_mod.DeviceProperty.__new__(dp_mod.DeviceProperty)
    dp.greenfuncs = 0
    dp.hamiltonian = _FakeHamiltonian(one)
    dp.structure = None
    dp.results_path = "/nonexistent-negf-results"
    dp.cdtype = torch.complex128
    dp.rgf_device = "cpu"
    dp.kBT = kBT
    dp.e_T = 300.0
    dp.chemiPot = None
    dp.E_ref = 0.0
    dp.kpoint = None
    dp.newK_flag = None
    dp.newV_flag = None
    dp.lead_L = _SelfEnergyLead(sg_mod, lead_blocks["lead_L"], 0.1, 0.0, kBT)
    dp.lead_R = _SelfEnergyLead(sg_mod, lead_blocks["lead_R"], -0.1, 0.0, kBT)
    dp.mu = 0.0                                   # mu_D: the device reference level
    dp.lead_L.mu = dp.lead_L.chemiPot_lead        # mu_L: the left lead's chemical potential
    oz = dens_mod.Ozaki(R=1e6, M_cut=20, n_gauss=6)
    DM_eq, DM_neq = oz.integrate(dp, kpoint=[0.0, 0.0, 0.0], eta_lead=1e-5, eta_device=0.0, block_tridiagonal=False)
    d = {}
    _put(d, "hd", one.hd)
    _put(d, "sd", one.sd)
    for tab in ("lead_L", "lead_R"):
        for name, t in zip(("hL", "hLL", "sL", "sLL", "hDL", "sDL"), lead_blocks[tab]):
            _put(d, f"{tab}/{name}", t)
    _put(d, "kBT", np.array(kBT))
    _put(d, "vL", np.array(0.1))
    _put(d, "vR", np.array(-0.1))
    _put(d, "mu_L", np.array(dp.lead_L.mu))
    _put(d, "R", np.array(1e6))
    _put(d, "M_cut", np.array(20))
    _put(d, "n_gauss", np.array(6))
    _put(d, "out/DM_eq", DM_eq)
    _put(d, "out/DM_neq", DM_neq)
    np.savez_compressed(os.path.join(HERE, "ozaki_integrate.npz"), **d)


def _current_case(dp_mod):
    from types import SimpleNamespace
    from scipy.constants import Boltzmann
    dp = dp_mod.DeviceProperty.__new__(dp_mod.DeviceProperty)
    dp.kBT = Boltzmann * 300 / 1.6021766208e-19
    dp.lead_L = SimpleNamespace(efermi=0.1)
    dp.lead_R = SimpleNamespace(efermi=0.1)
    E = torch.linspace(-1.0, 1.0, 41, dtype=torch.float64)
    tc = 1.0 + 0.5 * torch.sin(3 * E) ** 2
    vv, cc = dp._cal_current_nscf_(E, tc)
    d = {}
    _put(d, "energy", E)
    _put(d, "tc", tc)
    _put(d, "efermi", np.array(0.1))
    _put(d, "kBT", np.array(dp.kBT))
    _put(d, "out/vv", vv)
    _put(d, "out/cc", np.array([float(c) for c in cc]))
    np.savez_compressed(os.path.join(HERE, "current_nscf.npz"), **d)


class _LeadHamiltonian:
    """Lead blocks shifted by the lead voltage (H - v S), and the device's sub-block sizes."""

    def __init__(self, blocks, subblocks):
        self.blocks, self.subblocks = blocks, subblocks

    def get_hs_device(self, kpoint, V=None, block_tridiagonal=True, only_subblocks=False):
        return self.subblocks

    def get_hs_lead(self, kpoint, tab, v):
        hL, hLL, hDL, sL, sLL, sDL = self.blocks[tab]
        return hL - v * sL, hLL - v * sLL, hDL, sL, sLL, sDL


def _lead_property_blocks(seed=41, n=4, sub=(5, 7)):
    """Random non-orthogonal lead layers; H_DL / S_DL nonzero only in the rows of the device block
    the lead couples to (the first block for lead_L, the last for lead_R)."""
    gen = torch.Generator().manual_seed(seed)
    c = lambda *s: torch.complex(torch.randn(*s, generator=gen, dtype=torch.float64),
                                 torch.randn(*s, generator=gen, dtype=torch.float64))
    nd = sum(sub)
    blocks = {}
    for tab in ("lead_L", "lead_R"):
        h = c(n, n) * 0.2
        h = 0.5 * (h + h.mH) + torch.diag(torch.linspace(-1.0, 1.0, n, dtype=torch.float64)).to(torch.complex128)
        s = torch.eye(n, dtype=torch.complex128) + 0.01 * (lambda x: 0.5 * (x + x.mH))(c(n, n))
        hLL, sLL = 0.6 * c(n, n) / n ** 0.5, 0.01 * c(n, n) / n ** 0.5
        hDL, sDL = torch.zeros(nd, n, dtype=torch.complex128), torch.zeros(nd, n, dtype=torch.complex128)
        rows = slice(0, sub[0]) if tab == "lead_L" else slice(nd - sub[-1], nd)
        m = sub[0] if tab == "lead_L" else sub[-1]
        hDL[rows] = 0.5 * c(m, n) / n ** 0.5
        sDL[rows] = 0.01 * c(m, n) / n ** 0.5
        blocks[tab] = (h, hLL, hDL, s, sLL, sDL)
    return blocks, list(sub)


def _lead_property_case(lp_mod):
    blocks, sub = _lead_property_blocks()
    ham = _LeadHamiltonian(blocks, sub)
    energies = [-0.3, 0.25, torch.tensor(0.1 + 0.2j, dtype=torch.complex128)]
    d = {}
    _put(d, "subblocks", np.array(sub))
    for tab, v in (("lead_L", 0.05), ("lead_R", -0.05)):
        for name, t in zip(("hL", "hLL", "hDL", "sL", "sLL", "sDL"), blocks[tab]):
            _put(d, f"{tab}/{name}", t)
        _put(d, f"{tab}/voltage", np.array(v))
        lead = lp_mod.LeadProperty(tab, ham, None, "/nonexistent-negf-results", voltage=v, efermi=0.1)
        for i, e in enumerate(energies):
            lead.self_energy(kpoint=[0.0, 0.0, 0.0], energy=e, eta_lead=1e-5,
                             save_path="/nonexistent-negf-se/self_energy.h5")
            _put(d, f"out/{tab}/se/{i}", lead.se)
    _put(d, "efermi", np.array(0.1))
    np.savez_compressed(os.path.join(HERE, "lead_property.npz"), **d)


def _onsite_case(dens_mod):
    """Ozaki.get_density_onsite (negf/density.py:201-230): per-atom sums of diag(DM) beside the
    atom positions, for a matrix and for a vector DM."""
    from types import SimpleNamespace
    gen = torch.Generator().manual_seed(51)
    norbs = [2, 3, 1, 4]
    n = sum(norbs)
    DM = torch.randn(n, n, generator=gen, dtype=torch.float64)
    pos = torch.randn(len(norbs), 3, generator=gen, dtype=torch.float64).numpy()
    dp = SimpleNamespace(norbs_per_atom=norbs, structure=SimpleNamespace(positions=pos))
    oz = dens_mod.Ozaki(R=1e6, M_cut=4, n_gauss=2)
    d = {}
    _put(d, "DM", DM)
    _put(d, "norbs", np.array(norbs))
    _put(d, "positions", pos)
    _put(d, "out/matrix", oz.get_density_onsite(dp, DM))
    _put(d, "out/vector", oz.get_density_onsite(dp, DM.diag() * 2))
    np.savez_compressed(os.path.join(HERE, "density_onsite.npz"), **d)


def _lopez_cases(sg_mod):
    d = {}
    chain = workload.chain_device(L=4)
    ld = chain.lead_R
    es = np.array([-2.5, -1.0, 0.0, 0.7, 1.9, 2.6])
    gs_all, sig_all = [], []
    for e in es:
        gs = sg_mod.surface_green(ld.hL.numpy(), ld.hLL.numpy(), ld.sL.numpy(), ld.sLL.numpy(),
                                  complex(e) + 1e-6j)
        sig, _ = sg_mod.selfEnergy(hL=ld.hL, hLL=ld.hLL, sL=ld.sL, sLL=ld.sLL, ee=float(e),
                                   hDL=ld.hDL, sDL=ld.sDL, etaLead=1e-6)
        gs_all.append(gs)
        sig_all.append(sig.numpy())
    _put(d, "chain/energy", es)
    _put(d, "chain/eta", np.array(1e-6))
    for k in ("hL", "hLL", "sL", "sLL", "hDL", "sDL"):
        _put(d, "chain/" + k, getattr(ld, k))
    _put(d, "chain/gs", np.stack(gs_all))
    _put(d, "chain/sigma", np.stack(sig_all))

    dev = workload.random_device(6, 4, seed=7)
    for side, ld in (("left", dev.lead_L), ("right", dev.lead_R)):
        es = np.array([-1.7, -0.4, 0.3, 1.1])
        gs_all, sig_all = [], []
        for e in es:
            sig, gs = sg_mod.selfEnergy(hL=ld.hL, hLL=ld.hLL, sL=ld.sL, sLL=ld.sLL, ee=float(e),
                                        hDL=ld.hDL, sDL=ld.sDL, etaLead=1e-5, E_ref=0.02)
            gs_all.append(gs.numpy())
            sig_all.append(sig.numpy())
        p = f"rand_{side}/"
        _put(d, p + "energy", es)
        _put(d, p + "eta", np.array(1e-5))
        _put(d, p + "E_ref", np.array(0.02))
        for k in ("hL", "hLL", "sL", "sLL", "hDL", "sDL"):
            _put(d, p + k, getattr(ld, k))
        _put(d, p + "gs", np.stack(gs_all))
        _put(d, p + "sigma", np.stack(sig_all))
    np.savez_compressed(os.path.join(HERE, "lopez_sancho.npz"), **d)


def _lopez_bulk_case(sg_mod):
    """selfEnergy without H_DL: Sigma = (E S - H) - g_s^-1, and with Bulk=True g_s^-1 itself
    (surface_green.py:73-80)."""
    d = {}
    ld = workload.random_device(6, 4, seed=8).lead_R
    es = np.array([-1.3, 0.2, 0.9])
    for bulk in (False, True):
        sig_all, gs_all = [], []
        for e in es:
            sig, gs = sg_mod.selfEnergy(hL=ld.hL, hLL=ld.hLL, sL=ld.sL, sLL=ld.sLL, ee=float(e), etaLead=1e-5,
                                        E_ref=0.05, Bulk=bulk)
            sig_all.append(sig.numpy())
            gs_all.append(gs.numpy())
        _put(d, f"bulk{int(bulk)}/sigma", np.stack(sig_all))
        _put(d, f"bulk{int(bulk)}/gs", np.stack(gs_all))
    _put(d, "energy", es)
    _put(d, "eta", np.array(1e-5))
    _put(d, "E_ref", np.array(0.05))
    for k in ("hL", "hLL", "sL", "sLL"):
        _put(d, k, getattr(ld, k))
    np.savez_compressed(os.path.join(HERE, "lopez_bulk.npz"), **d)


def _ozaki_cases(oz_mod, nu_mod):
    d = {}
    for M in (30, 64):
        p, r = oz_mod.ozaki_residues(M)
        _put(d, f"M{M}/poles", p)
        _put(d, f"M{M}/res", r)
    xs, w = nu_mod.gauss_xw(xl=torch.scalar_tensor(-0.4, dtype=torch.float64),
                            xu=torch.scalar_tensor(0.5, dtype=torch.float64), n=10)
    _put(d, "gauss/x", xs)
    _put(d, "gauss/w", w)
    np.savez_compressed(os.path.join(HERE, "ozaki.npz"), **d)


def _adjoint_case(rgf_mod, name, dims, B, seed, eta=1e-5):
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    leaf = lambda xs: [x.clone().requires_grad_(True) for x in xs]
    hd, hu, hl, sd, su, sl = (leaf(getattr(dev, k)) for k in ("hd", "hu", "hl", "sd", "su", "sl"))
    seL = workload.random_self_energy(B, dims[0], seed=seed + 1).requires_grad_(True)
    seR = workload.random_self_energy(B, dims[-1], seed=seed + 2).requires_grad_(True)
    E = torch.linspace(-1.2, 1.3, B, dtype=torch.float64).to(torch.complex128)
    w = torch.linspace(0.5, 1.5, B, dtype=torch.float64)
    ans = rgf_mod.recursive_gf(E, hl=hl, hd=hd, hu=hu, sd=sd, su=su, sl=sl, left_se=seL, right_se=seR, eta=eta)
    G = ans[0]
    gL = 1j * (seL - seL.mH)
    gR = 1j * (seR - seR.mH)
    T = (gL @ G @ gR @ G.mH).diagonal(dim1=-2, dim2=-1).real.sum(-1)
    (w * T).sum().backward()
    d = {}
    _put(d, "dims", np.array(dims))
    _put(d, "energy", E)
    _put(d, "eta", np.array(eta))
    _put(d, "w", w)
    _put(d, "T", T.detach())
    for k, v in (("hd", hd), ("hu", hu), ("hl", hl), ("sd", sd), ("su", su), ("sl", sl)):
        _put(d, k, [x.detach() for x in v])
        _put(d, "grad/" + k, [x.grad for x in v])
    _put(d, "left_se", seL.detach())
    _put(d, "right_se", seR.detach())
    _put(d, "grad/left_se", seL.grad)
    _put(d, "grad/right_se", seR.grad)
    np.savez_compressed(os.path.join(HERE, f"adjoint_{name}.npz"), **d)


def _adjoint_dos_case(rgf_mod, name, dims, B, seed, with_t, eta=1e-5):
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    leaf = lambda xs: [x.clone().requires_grad_(True) for x in xs]
    hd, hu, hl, sd, su, sl = (leaf(getattr(dev, k)) for k in ("hd", "hu", "hl", "sd", "su", "sl"))
    seL = workload.random_self_energy(B, dims[0], seed=seed + 1).requires_grad_(True)
    seR = workload.random_self_energy(B, dims[-1], seed=seed + 2).requires_grad_(True)
    E = torch.linspace(-1.1, 0.9, B, dtype=torch.float64).to(torch.complex128)
    wT = torch.linspace(0.5, 1.5, B, dtype=torch.float64) if with_t else torch.zeros(B, dtype=torch.float64)
    wD = torch.linspace(1.0, -0.5, B, dtype=torch.float64)
    ans = rgf_mod.recursive_gf(E, hl=hl, hd=hd, hu=hu, sd=sd, su=su, sl=sl, left_se=seL, right_se=seR, eta=eta)
    G, grd, grl, gru = ans[0], ans[2], ans[3], ans[4]
    gL = 1j * (seL - seL.mH)
    gR = 1j * (seR - seR.mH)
    T = (gL @ G @ gR @ G.mH).diagonal(dim1=-2, dim2=-1).real.sum(-1)
    dos = 0
    K = len(grd)
    for j in range(K):  # _cal_dos_ (device_property.py:430-439)
        if K == 1:
            t = grd[j] @ sd[j]
        elif j == 0:
            t = grd[j] @ sd[j] + gru[j] @ sl[j]
        elif j == K - 1:
            t = grd[j] @ sd[j] + grl[j - 1] @ su[j - 1]
        else:
            t = grd[j] @ sd[j] + grl[j - 1] @ su[j - 1] + gru[j] @ sl[j]
        dos = dos - t.imag.diagonal(dim1=-2, dim2=-1).sum(-1) / np.pi
    dos = 2 * dos
    ((wT * T).sum() + (wD * dos).sum()).backward()
    d = {}
    _put(d, "dims", np.array(dims))
    _put(d, "energy", E)
    _put(d, "eta", np.array(eta))
    _put(d, "w", wT)
    _put(d, "wd", wD)
    _put(d, "T", T.detach())
    _put(d, "dos", dos.detach())
    for k, v in (("hd", hd), ("hu", hu), ("hl", hl), ("sd", sd), ("su", su), ("sl", sl)):
        _put(d, k, [x.detach() for x in v])
        _put(d, "grad/" + k, [x.grad for x in v])
    _put(d, "left_se", seL.detach())
    _put(d, "right_se", seR.detach())
    _put(d, "grad/left_se", seL.grad)
    _put(d, "grad/right_se", seR.grad)
    np.savez_compressed(os.path.join(HERE, f"adjoint_dos_{name}.npz"), **d)


def _hdf5_case(lp_mod):
    """The self-energy cache format: the reference's ``write_to_hdf5`` (negf/lead_property.py:932-941)
    for every (k, E) of a k grid and an energy grid, through the dict-backed h5py stand-in of
    tests/fake_h5py.py; records the group / dataset names it creates and the data, and checks that
    its ``read_from_hdf5`` (:944-951) returns them."""
    from tests import fake_h5py
    lp_mod.h5py = fake_h5py.module()
    fake_h5py.FILES.clear()
    kgrid = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [0.25, -0.25, 0.125]])
    egrid = np.array([-1.25, -0.1, 0.0, 0.123456789, 2.5])
    gen = torch.Generator().manual_seed(61)
    d = {}
    _put(d, "kgrid", kgrid)
    _put(d, "egrid", egrid)
    names = []
    for tab in ("L", "R"):
        path = f"/fake/self_energy_lead{tab}.h5"
        for ik, k in enumerate(kgrid):
            for ie, e in enumerate(egrid):
                se = torch.complex(torch.randn(3, 3, generator=gen, dtype=torch.float64),
                                   torch.randn(3, 3, generator=gen, dtype=torch.float64))
                lp_mod.write_to_hdf5(path, k, e, se)
                _put(d, f"se/{tab}/{ik}/{ie}", se)
                back = lp_mod.read_from_hdf5(path, k, e)
                assert np.array_equal(back, se.numpy())
        for g, dsets in fake_h5py.keys(path).items():
            for ds in dsets:
                names.append(f"{tab}|{g}|{ds}")
    d["names"] = np.array(sorted(names))
    np.savez_compressed(os.path.join(HERE, "hdf5_keys.npz"), **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=ref_import.ref_root_from_env(), required=ref_import.ref_root_from_env() is None,
                    help="root of the reference source tree (default: $DPNEGF_REF_ROOT)")
    ap.add_argument("--only", default=None, help="regenerate one family: rgf, devprop, lopez, ozaki, adjoint, fiori, ozaki_integrate, current, lead_property, lopez_bulk, onsite, hdf5")
    args = ap.parse_args()
    torch.set_num_threads(1)  # the container's threaded batched zgesv can hang
    rgf_mod = ref_import.load("recursive_green_cal", args.ref_root)
    sg_mod = ref_import.load("surface_green", args.ref_root)
    dp_mod = ref_import.load("device_property", args.ref_root)
    oz_mod = ref_import.load("ozaki_res_cal", args.ref_root)
    nu_mod = ref_import.load("negf_utils", args.ref_root)
    dens_mod = ref_import.load("density", args.ref_root)

    want = lambda fam: args.only in (None, fam)
    if want("rgf"):
        _rgf_case(rgf_mod, "nonuniform_retarded", [8, 6, 8], 6, seed=1)
        _rgf_case(rgf_mod, "uniform_retarded", [8] * 5, 6, seed=2, E_ref=0.1)
        _rgf_case(rgf_mod, "uniform_lesser", [6] * 4, 4, seed=3, lesser=True)
        _rgf_case(rgf_mod, "nonuniform_lesser", [5, 7, 4], 3, seed=4, lesser=True)
        _rgf_case(rgf_mod, "scalar_retarded", [4, 4, 4], 1, seed=5, scalar=True)
        _rgf_case(rgf_mod, "greater", [4, 5, 4], 3, seed=6, greater=True, lesser=True)
        _rgf_case(rgf_mod, "two_blocks", [3, 3], 2, seed=8)
        _rgf_case(rgf_mod, "wide_uniform", [20] * 4, 2, seed=9, gr_lc=False)
        _rgf_case(rgf_mod, "scattering_seP", [6, 7, 5, 6], 3, seed=10, sep=True)
    if want("devprop"):
        _devprop_case(dp_mod, "nonuniform", [4, 5, 4], 5, seed=10, norbs=[2, 3, 1, 3, 4])
        _devprop_case(dp_mod, "uniform", [6] * 4, 4, seed=11, norbs=[1] * 24)
        _devprop_case(dp_mod, "dense", [9], 4, seed=12, norbs=[2, 3, 4], block_tridiagonal=False)
    if want("lopez"):
        _lopez_cases(sg_mod)
    if want("lopez_bulk"):
        _lopez_bulk_case(sg_mod)
    if want("ozaki"):
        _ozaki_cases(oz_mod, nu_mod)
    if want("adjoint"):
        _adjoint_case(rgf_mod, "nonuniform", [6, 9, 5, 7], 3, seed=21)
        _adjoint_case(rgf_mod, "uniform", [10] * 5, 2, seed=22)
        _adjoint_case(rgf_mod, "single_block", [8], 2, seed=23)
        _adjoint_dos_case(rgf_mod, "nonuniform", [6, 9, 5, 7], 3, seed=24, with_t=False)
        _adjoint_dos_case(rgf_mod, "uniform_with_t", [10] * 5, 2, seed=25, with_t=True)
        _adjoint_dos_case(rgf_mod, "single_block", [8], 2, seed=26, with_t=False)
    if want("lead_property"):
        _lead_property_case(ref_import.load("lead_property", args.ref_root))
    if want("hdf5"):
        _hdf5_case(ref_import.load("lead_property", args.ref_root))
    if want("onsite"):
        _onsite_case(dens_mod)
    if want("current"):
        _current_case(dp_mod)
    if want("ozaki_integrate"):
        _ozaki_integrate_case(dp_mod, dens_mod, sg_mod)
    if want("fiori"):
        _fiori_case(dp_mod, dens_mod, "dense_direct", [9], [2, 3, 4], False, "direct", seed=31, nL=3, nR=4)
        _fiori_case(dp_mod, dens_mod, "dense_gauss", [9], [2, 3, 4], False, "gauss", seed=32, nL=3, nR=4)
        _fiori_case(dp_mod, dens_mod, "btd_direct", [4, 5, 4], [2, 3, 1, 3, 4], True, "direct", seed=33,
                    nL=3, nR=4)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
