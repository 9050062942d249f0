"""DeviceProperty / LeadProperty / Ozaki mirrors on the GPU against the
reference fixtures and the oracle (FP64, 1e-10 relative unless stated)."""
import numpy as np
import pytest
import torch

from oracle import lead_oracle, rgf_oracle
from tests.goldens import Golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    b = np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


class FakeHamiltonian:
    """Stands in for NEGFHamiltonianInit: serves fixed BTD blocks and lead blocks."""

    def __init__(self, dev, norbs, leads=None, subblocks=None):
        self._packed = (dev.hd, dev.sd, dev.hl, dev.su, dev.sl, dev.hu)
        self.device_norbs = norbs
        self.leads = leads or {}
        self.subblocks = subblocks

    def get_hs_device(self, kpoint, V=None, block_tridiagonal=True, only_subblocks=False):
        if only_subblocks:
            return self.subblocks
        return self._packed

    def get_hs_lead(self, kpoint, tab, v):
        L = self.leads[tab]
        return (L.hL - v * L.sL, L.hLL - v * L.sLL, L.hDL, L.sL, L.sLL, L.sDL)


class FakeLead:
    def __init__(self, mu, kBT=0.025, voltage=0.0, efermi=0.0):
        self.se = None
        self.chemiPot_lead = mu
        self.kBT = kBT
        self.voltage = voltage
        self.efermi = efermi

    def fermi_dirac(self, x):
        return 1.0 / (1.0 + torch.exp((x - self.chemiPot_lead) / self.kBT))

    @property
    def gamma(self):
        return 1j * (self.se - self.se.mH)


def _devprop_from_golden(g):
    from dpnegf_b200 import workload
    from dpnegf_b200.device_property import DeviceProperty
    dims = list(g["dims"])
    dev = workload.BTDDevice(*[[torch.as_tensor(x) for x in g[k]] for k in ("hd", "hu", "hl", "sd", "su", "sl")])
    dp = DeviceProperty(FakeHamiltonian(dev, list(g["norbs"])), None, "", e_T=300, E_ref=float(g["E_ref"]))
    dp.kBT = float(g["kBT"])
    dp.set_leadLR(FakeLead(float(g["muL"])), FakeLead(float(g["muR"])))
    return dp


@pytest.mark.parametrize("case", ["devprop_nonuniform", "devprop_uniform", "devprop_dense"])
def test_device_property_matches_reference_fixture(case):
    g = Golden(case)
    dp = _devprop_from_golden(g)
    dp.lead_L.se = torch.as_tensor(g["left_se"])
    dp.lead_R.se = torch.as_tensor(g["right_se"])
    dp.cal_green_function(energy=torch.as_tensor(g["energy"]), kpoint=[0.0, 0.0, 0.0],
                          eta_device=float(g["eta_device"]), block_tridiagonal=bool(g["block_tridiagonal"]),
                          need_lesser=True)
    assert _rel(dp.tc, g["out/tc"]) < 1e-10
    assert _rel(dp.dos, g["out/dos"]) < 1e-10
    assert _rel(dp.ldos, g["out/ldos"]) < 1e-10
    for got, want in zip(dp.gnd, g["out/gnd"]):
        assert _rel(got, want) < 1e-10


def test_device_property_scalar_energy_shapes():
    g = Golden("devprop_uniform")
    dp = _devprop_from_golden(g)
    dp.lead_L.se = torch.as_tensor(g["left_se"][1])
    dp.lead_R.se = torch.as_tensor(g["right_se"][1])
    dp.cal_green_function(energy=complex(g["energy"][1]), kpoint=[0.0, 0.0, 0.0],
                          eta_device=float(g["eta_device"]), need_lesser=True)
    assert dp.tc.ndim == 0 and dp.dos.ndim == 0 and dp.ldos.ndim == 1 and dp.grd[0].ndim == 2
    assert _rel(dp.tc, g["out/tc"][1]) < 1e-10
    assert _rel(dp.gnd[0], g["out/gnd"][0][1]) < 1e-10


def test_lead_property_self_energy_batch_matches_oracle():
    from dpnegf_b200 import workload
    from dpnegf_b200.lead_property import LeadProperty
    dev = workload.random_device(24, 4, seed=41)
    ham = FakeHamiltonian(dev, [1] * 96, leads={"lead_L": dev.lead_L, "lead_R": dev.lead_R})
    for tab in ("lead_L", "lead_R"):
        lp = LeadProperty(tab, ham, None, "", voltage=0.05, efermi=0.1)
        E = torch.tensor([-0.8, 0.0, 0.6], dtype=torch.float64)
        lp.self_energy(kpoint=[0.0, 0.0, 0.0], energy=E, eta_lead=1e-5)
        assert lp.se.shape == (3, 24, 24)
        L = (dev.lead_L if tab == "lead_L" else dev.lead_R)
        hL, hLL, hDL, sL, sLL, sDL = ham.get_hs_lead([0, 0, 0], tab, 0.05)
        for i, e in enumerate(E.numpy()):
            sig, _, st, _ = lead_oracle.self_energy(hL.numpy(), hLL.numpy(), sL.numpy(), sLL.numpy(), e,
                                                    hDL.numpy(), sDL.numpy(), etaLead=1e-5, E_ref=0.1)
            assert _rel(lp.se[i], sig) < 1e-9
        lp.self_energy(kpoint=[0.0, 0.0, 0.0], energy=0.6, eta_lead=1e-5)
        assert lp.se.ndim == 2
        g = lp.gamma
        assert torch.allclose(g, g.mH)


def test_hdl_reduced_matches_reference_rule():
    from dpnegf_b200.lead_property import LeadProperty
    H = torch.zeros(6, 4, dtype=torch.complex128)
    H[4:, :] = 1.0
    hr, sr = LeadProperty.HDL_reduced(H, H.clone(), None)
    assert hr.shape == (2, 4)
    H2 = torch.zeros(6, 4, dtype=torch.complex128)
    H2[:3, :] = 1.0
    hr, _ = LeadProperty.HDL_reduced(H2, H2.clone(), None)
    assert hr.shape == (3, 4)
    hr, _ = LeadProperty.HDL_reduced(H2, H2.clone(), [2, 3])
    assert hr.shape == (2, 4)


def _single_block_setup(n=12, seed=3):
    """One-block device with explicit leads (block_tridiagonal=False style)."""
    from dpnegf_b200 import workload
    dev = workload.random_device(n, 3, seed=seed)
    one = workload.BTDDevice([dev.hd[1]], [], [], [dev.sd[1]], [], [])
    return dev, one


def test_ozaki_equilibrium_density_matches_oracle():
    from dpnegf_b200.density import Ozaki
    from dpnegf_b200.device_property import DeviceProperty
    from dpnegf_b200.lead_property import LeadProperty
    dev, one = _single_block_setup()
    n = dev.block_dims[1]
    # leads couple into the single block from both sides
    leads = {"lead_L": dev.lead_L, "lead_R": dev.lead_R}
    ham = FakeHamiltonian(one, [1] * n, leads=leads)
    dp = DeviceProperty(ham, None, "", e_T=300, E_ref=0.0)
    lL = LeadProperty("lead_L", ham, None, "", voltage=0.1, efermi=0.0)
    lR = LeadProperty("lead_R", ham, None, "", voltage=-0.1, efermi=0.0)
    dp.set_leadLR(lL, lR)
    oz = Ozaki(R=1e6, M_cut=20, n_gauss=6)
    DM_eq, DM_neq = oz.integrate(dp, [0.0, 0.0, 0.0], eta_lead=1e-5, eta_device=0.0, mu=0.0,
                                 mu_lead=lL.chemiPot_lead)
    kBT = dp.kBT

    def se(lead, z, eta):
        hL, hLL, hDL, sL, sLL, sDL = ham.get_hs_lead([0, 0, 0], lead.tab, lead.voltage)
        s, _, st, _ = lead_oracle.self_energy(hL.numpy(), hLL.numpy(), sL.numpy(), sLL.numpy(), z, hDL.numpy(),
                                              sDL.numpy(), etaLead=eta, E_ref=0.0)
        return s

    def gf(z, eta=1e-5):
        out = rgf_oracle.rgf(np.array([z]), [], [one.hd[0].numpy()], [], [one.sd[0].numpy()], [], [],
                             se(lL, z, eta)[None], se(lR, z, eta)[None], eta=0.0)
        return out["grd"][0][0]

    def gamma_R(x):
        s = se(lR, x, 1e-5)
        return 1j * (s - s.conj().T)

    # the oracle passes float32 arguments (the reference's float32 bias-window quadrature)
    fL = lambda x: float(lL.fermi_dirac(torch.tensor(x)))
    fR = lambda x: float(lR.fermi_dirac(torch.tensor(x)))
    ref_eq, ref_neq = lead_oracle.ozaki_density(gf, lL.chemiPot_lead, 0.0, kBT, 1e6, 20, 6, lL.voltage,
                                                lR.voltage, fL, fR, gamma_R)
    assert _rel(DM_eq, ref_eq) < 1e-9
    assert _rel(DM_neq, ref_neq) < 1e-9


def test_compute_all_self_energy_batched_and_saved(tmp_path):
    """compute_all_self_energy: every (lead, k) in one decimation launch over the energy grid,
    equal to per-(k, E) selfEnergy (oracle) to 1e-9; its pth files are what
    LeadProperty.self_energy(save_format="pth") then loads."""
    from dpnegf_b200 import workload
    from dpnegf_b200.lead_property import LeadProperty, compute_all_self_energy
    dev = workload.random_device(16, 4, seed=61)
    ham = FakeHamiltonian(dev, [1] * 64, leads={"lead_L": dev.lead_L, "lead_R": dev.lead_R})
    leads = [LeadProperty(t, ham, None, str(tmp_path), voltage=v, efermi=0.1)
             for t, v in (("lead_L", 0.05), ("lead_R", -0.05))]
    ks = [[0.0, 0.0, 0.0], [0.0, 0.25, 0.0]]
    E = [-0.8, -0.1, 0.4, 0.9]
    out = compute_all_self_energy(1e-5, leads[0], leads[1], ks, E, save_format="pth")
    for lp in leads:
        L = dev.lead_L if lp.tab == "lead_L" else dev.lead_R
        for k in ks:
            se = out[lp.tab][tuple(k)]
            assert se.shape == (4, 16, 16)
            hL, hLL, hDL, sL, sLL, sDL = ham.get_hs_lead(k, lp.tab, lp.voltage)
            for i, e in enumerate(E):
                sig = lead_oracle.self_energy(hL.numpy(), hLL.numpy(), sL.numpy(), sLL.numpy(), e,
                                              hDL.numpy(), sDL.numpy(), etaLead=1e-5, E_ref=0.1)[0]
                assert _rel(se[i], sig) < 1e-9
        fresh = LeadProperty(lp.tab, ham, None, str(tmp_path), voltage=lp.voltage, efermi=0.1)
        fresh.self_energy(ks[1], E[2], eta_lead=1e-5, save_format="pth")
        assert torch.equal(fresh.se.cpu(), out[lp.tab][tuple(ks[1])][2].cpu())


def test_runner_nscf_loop_matches_oracle():
    """runner.negf_compute_nscf (one lead launch per (lead, k), one fused sweep per k over all
    energies) gives the oracle's T and DOS per energy, LDOS summing to DOS, T_avg = wk @ T_k."""
    from dpnegf_b200 import workload
    from dpnegf_b200.device_property import DeviceProperty
    from dpnegf_b200.lead_property import LeadProperty
    from dpnegf_b200.runner import negf_compute_nscf
    n = 12
    dev = workload.random_device(n, 4, seed=71)
    ham = FakeHamiltonian(dev, [2] * (2 * n), leads={"lead_L": dev.lead_L, "lead_R": dev.lead_R})
    dp = DeviceProperty(ham, None, "", e_T=300, E_ref=0.1)
    lL = LeadProperty("lead_L", ham, None, "", voltage=0.0, efermi=0.1)
    lR = LeadProperty("lead_R", ham, None, "", voltage=0.0, efermi=0.1)
    dp.set_leadLR(lL, lR)
    E = torch.linspace(-1.0, 1.0, 11, dtype=torch.float64)
    ks, wk = [[0.0, 0.0, 0.0], [0.0, 0.5, 0.0]], [0.25, 0.75]
    out = negf_compute_nscf(dp, ks, wk, E, eta_lead=1e-5, eta_device=1e-5, out_dos=True, out_ldos=True,
                            out_current_nscf=True)
    T_ref, D_ref = [], []
    for e in E.numpy():
        se = []
        for tab in ("lead_L", "lead_R"):
            hL, hLL, hDL, sL, sLL, sDL = ham.get_hs_lead([0, 0, 0], tab, 0.0)
            se.append(lead_oracle.self_energy(hL.numpy(), hLL.numpy(), sL.numpy(), sLL.numpy(), e,
                                              hDL.numpy(), sDL.numpy(), etaLead=1e-5, E_ref=0.1)[0])
        npy = lambda xs: [x.numpy() for x in xs]
        r = rgf_oracle.rgf(np.array([e]), npy(dev.hl), npy(dev.hd), npy(dev.hu), npy(dev.sd), npy(dev.su),
                           npy(dev.sl), se[0][None], se[1][None], E_ref=0.1, eta=1e-5)
        T_ref.append(rgf_oracle.transmission(r["g_trans"], rgf_oracle.gamma_from_se(se[0][None]),
                                             rgf_oracle.gamma_from_se(se[1][None]))[0])
        D_ref.append(rgf_oracle.dos(r["grd"], r["grl"], r["gru"], npy(dev.sd), npy(dev.su), npy(dev.sl))[0])
    for k in ks:
        assert _rel(out["T_k"][str(k)], np.array(T_ref)) < 1e-9
        assert _rel(out["DOS"][str(k)], np.array(D_ref)) < 1e-9
        assert _rel(out["LDOS"][str(k)].sum(-1), np.array(D_ref)) < 1e-9
    assert _rel(out["T_avg"], np.array(T_ref)) < 1e-9
    assert len(out["CURRENT_NSCF"]) == len(out["BIAS_POTENTIAL_NSCF"])
    vv, cc = lead_oracle.current_nscf(E.numpy(), np.array(T_ref), lL.efermi, lL.kBT)
    np.testing.assert_array_equal(out["BIAS_POTENTIAL_NSCF"].cpu().numpy(), vv)
    assert _rel(torch.stack([torch.as_tensor(c) for c in out["CURRENT_NSCF"]]), cc) < 1e-9


def test_local_current_matches_reference_loop():
    """lcurrent (dense device, G^< from the lesser sweep) equals the reference's atom-pair loop
    (device_property.py:491-501) evaluated on the same blocks; antisymmetric, zero diagonal."""
    from dpnegf_b200.device_property import DeviceProperty
    from dpnegf_b200.lead_property import LeadProperty
    dev, one = _single_block_setup()
    n = dev.block_dims[1]
    norbs = [3] * (n // 3)
    ham = FakeHamiltonian(one, norbs, leads={"lead_L": dev.lead_L, "lead_R": dev.lead_R})
    dp = DeviceProperty(ham, None, "", e_T=300, E_ref=0.0)
    lL = LeadProperty("lead_L", ham, None, "", voltage=0.1, efermi=0.0)
    lR = LeadProperty("lead_R", ham, None, "", voltage=-0.1, efermi=0.0)
    dp.set_leadLR(lL, lR)
    k, e = [0.0, 0.0, 0.0], 0.05
    lL.self_energy(kpoint=k, energy=e, eta_lead=1e-5)
    lR.self_energy(kpoint=k, energy=e, eta_lead=1e-5)
    dp.cal_green_function(energy=e, kpoint=k, eta_device=1e-5, block_tridiagonal=False, need_lesser=True)
    lc = dp.lcurrent.cpu().numpy()
    hd = one.hd[0].numpy()
    gnd = dp.gnd[0].cpu().numpy()
    acc = np.cumsum([0] + norbs)
    ref = np.zeros((len(norbs), len(norbs)))
    for i in range(len(norbs)):
        for j in range(len(norbs)):
            if i != j:
                a, b = slice(acc[i], acc[i + 1]), slice(acc[j], acc[j + 1])
                ki = hd[a, b] @ (1j * gnd[b, a])
                kj = hd[b, a] @ (1j * gnd[a, b])
                ref[i, j] = ki.real.diagonal().sum() - kj.real.diagonal().sum()
    assert np.abs(lc - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    assert np.abs(lc + lc.T).max() <= 1e-12 * max(1.0, np.abs(lc).max())
    assert np.abs(ref).max() > 0


def test_bloch_lead_self_energy_matches_reference_loop():
    """Bloch-unfolded lead (bloch_factor [1, 2, 1]): the batched GPU branch against the reference's
    per-unfolded-k loop (lead_property.py:330-379: surface Green's function of each unfolded k,
    phase-kron with exp(2 pi i (R_j - R_i).k), average, reorder, Sigma product), restated here with
    the oracle's decimation."""
    from dpnegf_b200.bloch import Bloch
    from dpnegf_b200.lead_property import LeadProperty
    n, nc = 4, 5
    rng = np.random.default_rng(8)
    c = lambda *s: torch.as_tensor(rng.normal(size=s) * 0.3 + 1j * rng.normal(size=s) * 0.3)
    H0 = c(n, n)
    H0 = (H0 + H0.mH) / 2 + torch.diag(torch.linspace(-1, 1, n)).to(torch.complex128)
    Hy, Hx = c(n, n), c(n, n)
    HDL, SDL = c(nc, 2 * n), 0.02 * c(nc, 2 * n)
    eye, zero = torch.eye(n, dtype=torch.complex128), torch.zeros(n, n, dtype=torch.complex128)

    class BlochHam:
        device_norbs = [1] * nc

        def get_hs_device(self, kpoint, V=None, block_tridiagonal=True, only_subblocks=False):
            return None

        def get_hs_lead(self, k, tab, v):
            ph = complex(np.exp(2j * np.pi * float(k[1])))
            hL = H0 + Hy * ph + Hy.mH * ph.conjugate() - v * eye
            return hL, Hx, HDL, eye, zero, SDL

    R = [torch.tensor([0.0, 0.0, 0.0], dtype=torch.float64), torch.tensor([0.0, 1.0, 0.0], dtype=torch.float64)]
    perm = torch.tensor([1, 0, 3, 2, 5, 4, 7, 6])
    ham = BlochHam()
    lp = LeadProperty("lead_L", ham, None, "", voltage=0.05, efermi=0.1, useBloch=True, bloch_factor=[1, 2, 1],
                      bloch_R_list=R, bloch_sorted_indice=perm, structure_leads_fold=object())
    k = [0.0, 0.13, 0.0]
    E = torch.tensor([-0.4, 0.3], dtype=torch.float64)
    lp.self_energy(kpoint=k, energy=E, eta_lead=1e-3)  # a well-conditioned g_s: this checks the assembly
    for i, e in enumerate(E.tolist()):
        z = e + 0.1 + 1e-3j
        sgf_k = []
        # the reference unfolds from torch.tensor(kpoint): a float32 copy of the k-point (:336-338)
        for kb in Bloch([1, 2, 1]).unfold_points(torch.tensor(k).tolist()):
            hL, hLL, hDL, sL, sLL, sDL = ham.get_hs_lead(torch.tensor(kb), "lead_L", 0.05)
            gs = lead_oracle.surface_green(hL.numpy(), hLL.numpy(), sL.numpy(), sLL.numpy(), z)[0]
            m = np.ones((2, 2), dtype=complex)
            for a in range(2):
                for b in range(2):
                    if a != b:
                        m[a, b] = np.exp(2j * np.pi * float(torch.dot(R[b] - R[a], torch.tensor(kb))))
            sgf_k.append(np.kron(m, gs))
        sgf = np.mean(sgf_k, axis=0)[perm.numpy()][:, perm.numpy()]
        Es = e + 0.1
        ref = (Es * SDL.numpy() - HDL.numpy()) @ sgf[:2 * n, :2 * n] @ (Es * SDL.numpy().conj().T - HDL.numpy().conj().T)
        assert _rel(lp.se[i], ref) < 1e-9


class TableLead(FakeLead):
    """Lead serving a fixture's self-energies, one per grid energy, scalar or batched."""

    def __init__(self, mu, energies, table):
        super().__init__(mu)
        self._keys = [float(x) for x in np.asarray(energies)]
        self._table = torch.as_tensor(table)

    def _lookup(self, energy):
        e = torch.as_tensor(energy).reshape(-1).tolist()
        idx = [min(range(len(self._keys)), key=lambda i: abs(self._keys[i] - x)) for x in e]
        se = self._table[idx]
        return se if torch.as_tensor(energy).ndim else se[0]

    def self_energy(self, kpoint, energy, eta_lead=1e-5, save_path=None, **kw):
        self.se = self._lookup(energy)

    def self_energy_cal(self, kpoint, energy, eta_lead=1e-5, **kw):
        return self._lookup(energy)


@pytest.mark.parametrize("case", ["fiori_dense_direct", "fiori_dense_gauss", "fiori_btd_direct"])
@pytest.mark.parametrize("dirichlet", [True, False])
def test_fiori_free_charge_matches_reference_fixture(case, dirichlet):
    """Fiori per-atom free charge (one lead launch per lead, one sweep over the grid) against the
    reference's own run: 1e-10 relative on the float64 grid, 1e-6 on the float32 Gauss grid
    (float32 Fermi factors on the GPU may differ from the host's by an ulp)."""
    from dpnegf_b200 import workload
    from dpnegf_b200.density import Fiori
    from dpnegf_b200.device_property import DeviceProperty
    g = Golden(case)
    dims, norbs = [int(n) for n in g["dims"]], [int(n) for n in g["norbs"]]
    bt = bool(g["block_tridiagonal"])
    way = str(g["integrate_way"])
    e_grid = torch.as_tensor(g["e_grid"])
    fi = Fiori(n_gauss=6 if way == "gauss" else None, integrate_way=way, e_grid=e_grid)
    assert fi.pre_factor.dtype == torch.float32
    np.testing.assert_array_equal(fi.pre_factor.numpy(), g["pre_factor"])
    np.testing.assert_array_equal(torch.as_tensor(fi.integrate_range).numpy(), g["integrate_range"])
    dev = workload.BTDDevice(*[[torch.as_tensor(x) for x in g[k]] for k in ("hd", "hu", "hl", "sd", "su", "sl")])
    dp = DeviceProperty(FakeHamiltonian(dev, norbs), None, "", e_T=300, E_ref=float(g["E_ref"]))
    dp.kBT = float(g["kBT"])
    dp.set_leadLR(TableLead(float(g["muL"]), g["integrate_range"], g["left_se"]),
                  TableLead(float(g["muR"]), g["integrate_range"], g["right_se"]))
    k = [0.0, 0.0, 0.0]
    fc = {str(k): torch.zeros(len(norbs), dtype=torch.complex128, device="cuda")}
    fi.density_integrate_Fiori(e_grid=e_grid, kpoint=k, Vbias=None, block_tridiagonal=bt, subblocks=dims,
                               integrate_way=way, deviceprop=dp, device_atom_norbs=norbs,
                               potential_at_atom=torch.as_tensor(g["potential_at_atom"]),
                               with_Dirichlet_leads=dirichlet, free_charge=fc, E_ref=float(g["E_ref"]),
                               eta_lead=1e-5, eta_device=float(g["eta_device"]))
    tol = 1e-6 if way == "gauss" else 1e-10
    want = g["out/free_charge"].real
    got = fc[str(k)].real.cpu().numpy()
    print(f"{case}: Fiori free charge relative error {np.abs(got - want).max() / np.abs(want).max():.2e}")
    assert np.abs(got - want).max() < tol * np.abs(want).max()
    for a in range(len(norbs)):
        bl, s0, s1 = fi.get_subblock_index(dims, a, norbs)
        assert list(bl) + [s0, s1] == [int(x) for x in g[f"out/subblock/{a}"]]


class _FixedLeadHamiltonian(FakeHamiltonian):
    """Serves the fixture's lead blocks unshifted by the lead voltage, as the reference run did."""

    def get_hs_lead(self, kpoint, tab, v):
        L = self.leads[tab]
        return (L.hL, L.hLL, L.hDL, L.sL, L.sLL, L.sDL)


def test_ozaki_integrate_matches_reference_fixture():
    """Ozaki.integrate (poles and bias window each in one lead launch per lead and one RGF launch)
    against the reference's own Ozaki.integrate on the same single-block device under +-0.1 V:
    DM_eq and DM_neq within 1e-9 relative (float32 bias-window quadrature as the reference)."""
    from types import SimpleNamespace
    from dpnegf_b200 import workload
    from dpnegf_b200.density import Ozaki
    from dpnegf_b200.device_property import DeviceProperty
    from dpnegf_b200.lead_property import LeadProperty
    g = Golden("ozaki_integrate")
    one = workload.BTDDevice([torch.as_tensor(x) for x in g["hd"]], [], [], [torch.as_tensor(x) for x in g["sd"]],
                             [], [])
    n = one.block_dims[0]
    leads = {t: SimpleNamespace(**{k: torch.as_tensor(g[f"{t}/{k}"]) for k in ("hL", "hLL", "sL", "sLL", "hDL", "sDL")})
             for t in ("lead_L", "lead_R")}
    ham = _FixedLeadHamiltonian(one, [1] * n, leads=leads, subblocks=[n])
    dp = DeviceProperty(ham, None, "", e_T=300, E_ref=0.0)
    assert dp.kBT == float(g["kBT"])
    lL = LeadProperty("lead_L", ham, None, "", voltage=float(g["vL"]), efermi=0.0)
    lR = LeadProperty("lead_R", ham, None, "", voltage=float(g["vR"]), efermi=0.0)
    dp.set_leadLR(lL, lR)
    oz = Ozaki(R=float(g["R"]), M_cut=int(g["M_cut"]), n_gauss=int(g["n_gauss"]))
    DM_eq, DM_neq = oz.integrate(dp, [0.0, 0.0, 0.0], eta_lead=1e-5, eta_device=0.0, mu=0.0,
                                 mu_lead=float(g["mu_L"]))
    print(f"Ozaki.integrate vs reference: DM_eq {_rel(DM_eq, g['out/DM_eq']):.2e}, "
          f"DM_neq {_rel(DM_neq, g['out/DM_neq']):.2e}")
    assert _rel(DM_eq, g["out/DM_eq"]) < 1e-9
    assert _rel(DM_neq, g["out/DM_neq"]) < 1e-9


class _LeadOnlyHamiltonian:
    """Lead blocks shifted by the lead voltage (H - v S) and the device's sub-block sizes."""

    def __init__(self, blocks, subblocks):
        self.blocks, self.subblocks = blocks, subblocks

    def get_hs_device(self, kpoint, V=None, block_tridiagonal=True, only_subblocks=False):
        return self.subblocks

    def get_hs_lead(self, kpoint, tab, v):
        hL, hLL, hDL, sL, sLL, sDL = self.blocks[tab]
        return hL - v * sL, hLL - v * sLL, hDL, sL, sLL, sDL


def test_lead_property_self_energy_matches_reference_fixture():
    """LeadProperty.self_energy against the reference's own: voltage-shifted lead layers, H_DL
    trimmed to the coupled device block by HDL_reduced, E_ref = E_F, Python-float energies
    (float32 as the reference's torch.tensor) and a complex tensor energy; each energy alone and
    all three in one batched launch, within 1e-9 relative."""
    from dpnegf_b200.lead_property import LeadProperty
    g = Golden("lead_property")
    blocks = {t: tuple(torch.as_tensor(g[f"{t}/{k}"]) for k in ("hL", "hLL", "hDL", "sL", "sLL", "sDL"))
              for t in ("lead_L", "lead_R")}
    ham = _LeadOnlyHamiltonian(blocks, [int(x) for x in g["subblocks"]])
    energies = [-0.3, 0.25, torch.tensor(0.1 + 0.2j, dtype=torch.complex128)]
    for tab in ("lead_L", "lead_R"):
        lead = LeadProperty(tab, ham, None, "", voltage=float(g[f"{tab}/voltage"]), efermi=float(g["efermi"]))
        want = [g[f"out/{tab}/se/{i}"] for i in range(3)]
        for e, w in zip(energies, want):
            lead.self_energy(kpoint=[0.0, 0.0, 0.0], energy=e, eta_lead=1e-5, save_path="/nonexistent-negf-se/x.h5")
            assert tuple(lead.se.shape) == w.shape
            assert _rel(lead.se, w) < 1e-9, (tab, e)
        batch = torch.tensor([np.float32(-0.3), np.float32(0.25), 0.1 + 0.2j], dtype=torch.complex128)
        lead.self_energy(kpoint=[0.0, 0.0, 0.0], energy=batch, eta_lead=1e-5)
        for i, w in enumerate(want):
            assert _rel(lead.se[i], w) < 1e-9, (tab, "batched", i)
