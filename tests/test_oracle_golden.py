"""The numpy oracle reproduces the reference's own outputs (CPU only).

The fixtures were produced by the reference implementation itself
(``tests/golden/make_golden.py``); this pins the oracle before it is used to
check the CUDA path.
"""
import numpy as np
import pytest
import torch

from oracle import lead_oracle, rgf_oracle
from tests.goldens import Golden, rgf_cases

TAGS = rgf_oracle.TAGS


def _close(a, b, atol=1e-10, rtol=1e-10):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape, (a.shape, b.shape)
    np.testing.assert_allclose(a, b, atol=atol, rtol=rtol)


def run_oracle_on(g):
    scalar = bool(g["scalar"])
    kw = dict(eta=float(g["eta"]), E_ref=float(g["E_ref"]),
              need_lesser=g.has("s_in"), need_greater=g.has("s_out"),
              need_gr_lc=g.has("out/gr_lc"))
    return rgf_oracle.rgf(g["energy"], g["hl"], g["hd"], g["hu"], g["sd"], g["su"], g["sl"],
                          g["left_se"], g["right_se"], seP=g.get("seP"), s_in=g.get("s_in"), s_out=g.get("s_out"),
                          **kw)


@pytest.mark.parametrize("case", rgf_cases())
def test_rgf_oracle_matches_reference(case):
    g = Golden(case)
    out = run_oracle_on(g)
    scalar = bool(g["scalar"])
    for t in TAGS:
        key = "out/" + t
        if not g.has(key):
            assert out[t] is None or t == "gr_lc" or t == "gr_left", t
            continue
        ref = g[key]
        mine = out[t]
        if isinstance(ref, list):
            assert len(ref) == len(mine), t
            for r, m in zip(ref, mine):
                _close(m[0] if scalar else m, r)
        else:
            _close(mine[0] if scalar else mine, ref)


@pytest.mark.parametrize("case", ["devprop_nonuniform", "devprop_uniform", "devprop_dense"])
def test_device_traces_match_reference(case):
    g = Golden(case)
    E = g["energy"]
    Eref = float(g["E_ref"])
    dims = list(g["dims"])
    kBT = float(g["kBT"])
    sinL_f = rgf_oracle.fermi_dirac(np.real(E) + Eref, float(g["muL"]), kBT)
    sinR_f = rgf_oracle.fermi_dirac(np.real(E) + Eref, float(g["muR"]), kBT)
    s_in = rgf_oracle.s_in_from_se(g["left_se"], g["right_se"], sinL_f, sinR_f, dims)
    out = rgf_oracle.rgf(E, g["hl"], g["hd"], g["hu"], g["sd"], g["su"], g["sl"],
                         g["left_se"], g["right_se"], E_ref=Eref, eta=float(g["eta_device"]),
                         s_in=s_in, need_lesser=True)
    tc = rgf_oracle.transmission(out["g_trans"], rgf_oracle.gamma_from_se(g["left_se"]),
                                 rgf_oracle.gamma_from_se(g["right_se"]))
    _close(tc, g["out/tc"])
    d = rgf_oracle.dos(out["grd"], out["grl"], out["gru"], g["sd"], g["su"], g["sl"])
    _close(d, g["out/dos"])
    ld = rgf_oracle.ldos(out["grd"], out["grl"], out["gru"], g["sd"], g["su"], g["sl"], list(g["norbs"]))
    _close(ld, g["out/ldos"])
    for r, m in zip(g["out/gnd"], out["gnd"]):
        _close(m, r)


@pytest.mark.parametrize("lead", ["chain", "rand_left", "rand_right"])
def test_lopez_sancho_oracle_matches_reference(lead):
    g = Golden("lopez_sancho")
    p = lead + "/"
    Eref = float(g[p + "E_ref"]) if g.has(p + "E_ref") else 0.0
    eta = float(g[p + "eta"])
    for i, e in enumerate(g[p + "energy"]):
        sig, gs, st, it = lead_oracle.self_energy(g[p + "hL"], g[p + "hLL"], g[p + "sL"], g[p + "sLL"], e,
                                                  g[p + "hDL"], g[p + "sDL"], etaLead=eta, E_ref=Eref)
        assert st in (lead_oracle.LS_OK, lead_oracle.LS_WARN)
        _close(gs, g[p + "gs"][i], atol=1e-9, rtol=1e-8)
        _close(sig, g[p + "sigma"][i], atol=1e-9, rtol=1e-8)


def test_chain_surface_green_is_analytic():
    """1-D chain (t=-1): the lead self-energy is t^2 g_s with g_s the closed form."""
    g = Golden("lopez_sancho")
    for i, e in enumerate(g["chain/energy"]):
        z = complex(e) + 1j * float(g["chain/eta"])
        # surface site Green function of a semi-infinite chain with hopping t=-1
        root = np.sqrt(z * z - 4.0 + 0j)
        gs1 = (z - root) / 2.0
        if gs1.imag > 0:
            gs1 = (z + root) / 2.0
        sig = g["chain/sigma"][i]
        # the single coupled site of the last device block carries t^2 g_s
        assert abs(sig[1, 1] - gs1) < 1e-5, (e, sig[1, 1], gs1)


def test_ozaki_and_gauss_match_reference():
    g = Golden("ozaki")
    for M in (30, 64):
        p, r = lead_oracle.ozaki_residues(M)
        _close(p, g[f"M{M}/poles"], atol=0, rtol=1e-12)
        _close(r, g[f"M{M}/res"], atol=0, rtol=1e-10)
    x, w = lead_oracle.gauss_xw(-0.4, 0.5, 10)
    _close(x, g["gauss/x"], atol=1e-15, rtol=0)
    _close(w, g["gauss/w"], atol=1e-15, rtol=0)


FIORI_CASES = ("fiori_dense_direct", "fiori_dense_gauss", "fiori_btd_direct")


def _fiori_oracle(g):
    mu_l, mu_r, kBT = float(g["muL"]), float(g["muR"]), float(g["kBT"])
    blocks = tuple(g[k] for k in ("hd", "hu", "hl", "sd", "su", "sl"))
    return lead_oracle.fiori_free_charge(
        g["integrate_range"], g["pre_factor"], blocks, g["left_se"], g["right_se"], float(g["eta_device"]),
        float(g["E_ref"]), lambda x: 1.0 / (1.0 + np.exp((x - mu_l) / kBT)),
        lambda x: 1.0 / (1.0 + np.exp((x - mu_r) / kBT)), float(g["E_ref"]), [int(n) for n in g["norbs"]],
        g["potential_at_atom"], bool(g["block_tridiagonal"]), [int(n) for n in g["dims"]])


@pytest.mark.parametrize("case", FIORI_CASES)
def test_fiori_free_charge_matches_reference(case):
    """The Fiori charge restatement against the reference's own Fiori run, within 1e-10 relative.
    The Gauss grid is float32 in the reference (nodes and weights from float32 limits, Fermi
    factors in float32); numpy 2 keeps the same float32 arithmetic here."""
    g = Golden(case)
    got = _fiori_oracle(g)
    want = g["out/free_charge"]
    assert np.abs(got.real - want.real).max() < 1e-10 * np.abs(want.real).max()


@pytest.mark.parametrize("case", FIORI_CASES)
def test_fiori_subblock_index_matches_reference(case):
    g = Golden(case)
    dims, norbs = [int(n) for n in g["dims"]], [int(n) for n in g["norbs"]]
    for a in range(len(norbs)):
        bl, s0, s1 = lead_oracle.fiori_subblock_index(dims, a, norbs)
        assert list(bl) + [s0, s1] == [int(x) for x in g[f"out/subblock/{a}"]]


def test_ozaki_integrate_matches_reference():
    """The Ozaki density restatement against the reference's own Ozaki.integrate (single-block device
    under +-0.1 V, mu set on the fake objects it reads): DM_eq and DM_neq within 1e-10 relative,
    the bias-window quadrature and Fermi factors in float32 as the reference forms them."""
    g = Golden("ozaki_integrate")
    kBT, vL, vR, muL = float(g["kBT"]), float(g["vL"]), float(g["vR"]), float(g["mu_L"])
    leads = {t: [g[f"{t}/{k}"] for k in ("hL", "hLL", "sL", "sLL", "hDL", "sDL")] for t in ("lead_L", "lead_R")}

    def se(t, z, eta=1e-5):
        hL, hLL, sL, sLL, hDL, sDL = leads[t]
        return lead_oracle.self_energy(hL, hLL, sL, sLL, z, hDL, sDL, etaLead=eta, E_ref=0.0)[0]

    def gf(z):
        return rgf_oracle.rgf(np.array([z]), [], g["hd"], [], g["sd"], [], [], se("lead_L", z)[None],
                              se("lead_R", z)[None], eta=0.0)["grd"][0][0]

    def gamma_R(x):
        s = se("lead_R", x)
        return 1j * (s - s.conj().T)

    fL = lambda x: 1.0 / (1.0 + np.exp((x - (0.0 - vL)) / kBT))
    fR = lambda x: 1.0 / (1.0 + np.exp((x - (0.0 - vR)) / kBT))
    eq, neq = lead_oracle.ozaki_density(gf, muL, 0.0, kBT, float(g["R"]), int(g["M_cut"]), int(g["n_gauss"]),
                                        vL, vR, fL, fR, gamma_R)
    for got, want in ((eq, g["out/DM_eq"]), (neq, g["out/DM_neq"])):
        assert np.abs(got - want).max() < 1e-10 * np.abs(want).max()


def test_current_nscf_matches_reference():
    """The NSCF I-V restatement and the product's torch version (CPU tensors) against the reference's
    _cal_current_nscf_: the float32 bias grid exactly, the currents within 1e-12 relative."""
    from types import SimpleNamespace
    from dpnegf_b200.device_property import DeviceProperty
    g = Golden("current_nscf")
    E, tc, efermi, kBT = g["energy"], g["tc"], float(g["efermi"]), float(g["kBT"])
    vv, cc = lead_oracle.current_nscf(E, tc, efermi, kBT)
    np.testing.assert_array_equal(vv, g["out/vv"])
    assert np.abs(cc - g["out/cc"]).max() < 1e-12 * np.abs(g["out/cc"]).max()
    dp = DeviceProperty.__new__(DeviceProperty)
    dp.kBT = kBT
    dp.lead_L = dp.lead_R = SimpleNamespace(efermi=efermi)
    v2, c2 = dp._cal_current_nscf_(torch.as_tensor(E), torch.as_tensor(tc))
    assert v2.dtype == torch.float32
    np.testing.assert_array_equal(v2.numpy(), g["out/vv"])
    c2 = np.array([float(c) for c in c2])
    assert np.abs(c2 - g["out/cc"]).max() < 1e-12 * np.abs(g["out/cc"]).max()


def test_lead_self_energy_restatement_matches_reference_lead_property():
    """The Lopez-Sancho + self-energy restatement against the reference's LeadProperty.self_energy
    (voltage-shifted lead layers, H_DL trimmed to the coupled device block, E_ref = E_F,
    Python-float energies rounded to float32 as the reference's torch.tensor does): 1e-9."""
    g = Golden("lead_property")
    sub = [int(x) for x in g["subblocks"]]
    energies = [float(np.float32(-0.3)), float(np.float32(0.25)), 0.1 + 0.2j]
    for tab in ("lead_L", "lead_R"):
        hL, hLL, hDL, sL, sLL, sDL = (g[f"{tab}/{k}"] for k in ("hL", "hLL", "hDL", "sL", "sLL", "sDL"))
        v = float(g[f"{tab}/voltage"])
        rows = slice(0, sub[0]) if tab == "lead_L" else slice(hDL.shape[0] - sub[-1], hDL.shape[0])
        for i, e in enumerate(energies):
            se = lead_oracle.self_energy(hL - v * sL, hLL - v * sLL, sL, sLL, e, hDL[rows], sDL[rows],
                                         etaLead=1e-5, E_ref=float(g["efermi"]))[0]
            want = g[f"out/{tab}/se/{i}"]
            assert np.abs(se - want).max() < 1e-9 * np.abs(want).max(), (tab, i)


def test_self_energy_bulk_forms_match_reference():
    """selfEnergy without H_DL: (E S - H) - g_s^-1 (and g_s^-1 with Bulk=True) against the
    reference's own, 1e-9."""
    g = Golden("lopez_bulk")
    for i, e in enumerate(g["energy"]):
        sig, gs, st, _ = lead_oracle.self_energy(g["hL"], g["hLL"], g["sL"], g["sLL"], e, etaLead=float(g["eta"]),
                                                 E_ref=float(g["E_ref"]))
        assert st in (lead_oracle.LS_OK, lead_oracle.LS_WARN)
        _close(gs, g["bulk0/gs"][i], atol=1e-9, rtol=1e-8)
        _close(sig, g["bulk0/sigma"][i], atol=1e-9, rtol=1e-8)
        _close(np.linalg.inv(gs), g["bulk1/sigma"][i], atol=1e-9, rtol=1e-8)
