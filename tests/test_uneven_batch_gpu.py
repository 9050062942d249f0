"""Uneven batch (the shape of the 512-device benchmark case, scaled down): many
devices of different block size and length, Ozaki poles plus real-axis points,
per-orbital density and T(E) from one Lopez-Sancho launch and one persistent RGF
launch, FP64 (1e-9 relative) and mixed (refined T within 1e-6; densities within
1e-4 relative) against the oracle applied to each device separately."""
import numpy as np
import pytest
import torch

from oracle import rgf_oracle

pytestmark = pytest.mark.gpu


def _batch(seed=7, nd=8):
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.surface_green import LeadBlocks
    rng = np.random.default_rng(seed)
    devs, leads, raw = [], [], []
    for d in range(nd):
        b = int(rng.integers(1, 7)) * 16   # 16..96, step 16
        L = int(rng.integers(2, 6))        # 2..5 blocks
        dev = workload.random_device(b, L, seed=100 + d)
        raw.append(dev)
        devs.append(rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl))
        lb = lambda ld: LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
        leads.append((lb(dev.lead_L), lb(dev.lead_R)))
    return devs, leads, raw


def _oracle_device(dev, zs, seL, seR, eta, P, R, kBT, res, wlg, df):
    ref = rgf_oracle.rgf(zs, [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL, seR, eta=eta, need_gr_lc=True)
    g = np.concatenate([np.diagonal(b, axis1=1, axis2=2) for b in ref["grd"]], axis=1)  # [E, n_orb]
    n_eq = (1j * R * g[0] - ((-4j * kBT) * g[1:1 + P] * res.reshape(-1, 1)).imag.sum(0)).real
    gam = rgf_oracle.gamma_from_se(seR)
    a = np.concatenate([np.einsum("eij,ejk,eik->ei", c, gam, c.conj()).real for c in ref["gr_lc"]], axis=1)
    n_neq = (wlg.reshape(-1, 1) * a[1 + P:] * df.reshape(-1, 1)).sum(0)
    T = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL), gam)[1 + P:]
    return n_eq, n_neq, T


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_uneven_batch_density_and_transmission(precision):
    from dpnegf_b200.density import Ozaki
    from dpnegf_b200.surface_green import LeadArena, self_energies
    devs, leads, raw = _batch()
    kBT, mu_L, vL, vR, eta_lead, eta_dev = 0.025, 0.05, 0.15, -0.15, 1e-5, 1e-5
    oz = Ozaki(R=1e6, M_cut=8, n_gauss=12)
    fL = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vL)) / kBT))
    fR = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vR)) / kBT))
    out = oz.uneven_batch(devs, leads, kBT, mu_L, vL=vL, vR=vR, fermi_L=fL, fermi_R=fR, eta_lead=eta_lead,
                          eta_device=eta_dev, precision=precision, refine=precision == "mixed")
    # the oracle, device by device, on the same self-energies
    P = len(oz.poles)
    xs = out[0]["energy"].numpy()
    zs = np.concatenate([[1j * oz.R], 1j * oz.poles.numpy() * kBT + mu_L, xs]).astype(np.complex128)
    from oracle import lead_oracle
    _, wlg = lead_oracle.gauss_xw(min(vL, vR) - 8 * kBT, max(vL, vR) + 8 * kBT, oz.n_gauss)
    df = (fR(torch.as_tensor(xs)) - fL(torch.as_tensor(xs))).numpy()
    arena = LeadArena([ld for pair in leads for ld in pair])
    nE = len(zs)
    ls = self_energies(arena, np.repeat(np.arange(2 * len(devs)), nE), np.tile(zs, 2 * len(devs)), eta_lead)
    worst = {"n_eq": 0.0, "n_neq": 0.0, "T": 0.0}
    for d, dev in enumerate(raw):
        seL = torch.stack(ls.sigma[2 * d * nE:(2 * d + 1) * nE]).cpu().numpy()
        seR = torch.stack(ls.sigma[(2 * d + 1) * nE:(2 * d + 2) * nE]).cpu().numpy()
        n_eq, n_neq, T = _oracle_device(dev, zs, seL, seR, eta_dev, P, oz.R, kBT, oz.residues.numpy(), wlg, df)
        got = out[d]
        for name, want, have in (("n_eq", n_eq, got["n_eq"]), ("n_neq", n_neq, got["n_neq"])):
            have = have.cpu().numpy()
            worst[name] = max(worst[name], np.abs(have - want).max() / max(np.abs(want).max(), 1e-300))
        worst["T"] = max(worst["T"], np.abs(got["trans"].cpu().numpy() - T).max())
    print(precision, worst)
    if precision == "fp64":
        assert worst["n_eq"] < 1e-9 and worst["n_neq"] < 1e-9 and worst["T"] < 1e-9, worst
    else:
        assert worst["n_eq"] < 1e-4 and worst["n_neq"] < 1e-4 and worst["T"] < 1e-6, worst
