"""The benchmark workloads at their stated sizes on the GPU, each against the oracle or a
closed form: the b=256, L=64 metric shape, the 1-D chain with a defect (Fisher-Lee), the
b=128, L=48 device with lead-derived self-energies and the lesser diagonal under bias, and the
b=96, L=32 current + density gradient against central finite differences.

Tolerances: FP64 sweep within 1e-10 relative of the oracle; the chain within 2e-4 of the
closed form in the band (the deficit of a clean chain at eta = 1e-6 is 2e-5..4e-5); the
adjoint within 1e-5 max|g| + 1e-4 |g| of central differences with step 1e-6 (normwise over the
64 entries: the summed onsite density counts every occupied state of the 3072 orbitals, so the
loss is large and forward rounding alone puts difference-quotient noise of ~1e-15 |L| / h into
each entry, up to 1e-3 of the smallest checked gradients).
"""
import numpy as np
import pytest
import torch

from oracle import lead_oracle, rgf_oracle

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def _np(xs):
    return [x.numpy() for x in xs]


def _rel(got, want):
    got, want = np.asarray(got), np.asarray(want)
    return float(np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-300)))


def test_metric_shape_fp64_matches_oracle():
    """b=256, L=64 (the benchmark's device and self-energy distribution), 8 energies across
    [-3, 3] eV at eta = 1e-5: T(E), DOS and per-orbital DOS of the FP64 sweep against the
    oracle at 1e-10."""
    from dpnegf_b200 import rgf_plan, workload
    b, L, B = 256, 64, 8
    d = workload.random_device(b, L, seed=3)
    seL = workload.random_self_energy(B, b, seed=101)
    seR = workload.random_self_energy(B, b, seed=102)
    E = torch.linspace(-2.9, 2.9, B, dtype=torch.float64).to(torch.complex128)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl)])
    res = rgf_plan.run(geom, [E.cuda()], [seL.cuda()], [seR.cuda()], eta=1e-5, outputs=(), trans=True,
                       dos=True, orb_dos=True)
    ref = rgf_oracle.rgf(E.numpy(), _np(d.hl), _np(d.hd), _np(d.hu), _np(d.sd), _np(d.su), _np(d.sl),
                         seL.numpy(), seR.numpy(), eta=1e-5)
    T = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL.numpy()),
                                rgf_oracle.gamma_from_se(seR.numpy()))
    D = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], _np(d.sd), _np(d.su), _np(d.sl))
    assert _rel(res.trans.cpu().numpy(), T) < RTOL
    assert _rel(res.dos.cpu().numpy(), D) < RTOL
    orb = res.orb_dos.cpu().numpy().reshape(B, -1)
    orb_ref = rgf_oracle.ldos(ref["grd"], ref["grl"], ref["gru"], _np(d.sd), _np(d.su), _np(d.sl),
                              [1] * (b * L)) / 2.0  # ldos carries the spin factor 2
    scale = np.abs(orb_ref).max()
    assert np.abs(orb - orb_ref).max() < RTOL * scale


def test_defect_chain_matches_fisher_lee():
    """Single-orbital chain (t = -1 eV, 2-site layers, L = 10) with +0.5 eV on the centre site,
    1000 energies in [-3, 3] eV, eta = 1e-6, leads decimated on the GPU to tolerance 1e-10:
    T(E) = (4t^2 - E^2) / (4t^2 - E^2 + e^2) in the band, 0 outside; T and DOS equal the
    oracle's sweep on the same self-energies."""
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.surface_green import LeadArena, LeadBlocks, self_energies
    eps, t = 0.5, -1.0
    chain = workload.chain_device(L=10, defect=eps)
    E = np.linspace(-3.0, 3.0, 1000)
    lb = lambda ld: LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
    arena = LeadArena([lb(chain.lead_L), lb(chain.lead_R)])
    ls = self_energies(arena, np.repeat([0, 1], len(E)), np.tile(E, 2), 1e-6, tol=1e-10)
    seL = torch.stack(ls.sigma[:len(E)])
    seR = torch.stack(ls.sigma[len(E):])
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(chain.hd, chain.hu, chain.hl, chain.sd, chain.su, chain.sl)])
    res = rgf_plan.run(geom, [torch.as_tensor(E).to(torch.complex128).cuda()], [seL], [seR], eta=1e-6,
                       outputs=(), trans=True, dos=True)
    T = res.trans.cpu().numpy()
    band = np.abs(E) < 1.9
    fl = (4 * t * t - E[band] ** 2) / (4 * t * t - E[band] ** 2 + eps ** 2)
    assert np.max(np.abs(T[band] - fl)) < 2e-4, np.max(np.abs(T[band] - fl))
    assert np.all(T[np.abs(E) > 2.1] < 1e-8)
    sL, sR = seL.cpu().numpy(), seR.cpu().numpy()
    ref = rgf_oracle.rgf(E.astype(np.complex128), _np(chain.hl), _np(chain.hd), _np(chain.hu), _np(chain.sd),
                         _np(chain.su), _np(chain.sl), sL, sR, eta=1e-6)
    T_ref = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(sL), rgf_oracle.gamma_from_se(sR))
    D_ref = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], _np(chain.sd), _np(chain.su), _np(chain.sl))
    # absolute on T (it vanishes outside the band); max-norm relative on the DOS (it falls to
    # O(eta) outside the band)
    assert np.max(np.abs(T - T_ref)) < 1e-10
    assert np.max(np.abs(res.dos.cpu().numpy() - D_ref)) < RTOL * np.max(np.abs(D_ref))


def test_config2_lead_self_energies_and_lesser_diagonal():
    """b=128, L=48 device whose leads repeat its first / last block pair: both self-energies by
    the GPU decimation at eta = 1e-5 (against the oracle's decimation), then the retarded and
    lesser sweep with Sigma^in = Gamma_L f_L + Gamma_R f_R at a 0.2 V bias, kT = 25 meV; T(E)
    and the G^< (gnd) diagonal of every block against the oracle sweep at 1e-10."""
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.surface_green import LeadArena, LeadBlocks, self_energies
    b, L = 128, 48
    d = workload.random_device(b, L, seed=2)
    E = np.array([-1.3, -0.2, 0.45, 1.7])
    B = len(E)
    lb = lambda ld: LeadBlocks(ld.hL, ld.hLL, ld.sL, ld.sLL, ld.hDL, ld.sDL)
    arena = LeadArena([lb(d.lead_L), lb(d.lead_R)])
    ls = self_energies(arena, np.repeat([0, 1], B), np.tile(E, 2), 1e-5)
    assert int(np.max(ls.status)) == 0, ls.resid
    seL = torch.stack(ls.sigma[:B]).cpu().numpy()
    seR = torch.stack(ls.sigma[B:]).cpu().numpy()
    for i, e in enumerate(E):
        for side, got in ((d.lead_L, seL[i]), (d.lead_R, seR[i])):
            want, _, st, _ = lead_oracle.self_energy(side.hL.numpy(), side.hLL.numpy(), side.sL.numpy(),
                                                     side.sLL.numpy(), e, side.hDL.numpy(), side.sDL.numpy(),
                                                     etaLead=1e-5)
            assert st == 0
            assert np.abs(got - want).max() < 1e-8 * np.abs(want).max()
    kT, V = 0.025, 0.2
    fL = 1.0 / (1.0 + np.exp((E - V / 2) / kT))
    fR = 1.0 / (1.0 + np.exp((E + V / 2) / kT))
    s_in = rgf_oracle.s_in_from_se(seL, seR, fL, fR, [b] * L)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl)])
    res = rgf_plan.run(geom, [torch.as_tensor(E).to(torch.complex128).cuda()], [torch.as_tensor(seL).cuda()],
                       [torch.as_tensor(seR).cuda()], eta=1e-5, outputs=("gnd",), trans=True,
                       s_in=[[None if s is None else torch.as_tensor(s).cuda() for s in s_in]])
    ref = rgf_oracle.rgf(E.astype(np.complex128), _np(d.hl), _np(d.hd), _np(d.hu), _np(d.sd), _np(d.su),
                         _np(d.sl), seL, seR, eta=1e-5, s_in=s_in, need_lesser=True)
    T_ref = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL), rgf_oracle.gamma_from_se(seR))
    assert _rel(res.trans.cpu().numpy(), T_ref) < RTOL
    got = np.concatenate([np.diagonal(x.cpu().numpy(), axis1=-2, axis2=-1) for x in res.blocks[0]["gnd"]], -1)
    want = np.concatenate([np.diagonal(x, axis1=-2, axis2=-1) for x in ref["gnd"]], -1)
    assert np.abs(got - want).max() < RTOL * np.abs(want).max()


def test_config4_gradient_matches_finite_differences():
    """b=96, L=32, 1024 energies in [-0.3, 0.3] eV; loss = Landauer current at V = 0.3 V,
    kT = 25 meV (trapezoid weights) + the occupied summed onsite density, with both
    self-energies from the GPU decimation of the edge-pair leads (differentiable through the
    decimation fixed point).  The gradient from one adjoint launch (plus the lead chain rule)
    against central differences with h = 1e-6 on 64 random entries: 56 of the device blocks
    (leads at eta = 1e-5) and 8 of the leads' inter-layer couplings.

    The lead entries are checked with the leads broadened to 1e-3: at 1e-5 the self-energies
    have features of width 1e-5 at the leads' band edges (about 20 in this window), so a step of
    1e-6 in a coupling moves them by a tenth of their width and the difference quotient itself is
    off by up to ~1e-3 relative; at 1e-3 the same code path (decimation, implicit-function
    adjoint, lead chain rule) is checked to the tolerance of the device entries."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import lead_self_energy, transmission_dos
    b, L, nE = 96, 32, 1024
    d = workload.random_device(b, L, seed=4242)
    E = torch.linspace(-0.3, 0.3, nE, dtype=torch.float64)
    dx = float(E[1] - E[0])
    tw = torch.full((nE,), dx, dtype=torch.float64)
    tw[0] = tw[-1] = dx / 2
    kT, V = 0.025, 0.3
    fL = 1 / (1 + torch.exp((E - V / 2) / kT))
    fR = 1 / (1 + torch.exp((E + V / 2) / kT))
    wI = ((fL - fR) * tw).cuda()
    wn = (0.5 * (fL + fR) * tw).cuda()
    Ez = E.to(torch.complex128).cuda()
    eta = 1e-5
    names = ("hd", "hu", "hl", "sd", "su", "sl")
    rng = np.random.default_rng(7)
    h = 1e-6

    def sigmas(ld, eta_lead):
        return {s: lead_self_energy(ld[s]["hL"], ld[s]["hLL"], ld[s]["sL"], ld[s]["sLL"], E, eta_lead,
                                    ld[s]["hDL"], ld[s]["sDL"]) for s in ("L", "R")}

    def loss(bl, sig):
        T, D = transmission_dos(bl["hd"], bl["hu"], bl["hl"], bl["sd"], bl["su"], bl["sl"], Ez, sig["L"],
                                sig["R"], eta=eta)
        return (wI * T).sum() + (wn * D).sum()

    def grads(eta_lead):
        blocks = {k: [x.cuda().requires_grad_(True) for x in getattr(d, k)] for k in names}
        lead = {s: {k: getattr(ld, k).cuda() for k in ("hL", "hLL", "sL", "sLL", "hDL", "sDL")}
                for s, ld in (("L", d.lead_L), ("R", d.lead_R))}
        for s in ("L", "R"):
            lead[s]["hLL"].requires_grad_(True)
        Lv = loss(blocks, sigmas(lead, eta_lead))
        Lv.backward()
        return blocks, lead, float(Lv.item())

    checks = []
    # device entries, leads at eta = 1e-5
    blocks, lead, L0 = grads(1e-5)
    with torch.no_grad():
        base = {k: [x.detach().clone() for x in v] for k, v in blocks.items()}
        sig0 = sigmas({s: {k: v.detach() for k, v in lead[s].items()} for s in lead}, 1e-5)
        for _ in range(56):
            name = names[rng.integers(len(names))]
            q = int(rng.integers(len(base[name])))
            i, j = int(rng.integers(base[name][q].shape[0])), int(rng.integers(base[name][q].shape[1]))
            ph = np.exp(2j * np.pi * rng.random())  # a random complex direction of unit modulus

            def shifted(sgn):
                bl = {k: list(v) for k, v in base.items()}
                bl[name][q] = bl[name][q].clone()
                bl[name][q][i, j] += sgn * h * ph
                return loss(bl, sig0).item()

            g = blocks[name][q].grad[i, j].item()
            checks.append(("dev", name, q, i, j, (shifted(1) - shifted(-1)) / (2 * h),
                           g.real * ph.real + g.imag * ph.imag))
    # lead couplings, leads at eta = 1e-3
    blocks, lead, _ = grads(1e-3)
    with torch.no_grad():
        base = {k: [x.detach() for x in v] for k, v in blocks.items()}
        lbase = {s: {k: v.detach().clone() for k, v in lead[s].items()} for s in lead}
        for side in ("L", "R"):
            for _ in range(4):
                i, j = int(rng.integers(b)), int(rng.integers(b))
                ph = np.exp(2j * np.pi * rng.random())

                def shifted(sgn):
                    ld = {s: dict(v) for s, v in lbase.items()}
                    ld[side]["hLL"] = ld[side]["hLL"].clone()
                    ld[side]["hLL"][i, j] += sgn * h * ph
                    return loss(base, sigmas(ld, 1e-3)).item()

                g = lead[side]["hLL"].grad[i, j].item()
                checks.append(("lead", side, 0, i, j, (shifted(1) - shifted(-1)) / (2 * h),
                               g.real * ph.real + g.imag * ph.imag))
    gmax = max(abs(c[6]) for c in checks)
    for kind, name, q, i, j, fd, ad in checks:
        tol = 1e-5 * gmax + 1e-4 * abs(ad)
        assert abs(fd - ad) <= tol, (kind, name, q, i, j, fd, ad, gmax, L0)
