"""Adjoint RGF on the GPU: gradients of sum_E w_E T(E) against torch autograd
through the reference recursive_gf (fixtures) and central finite differences
of the CUDA forward sweep."""
import numpy as np
import pytest
import torch

from tests.goldens import Golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else np.asarray(a)
    b = np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _inputs(g):
    cu = lambda xs: [torch.as_tensor(x).cuda().requires_grad_(True) for x in xs]
    blocks = {k: cu(g[k]) for k in ("hd", "hu", "hl", "sd", "su", "sl")}
    seL = torch.as_tensor(g["left_se"]).cuda().requires_grad_(True)
    seR = torch.as_tensor(g["right_se"]).cuda().requires_grad_(True)
    return blocks, seL, seR


@pytest.mark.parametrize("case", ["adjoint_nonuniform", "adjoint_uniform", "adjoint_single_block"])
def test_gradients_match_reference_autograd(case):
    from dpnegf_b200.adjoint import transmission
    g = Golden(case)
    b, seL, seR = _inputs(g)
    E = torch.as_tensor(g["energy"]).cuda()
    T = transmission(b["hd"], b["hu"], b["hl"], b["sd"], b["su"], b["sl"], E, seL, seR, eta=float(g["eta"]))
    assert _rel(T, g["T"]) < 1e-10
    w = torch.as_tensor(g["w"]).cuda()
    (w * T).sum().backward()
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        for q, (x, ref) in enumerate(zip(b[k], g["grad/" + k])):
            assert _rel(x.grad, ref) < 1e-9, (k, q, _rel(x.grad, ref))
    assert _rel(seL.grad, g["grad/left_se"]) < 1e-9
    assert _rel(seR.grad, g["grad/right_se"]) < 1e-9


def test_gradients_match_finite_differences():
    """Central differences (h = 1e-6) of the CUDA forward on random entries."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import transmission
    dims = [12, 16, 12]
    dev = workload.random_device(0, 0, seed=5, block_dims=dims)
    B = 3
    seL = workload.random_self_energy(B, dims[0], seed=6).cuda()
    seR = workload.random_self_energy(B, dims[-1], seed=7).cuda()
    E = torch.tensor([-0.7, 0.1, 0.9], dtype=torch.complex128).cuda()
    w = torch.tensor([1.0, -0.5, 2.0], dtype=torch.float64).cuda()
    blocks = {k: [x.cuda().requires_grad_(True) for x in getattr(dev, k)] for k in ("hd", "hu", "hl", "sd", "su", "sl")}
    seLr = seL.clone().requires_grad_(True)
    seRr = seR.clone().requires_grad_(True)

    def loss(bl, sL, sR):
        T = transmission(bl["hd"], bl["hu"], bl["hl"], bl["sd"], bl["su"], bl["sl"], E, sL, sR, eta=1e-5)
        return (w * T).sum()

    loss(blocks, seLr, seRr).backward()
    rng = np.random.default_rng(0)
    h = 1e-6
    checks = [("hd", 1), ("hu", 0), ("hl", 1), ("sd", 2), ("su", 1), ("sl", 0)]
    with torch.no_grad():
        base = {k: [x.detach().clone() for x in v] for k, v in blocks.items()}
        for name, q in checks:
            X = base[name][q]
            for _ in range(3):
                i, j = rng.integers(X.shape[0]), rng.integers(X.shape[1])
                for part, unit in (("re", 1.0), ("im", 1j)):
                    def shifted(s):
                        bl = {k: [x.clone() for x in v] for k, v in base.items()}
                        bl[name][q][i, j] += s * unit
                        return loss(bl, seL, seR).item()
                    fd = (shifted(h) - shifted(-h)) / (2 * h)
                    gr = blocks[name][q].grad[i, j]
                    ad = gr.real.item() if part == "re" else gr.imag.item()
                    assert abs(fd - ad) <= 1e-6 * max(1.0, abs(ad)), (name, q, i, j, part, fd, ad)
        for which, S, gradS in (("L", seL, seLr.grad), ("R", seR, seRr.grad)):
            for _ in range(3):
                e, i, j = rng.integers(B), rng.integers(S.shape[1]), rng.integers(S.shape[2])
                for part, unit in (("re", 1.0), ("im", 1j)):
                    def shifted(s):
                        S2 = S.clone()
                        S2[e, i, j] += s * unit
                        return loss(base, S2, seR).item() if which == "L" else loss(base, seL, S2).item()
                    fd = (shifted(h) - shifted(-h)) / (2 * h)
                    gr = gradS[e, i, j]
                    ad = gr.real.item() if part == "re" else gr.imag.item()
                    assert abs(fd - ad) <= 1e-6 * max(1.0, abs(ad)), (which, e, i, j, part, fd, ad)


def test_current_gradient_chains_through_simpson():
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import current, transmission
    dims = [10, 10, 10]
    dev = workload.random_device(0, 0, seed=9, block_dims=dims)
    n_e = 9
    E = torch.linspace(-0.3, 0.3, n_e, dtype=torch.float64)
    seL = workload.random_self_energy(n_e, 10, seed=1).cuda()
    seR = workload.random_self_energy(n_e, 10, seed=2).cuda()
    hd1 = dev.hd[1].cuda().requires_grad_(True)
    blocks = [x.cuda() for x in dev.hd]
    kT = 0.025
    fL = 1 / (1 + torch.exp((E - 0.15) / kT))
    fR = 1 / (1 + torch.exp((E + 0.15) / kT))

    def I(h1):
        T = transmission([blocks[0], h1, blocks[2]], [x.cuda() for x in dev.hu], [x.cuda() for x in dev.hl],
                         [x.cuda() for x in dev.sd], [x.cuda() for x in dev.su], [x.cuda() for x in dev.sl],
                         E.to(torch.complex128).cuda(), seL, seR, eta=1e-5)
        return current(T, E.cuda(), fL.cuda(), fR.cuda())

    I(hd1).backward()
    with torch.no_grad():
        h = 1e-6
        d = torch.zeros_like(hd1)
        d[2, 3] = h
        fd = (I(hd1.detach() + d) - I(hd1.detach() - d)).item() / (2 * h)
    assert abs(fd - hd1.grad[2, 3].real.item()) <= 1e-6 * max(1.0, abs(fd))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_value_and_gradient_equals_autograd(precision):
    """transmission_and_grad (one adjoint launch) gives the forward's T(E) and autograd's gradient of
    sum w T: equal to rounding for FP64; for mixed, within the mixed path's tolerance."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import transmission, transmission_and_grad
    dims = [24, 40, 24]
    dev = workload.random_device(0, 0, seed=31, block_dims=dims)
    B = 4
    seL = workload.random_self_energy(B, dims[0], seed=32).cuda()
    seR = workload.random_self_energy(B, dims[-1], seed=33).cuda()
    E = torch.linspace(-1.0, 1.0, B, dtype=torch.float64).to(torch.complex128).cuda()
    w = torch.tensor([0.5, 1.0, -1.5, 2.0], dtype=torch.float64).cuda()
    blocks = {k: [x.cuda().requires_grad_(True) for x in getattr(dev, k)] for k in ("hd", "hu", "hl", "sd", "su", "sl")}
    sL, sR = seL.clone().requires_grad_(True), seR.clone().requires_grad_(True)
    T = transmission(blocks["hd"], blocks["hu"], blocks["hl"], blocks["sd"], blocks["su"], blocks["sl"], E, sL, sR,
                     eta=1e-5, precision=precision)
    (w * T).sum().backward()
    Tf, g = transmission_and_grad(blocks["hd"], blocks["hu"], blocks["hl"], blocks["sd"], blocks["su"],
                                  blocks["sl"], E, seL, seR, w, eta=1e-5, precision=precision)
    tol = 1e-12 if precision == "fp64" else 1e-4
    assert _rel(Tf, T.detach().cpu().numpy()) < tol
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        for q, x in enumerate(blocks[k]):
            assert _rel(g[k][q], x.grad.cpu().numpy()) < tol, (k, q)
    assert _rel(g["se_l"], sL.grad.cpu().numpy()) < tol
    assert _rel(g["se_r"], sR.grad.cpu().numpy()) < tol


@pytest.mark.parametrize("case", ["adjoint_dos_nonuniform", "adjoint_dos_uniform_with_t", "adjoint_dos_single_block"])
def test_density_gradients_match_reference_autograd(case):
    """Gradient of sum wT T + sum wD DOS (DOS as the reference's _cal_dos_) against torch autograd
    through the reference recursive_gf (fixtures; the first and last cases have wT = 0)."""
    from dpnegf_b200.adjoint import transmission_dos
    g = Golden(case)
    b, seL, seR = _inputs(g)
    E = torch.as_tensor(g["energy"]).cuda()
    T, D = transmission_dos(b["hd"], b["hu"], b["hl"], b["sd"], b["su"], b["sl"], E, seL, seR, eta=float(g["eta"]))
    assert _rel(T, g["T"]) < 1e-10
    assert _rel(D, g["dos"]) < 1e-10
    wT = torch.as_tensor(g["w"]).cuda()
    wD = torch.as_tensor(g["wd"]).cuda()
    ((wT * T).sum() + (wD * D).sum()).backward()
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        for q, (x, ref) in enumerate(zip(b[k], g["grad/" + k])):
            assert _rel(x.grad, ref) < 1e-9, (k, q, _rel(x.grad, ref))
    assert _rel(seL.grad, g["grad/left_se"]) < 1e-9
    assert _rel(seR.grad, g["grad/right_se"]) < 1e-9


def test_density_gradient_matches_finite_differences():
    """Central differences (h = 1e-6) of the CUDA DOS on random H, S and Sigma entries."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import transmission_dos
    dims = [14, 10, 16]
    dev = workload.random_device(0, 0, seed=15, block_dims=dims)
    B = 3
    seL = workload.random_self_energy(B, dims[0], seed=16).cuda()
    seR = workload.random_self_energy(B, dims[-1], seed=17).cuda()
    E = torch.tensor([-0.6, 0.2, 1.1], dtype=torch.complex128).cuda()
    wD = torch.tensor([0.7, -1.2, 0.4], dtype=torch.float64).cuda()
    blocks = {k: [x.cuda().requires_grad_(True) for x in getattr(dev, k)] for k in ("hd", "hu", "hl", "sd", "su", "sl")}
    seLr = seL.clone().requires_grad_(True)
    seRr = seR.clone().requires_grad_(True)

    def loss(bl, sL, sR):
        _, D = transmission_dos(bl["hd"], bl["hu"], bl["hl"], bl["sd"], bl["su"], bl["sl"], E, sL, sR, eta=1e-5)
        return (wD * D).sum()

    loss(blocks, seLr, seRr).backward()
    rng = np.random.default_rng(1)
    h = 1e-6
    with torch.no_grad():
        base = {k: [x.detach().clone() for x in v] for k, v in blocks.items()}
        for name, q in (("hd", 0), ("hd", 2), ("hu", 1), ("hl", 0), ("sd", 1), ("su", 0), ("sl", 1)):
            X = base[name][q]
            for _ in range(2):
                i, j = rng.integers(X.shape[0]), rng.integers(X.shape[1])
                for part, unit in (("re", 1.0), ("im", 1j)):
                    def shifted(s):
                        bl = {k: [x.clone() for x in v] for k, v in base.items()}
                        bl[name][q][i, j] += s * unit
                        return loss(bl, seL, seR).item()
                    fd = (shifted(h) - shifted(-h)) / (2 * h)
                    gr = blocks[name][q].grad[i, j]
                    ad = gr.real.item() if part == "re" else gr.imag.item()
                    assert abs(fd - ad) <= 1e-5 * max(1.0, abs(ad)), (name, q, i, j, part, fd, ad)
        for which, S, gradS in (("L", seL, seLr.grad), ("R", seR, seRr.grad)):
            e, i, j = rng.integers(B), rng.integers(S.shape[1]), rng.integers(S.shape[2])
            for part, unit in (("re", 1.0), ("im", 1j)):
                def shifted(s):
                    S2 = S.clone()
                    S2[e, i, j] += s * unit
                    return loss(base, S2, seR).item() if which == "L" else loss(base, seL, S2).item()
                fd = (shifted(h) - shifted(-h)) / (2 * h)
                gr = gradS[e, i, j]
                ad = gr.real.item() if part == "re" else gr.imag.item()
                assert abs(fd - ad) <= 1e-5 * max(1.0, abs(ad)), (which, e, i, j, part, fd, ad)


def test_fused_current_and_density_gradient_equals_autograd():
    """One adjoint launch for sum wT T + sum wD DOS equals autograd through transmission_dos."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import transmission_and_grad, transmission_dos
    dims = [32, 32, 32, 32]
    dev = workload.random_device(0, 0, seed=41, block_dims=dims)
    B = 4
    seL = workload.random_self_energy(B, 32, seed=42).cuda()
    seR = workload.random_self_energy(B, 32, seed=43).cuda()
    E = torch.linspace(-0.8, 0.8, B, dtype=torch.float64).to(torch.complex128).cuda()
    wT = torch.tensor([1.0, 0.5, -0.25, 2.0], dtype=torch.float64).cuda()
    wD = torch.tensor([0.3, 0.3, 0.3, 0.3], dtype=torch.float64).cuda()
    blocks = {k: [x.cuda().requires_grad_(True) for x in getattr(dev, k)] for k in ("hd", "hu", "hl", "sd", "su", "sl")}
    sL, sR = seL.clone().requires_grad_(True), seR.clone().requires_grad_(True)
    T, D = transmission_dos(blocks["hd"], blocks["hu"], blocks["hl"], blocks["sd"], blocks["su"], blocks["sl"],
                            E, sL, sR, eta=1e-5)
    ((wT * T).sum() + (wD * D).sum()).backward()
    Tf, g = transmission_and_grad(blocks["hd"], blocks["hu"], blocks["hl"], blocks["sd"], blocks["su"],
                                  blocks["sl"], E, seL, seR, wT, eta=1e-5, dos_weights=wD)
    assert _rel(Tf, T.detach().cpu().numpy()) < 1e-12
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        for q, x in enumerate(blocks[k]):
            assert _rel(g[k][q], x.grad.cpu().numpy()) < 1e-12, (k, q)
    assert _rel(g["se_l"], sL.grad.cpu().numpy()) < 1e-12
    assert _rel(g["se_r"], sR.grad.cpu().numpy()) < 1e-12


def test_mixed_density_gradient_close_to_fp64():
    """The mixed-precision (3xTF32 products) current + density gradient stays within the mixed
    path's block tolerance (1e-3 relative) of the FP64 one on a short chain."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import transmission_and_grad
    dims = [48, 48, 48]
    dev = workload.random_device(0, 0, seed=51, block_dims=dims)
    B = 3
    seL = workload.random_self_energy(B, 48, seed=52).cuda()
    seR = workload.random_self_energy(B, 48, seed=53).cuda()
    E = torch.tensor([-0.4, 0.1, 0.5], dtype=torch.complex128).cuda()
    wT = torch.tensor([1.0, 1.0, 1.0], dtype=torch.float64).cuda()
    wD = torch.tensor([0.5, 0.5, 0.5], dtype=torch.float64).cuda()
    blocks = {k: [x.cuda() for x in getattr(dev, k)] for k in ("hd", "hu", "hl", "sd", "su", "sl")}
    args = (blocks["hd"], blocks["hu"], blocks["hl"], blocks["sd"], blocks["su"], blocks["sl"], E, seL, seR, wT)
    T64, g64 = transmission_and_grad(*args, eta=1e-5, dos_weights=wD)
    Tmx, gmx = transmission_and_grad(*args, eta=1e-5, dos_weights=wD, precision="mixed")
    assert _rel(Tmx, T64.cpu().numpy()) < 1e-3
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        for q in range(len(g64[k])):
            assert _rel(gmx[k][q], g64[k][q].cpu().numpy()) < 1e-3, (k, q)


def _lead(n, nc, seed):
    rng = np.random.default_rng(seed)
    c = lambda shape, s: torch.as_tensor(rng.normal(size=shape) * s + 1j * rng.normal(size=shape) * s)
    h = c((n, n), 0.3)
    hL = (h + h.mH) / 2 + torch.diag(torch.linspace(-1, 1, n)).to(torch.complex128)
    s = c((n, n), 0.02)
    sL = torch.eye(n, dtype=torch.complex128) + (s + s.mH) / 2
    return [x.cuda() for x in (hL, c((n, n), 0.5), sL, c((n, n), 0.02), c((nc, n), 0.5), c((nc, n), 0.02))]


def test_lead_self_energy_gradient_matches_finite_differences():
    """dL/d(H, H01, S, S01, H_DL, S_DL) of a lead through the decimation fixed point (implicit
    adjoint) against central differences of the CUDA decimation; Sigma itself against the oracle."""
    from oracle import lead_oracle
    from dpnegf_b200.adjoint import lead_self_energy
    n, nc = 6, 5
    base = _lead(n, nc, seed=3)
    E = torch.tensor([-0.7, 0.2, 0.9], dtype=torch.float64)
    eta = 1e-3
    rng = np.random.default_rng(4)
    W = torch.as_tensor(rng.normal(size=(3, nc, nc)) + 1j * rng.normal(size=(3, nc, nc))).cuda()

    def loss(bl):
        sig = lead_self_energy(*bl[:4], E, eta, hDL=bl[4], sDL=bl[5])
        return (W * sig).sum().real, sig

    leaves = [x.clone().requires_grad_(True) for x in base]
    L0, sig = loss(leaves)
    for e in range(3):
        ref = lead_oracle.self_energy(*(x.cpu().numpy() for x in base[:4]), float(E[e]),
                                      base[4].cpu().numpy(), base[5].cpu().numpy(), etaLead=eta)[0]
        assert _rel(sig[e], ref) < 1e-9
    L0.backward()
    h = 1e-6
    with torch.no_grad():
        for k in range(6):
            X = leaves[k]
            for _ in range(2):
                i, j = rng.integers(X.shape[0]), rng.integers(X.shape[1])
                for part, unit in (("re", 1.0), ("im", 1j)):
                    def shifted(sgn):
                        bl = [x.clone() for x in base]
                        bl[k][i, j] += sgn * h * unit
                        return loss(bl)[0].item()
                    fd = (shifted(1) - shifted(-1)) / (2 * h)
                    ad = X.grad[i, j].real.item() if part == "re" else X.grad[i, j].imag.item()
                    assert abs(fd - ad) <= 1e-5 * max(1.0, abs(ad)), (k, i, j, part, fd, ad)


def test_transmission_gradient_reaches_lead_blocks():
    """T(E) with Sigma_L from lead_self_energy: d(sum T)/d(lead H01) by autograd (device adjoint ->
    dT/dSigma -> decimation adjoint) against central differences."""
    from dpnegf_b200 import workload
    from dpnegf_b200.adjoint import lead_self_energy, transmission
    n = 8
    hL, hLL, sL, sLL, hDL, sDL = _lead(n, n, seed=7)
    dims = [n, 10, n]
    dev = workload.random_device(0, 0, seed=8, block_dims=dims)
    blocks = [[x.cuda() for x in getattr(dev, k)] for k in ("hd", "hu", "hl", "sd", "su", "sl")]
    E = torch.tensor([-0.5, 0.3], dtype=torch.float64)
    seR = workload.random_self_energy(2, n, seed=9).cuda()

    def total(h01):
        sigL = lead_self_energy(hL, h01, sL, sLL, E, 1e-3, hDL=hDL, sDL=sDL)
        T = transmission(*blocks, E.to(torch.complex128).cuda(), sigL, seR, eta=1e-5)
        return T.sum()

    h01 = hLL.clone().requires_grad_(True)
    total(h01).backward()
    h = 1e-6
    with torch.no_grad():
        for (i, j) in ((0, 1), (3, 5)):
            for part, unit in (("re", 1.0), ("im", 1j)):
                d = torch.zeros_like(hLL)
                d[i, j] = h * unit
                fd = (total(hLL + d) - total(hLL - d)).item() / (2 * h)
                ad = h01.grad[i, j].real.item() if part == "re" else h01.grad[i, j].imag.item()
                assert abs(fd - ad) <= 1e-5 * max(1.0, abs(ad)), (i, j, part, fd, ad)


@pytest.mark.parametrize("dims,ckpt", [([24] * 13, 4), ([24] * 13, "sqrt"), ([20, 16, 24, 32, 16, 20], 2),
                                       ([16] * 3, 5)])
def test_checkpointed_adjoint_equals_full_storage(dims, ckpt):
    """sqrt(K) checkpointing (every s-th g_q kept, segments recomputed in the backward sweep and
    the adjoint pass) gives the same T(E), block gradients and self-energy gradients as keeping
    every g_q, for the T and density weights together, on uniform and ragged devices, with K not
    a multiple of s and s >= K; the slot needs less scratch."""
    from dpnegf_b200 import rgf_plan, workload
    dev = workload.random_device(0, 0, seed=41, block_dims=dims)
    B = 5
    seL = workload.random_self_energy(B, dims[0], seed=42).cuda()
    seR = workload.random_self_energy(B, dims[-1], seed=43).cuda()
    E = torch.linspace(-1.2, 1.3, B, dtype=torch.float64).to(torch.complex128).cuda()
    w = torch.linspace(0.5, 1.5, B, dtype=torch.float64)
    wd = torch.linspace(-0.3, 0.8, B, dtype=torch.float64)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)],
                             detect_zero_offdiag=False)
    kw = dict(eta=1e-5, outputs=(), adjoint_w=w, adjoint_w_dos=wd)
    full = rgf_plan.run(geom, [E], [seL], [seR], **kw)
    ck = rgf_plan.run(geom, [E], [seL], [seR], checkpoint=ckpt, **kw)
    assert torch.allclose(ck.trans, full.trans, rtol=1e-13, atol=0)
    # the per-slot gradient sums take the items in scheduling order, so the two runs agree to
    # rounding of those sums: compare each family in the max norm over its blocks
    for k in ("hd", "hu", "hl", "sd", "su", "sl"):
        scale = max(float(b.abs().max()) for b in full.grads[k])
        err = max(float((a - b).abs().max()) for a, b in zip(ck.grads[k], full.grads[k]))
        assert err <= 1e-11 * scale, (k, err, scale)
    for k in ("se_l", "se_r"):
        assert _rel(ck.grads[k], full.grads[k].cpu().numpy()) < 1e-11, k

