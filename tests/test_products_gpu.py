"""The product-chain kernels (negf_gamma_sum_run, the decimation kernel's coupling-product mode,
negf_lead_adjoint_run) against plain torch complex128 restatements of the same products."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
C128 = torch.complex128


def _rand(shape, gen, scale=1.0):
    return (torch.randn(*shape, generator=gen, dtype=torch.float64)
            + 1j * torch.randn(*shape, generator=gen, dtype=torch.float64)) * scale


def _rel(a, b):
    return float((a - b).abs().max() / b.abs().max().clamp_min(1e-300))


@pytest.mark.parametrize("B,n,m,k,c0", [(1, 7, 7, 3, 4), (6, 40, 40, 17, 23), (20, 130, 150, 64, 70),
                                        (3, 200, 200, 200, 0)])
def test_gamma_sum_matches_torch(B, n, m, k, c0):
    from dpnegf_b200.products import gamma_sum
    gen = torch.Generator().manual_seed(B * 1000 + n)
    G = _rand((B, n, m), gen).cuda()
    gam_full = _rand((B, k + 5, k + 5), gen).cuda()
    gam = gam_full[:, 5:, 5:]                      # a strided view, as the density's corner block
    w = torch.rand(B, generator=gen, dtype=torch.float64) - 0.3
    out = gamma_sum(G, gam, c0, w)
    Gc = G[:, :, c0:c0 + k]
    ref = (w.cuda().view(-1, 1, 1) * (Gc @ gam @ Gc.mH).real).sum(0)
    assert out.shape == (n, n) and out.dtype == torch.float64
    assert _rel(out, ref) < 1e-12
    assert torch.equal(out, gamma_sum(G, gam, c0, w))  # fixed summation order


def test_coupling_sigma_matches_torch():
    from dpnegf_b200.products import coupling_sigma
    gen = torch.Generator().manual_seed(7)
    B, N, nc, b = 5, 48, 20, 30
    g = _rand((B, N, N), gen).cuda()
    hdl, sdl = _rand((nc, b), gen).cuda(), _rand((nc, b), gen, 0.1).cuda()
    E = np.linspace(-1.0, 1.0, B) + 0.02j
    sig = coupling_sigma(g, hdl, sdl, E, E_ref=-0.5)
    Es = torch.as_tensor(E + (-0.5)).cuda().view(-1, 1, 1)
    ref = (Es * sdl - hdl) @ g[:, :b, :b] @ (Es * sdl.mH - hdl.mH)
    assert _rel(sig, ref) < 1e-13
    sig0 = coupling_sigma(g, hdl, None, E)           # no overlap coupling
    assert _rel(sig0, hdl @ g[:, :b, :b] @ hdl.mH) < 1e-13


def _lead_blocks(n, gen):
    """A random lead principal layer whose decimation converges at eta = 1e-3 (spread onsite
    levels, hopping 0.5, near-identity overlap)."""
    h = _rand((n, n), gen, 0.3)
    hL = (h + h.mH) / 2 + torch.diag(torch.linspace(-1, 1, n)).to(C128)
    s = _rand((n, n), gen, 0.02)
    sL = torch.eye(n, dtype=C128) + (s + s.mH) / 2
    return [x.cuda() for x in (hL, _rand((n, n), gen, 0.5), sL, _rand((n, n), gen, 0.02))]


def _torch_lead_adjoint(hL, hLL, sL, sLL, hDL, sDL, E, eta, gs, gsig, form):
    """The implicit-function adjoint by torch autograd and a torch doubling loop (test reference)."""
    E = torch.as_tensor(E).to(gs.device).view(-1, 1, 1)
    z = E + 1j * eta
    with torch.enable_grad():
        th = [t.detach().clone().requires_grad_(True) for t in (hL, hLL, sL, sLL)]
        tHL, tHLL, tSL, tSLL = th
        dl = [None if t is None else t.detach().clone().requires_grad_(True) for t in (hDL, sDL)]
        g = gs.detach().clone().requires_grad_(True)
        if form == 0:
            b = hDL.shape[-1]
            sdl = dl[1] if dl[1] is not None else torch.zeros_like(dl[0])
            sig = (E * sdl - dl[0]) @ g[:, :b, :b] @ (E * sdl.mH - dl[0].mH)
        elif form == 1:
            sig = torch.linalg.inv(g)
        else:
            sig = E * tSL - tHL - torch.linalg.inv(g)
        ins = [g] + th + [t for t in dl if t is not None]
        grads = torch.autograd.grad(sig, ins, grad_outputs=gsig, allow_unused=True)
        lam = grads[0]
        tau = z * tSLL.detach() - tHLL.detach()
        taup = z * tSLL.detach().mH - tHLL.detach().mH
        A = (gs @ tau).mH
        Bm = (taup @ gs).mH
        for _ in range(64):
            lam = lam + A @ lam @ Bm
            A = A @ A
            Bm = Bm @ Bm
            if float(A.abs().amax()) * float(Bm.abs().amax()) < 1e-32:
                break
        fval = torch.linalg.inv(z * tSL - tHL - (z * tSLL - tHLL) @ gs @ (z * tSLL.mH - tHLL.mH))
        gth = torch.autograd.grad(fval, th, grad_outputs=lam, allow_unused=True)
    out = [(grads[1 + i] if grads[1 + i] is not None else 0) + gth[i] for i in range(4)]
    k = 5
    for t in dl:
        if t is None:
            out.append(None)
        else:
            out.append(grads[k])
            k += 1
    return out


@pytest.mark.parametrize("form", [0, 1, 2])
def test_lead_adjoint_matches_torch_doubling(form):
    from dpnegf_b200 import surface_green as sg
    from dpnegf_b200.products import lead_adjoint
    gen = torch.Generator().manual_seed(11 + form)
    n, nc, b, B, eta, E_ref = 24, 10, 8, 6, 1e-3, 0.3
    hL, hLL, sL, sLL = _lead_blocks(n, gen)
    hDL, sDL = (_rand((nc, b), gen, 0.4).cuda(), _rand((nc, b), gen, 0.02).cuda()) if form == 0 else (None, None)
    E = np.linspace(-1.0, 1.5, B)
    arena = sg.LeadArena([sg.LeadBlocks(hL, hLL, sL, sLL, hDL, sDL)], device="cuda")
    res = sg.self_energies(arena, [0] * B, E, eta, E_ref=E_ref, want_gs=True)
    gs = torch.stack(res.gs)
    m = nc if form == 0 else n
    gsig = _rand((B, m, m), gen).cuda()
    got = lead_adjoint(hL, hLL, sL, sLL, hDL, sDL, E + E_ref, eta, gs, gsig, form)
    ref = _torch_lead_adjoint(hL, hLL, sL, sLL, hDL, sDL, E + E_ref, eta, gs, gsig, form)
    names = ["H", "H01", "S", "S01", "H_DL", "S_DL"]
    for name, x, y in zip(names, got, ref):
        if y is None:
            assert x is None, name
            continue
        assert _rel(x, y) < 1e-10, (name, _rel(x, y))
    again = lead_adjoint(hL, hLL, sL, sLL, hDL, sDL, E + E_ref, eta, gs, gsig, form)
    assert all(x is None or torch.equal(x, y) for x, y in zip(got, again))  # fixed summation order


def test_lead_adjoint_without_s_dl():
    """S_DL absent: zero overlap coupling, and no S_DL gradient is returned."""
    from dpnegf_b200 import surface_green as sg
    from dpnegf_b200.products import lead_adjoint
    gen = torch.Generator().manual_seed(5)
    n, nc, b, B, eta = 12, 6, 12, 3, 1e-3
    hL, hLL, sL, sLL = _lead_blocks(n, gen)
    hDL = _rand((nc, b), gen, 0.4).cuda()
    E = np.array([-0.4, 0.1, 0.7])
    arena = sg.LeadArena([sg.LeadBlocks(hL, hLL, sL, sLL, hDL, None)], device="cuda")
    gs = torch.stack(sg.self_energies(arena, [0] * B, E, eta, want_gs=True).gs)
    gsig = _rand((B, nc, nc), gen).cuda()
    got = lead_adjoint(hL, hLL, sL, sLL, hDL, None, E, eta, gs, gsig, 0)
    ref = _torch_lead_adjoint(hL, hLL, sL, sLL, hDL, None, E, eta, gs, gsig, 0)
    assert got[5] is None and ref[5] is None
    for x, y in zip(got[:5], ref[:5]):
        assert _rel(x, y) < 1e-10


def test_wrappers_on_a_side_stream_match_the_current_stream():
    """Called with a side stream, the wrappers stage, launch and read back on that stream: results
    equal the current-stream call bit for bit."""
    from dpnegf_b200 import surface_green as sg
    from dpnegf_b200.products import coupling_sigma, gamma_sum, lead_adjoint
    gen = torch.Generator().manual_seed(21)
    G, gam, w = _rand((9, 40, 40), gen).cuda(), _rand((9, 12, 12), gen).cuda(), torch.rand(9, dtype=torch.float64)
    hL, hLL, sL, sLL = _lead_blocks(16, gen)
    hDL = _rand((10, 16), gen, 0.4).cuda()
    E = np.linspace(-0.8, 0.8, 5)
    arena = sg.LeadArena([sg.LeadBlocks(hL, hLL, sL, sLL, hDL, None)], device="cuda")
    gsig = _rand((5, 10, 10), gen).cuda()

    def run(stream):
        def inputs_ready():  # the glue below runs on the current stream
            if stream is not None:
                stream.wait_stream(torch.cuda.current_stream())
        inputs_ready()
        out = [gamma_sum(G, gam, 28, w, stream=stream)]
        inputs_ready()
        res = sg.self_energies(arena, [0] * 5, E, 1e-3, want_gs=True, stream=stream)
        gs = torch.stack(res.gs)
        out += [gs, torch.stack(res.sigma)]
        inputs_ready()
        out.append(coupling_sigma(gs, hDL, None, E, stream=stream))
        inputs_ready()
        out += [x for x in lead_adjoint(hL, hLL, sL, sLL, hDL, None, E, 1e-3, gs, gsig, 0, stream=stream)
                if x is not None]
        return out

    ref = run(None)
    side = torch.cuda.Stream()
    got = run(side)
    side.synchronize()
    for x, y in zip(got, ref):
        assert torch.equal(x, y)
