"""RGF parity on the GPU: the CUDA sweep against the reference fixtures and
the numpy oracle.  Tolerance: FP64 path within 1e-10 relative (max-norm of
each block), as required for the plain path."""
import numpy as np
import pytest
import torch

from oracle import lead_oracle, rgf_oracle
from tests.goldens import Golden, rgf_cases

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def _cu(xs):
    return [torch.as_tensor(x).cuda() for x in xs]


def _assert_block_close(got, want, tag, rtol=RTOL):
    got = got.detach().cpu().numpy() if torch.is_tensor(got) else np.asarray(got)
    want = np.asarray(want)
    assert got.shape == want.shape, (tag, got.shape, want.shape)
    scale = max(np.abs(want).max(), 1e-300)
    err = np.abs(got - want).max() / scale
    assert err < rtol, f"{tag}: relative max error {err:.3e}"


def _compare(ans, ref_get, scalar=False):
    for i, tag in enumerate(rgf_oracle.TAGS):
        want = ref_get(tag)
        got = ans[i]
        if want is None:
            continue
        assert got is not None, tag
        if isinstance(want, list):
            assert len(got) == len(want), tag
            for q, (g, w) in enumerate(zip(got, want)):
                _assert_block_close(g, w, f"{tag}[{q}]")
        else:
            _assert_block_close(got, want, tag)


@pytest.mark.parametrize("case", rgf_cases())
def test_rgf_matches_reference_fixture(case):
    from dpnegf_b200.recursive_green_cal import recursive_gf
    g = Golden(case)
    scalar = bool(g["scalar"])
    E = torch.as_tensor(g["energy"]).cuda()
    seL, seR = torch.as_tensor(g["left_se"]).cuda(), torch.as_tensor(g["right_se"]).cuda()
    lesser, greater = g.has("s_in"), g.has("s_out")
    kw = dict(eta=float(g["eta"]), E_ref=float(g["E_ref"]), need_gr_lc=g.has("out/gr_lc"))
    if g.has("seP"):  # tensors per block, plain numbers (the reference's 0 placeholders) as numbers
        kw["seP"] = [torch.as_tensor(x).cuda() if np.ndim(x) else complex(x) for x in g["seP"]]
    if scalar:
        ans = recursive_gf(E[0], _cu(g["hl"]), _cu(g["hd"]), _cu(g["hu"]), _cu(g["sd"]), _cu(g["su"]),
                           _cu(g["sl"]), seL[0], seR[0],
                           s_in=[torch.as_tensor(s[0]).cuda() for s in g["s_in"]] if lesser else 0,
                           s_out=[torch.as_tensor(s[0]).cuda() for s in g["s_out"]] if greater else 0,
                           need_lesser=lesser, need_greater=greater, **kw)
    else:
        ans = recursive_gf(E, _cu(g["hl"]), _cu(g["hd"]), _cu(g["hu"]), _cu(g["sd"]), _cu(g["su"]),
                           _cu(g["sl"]), seL, seR, s_in=_cu(g["s_in"]) if lesser else 0,
                           s_out=_cu(g["s_out"]) if greater else 0,
                           need_lesser=lesser, need_greater=greater, **kw)
    _compare(ans, lambda t: g.get("out/" + t))


def _oracle_case(dims, B, seed, lesser=False, eta=1e-5):
    from dpnegf_b200 import workload
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    seL = workload.random_self_energy(B, dims[0], seed=seed + 1)
    seR = workload.random_self_energy(B, dims[-1], seed=seed + 2)
    E = torch.linspace(-2.0, 2.0, B, dtype=torch.float64).to(torch.complex128)
    s_in = None
    if lesser:
        f = np.linspace(0.1, 0.9, B)
        s_in = rgf_oracle.s_in_from_se(seL.numpy(), seR.numpy(), f, 1 - f, dims)
    return dev, seL, seR, E, s_in


@pytest.mark.parametrize("dims,B", [([64] * 4, 3), ([70, 33, 128, 65], 2), ([256] * 3, 2),
                                     ([300, 280], 1), ([17], 3), ([96, 96], 5), ([240, 300], 1)])
def test_rgf_matches_oracle_sizes(dims, B):
    """Ragged tiles (n not a multiple of 64), the NB=16 inverse (n>256), K=1, K=2, and a
    device mixing both inverse layouts (the shared-memory size covers the larger)."""
    from dpnegf_b200.recursive_green_cal import recursive_gf
    dev, seL, seR, E, _ = _oracle_case(dims, B, seed=len(dims) * 7 + dims[0])
    ans = recursive_gf(E.cuda(), _cu(dev.hl), _cu(dev.hd), _cu(dev.hu), _cu(dev.sd), _cu(dev.su),
                       _cu(dev.sl), seL.cuda(), seR.cuda(), eta=1e-5, need_gr_lc=True)
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5, need_gr_lc=True)
    _compare(ans, lambda t: ref.get(t))


def test_rgf_lesser_matches_oracle():
    from dpnegf_b200.recursive_green_cal import recursive_gf
    dims = [40, 72, 40]
    dev, seL, seR, E, s_in = _oracle_case(dims, 3, seed=11, lesser=True)
    ans = recursive_gf(E.cuda(), _cu(dev.hl), _cu(dev.hd), _cu(dev.hu), _cu(dev.sd), _cu(dev.su),
                       _cu(dev.sl), seL.cuda(), seR.cuda(), eta=1e-5, need_lesser=True,
                       s_in=[torch.as_tensor(s).cuda() for s in s_in])
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5, s_in=s_in, need_lesser=True)
    _compare(ans, lambda t: ref.get(t))


@pytest.mark.parametrize("dims,lesser", [([40, 72, 40], False), ([40, 72, 40], True), ([128] * 3, True),
                                          ([33], False)])
def test_rgf_greater_matches_oracle(dims, lesser):
    """G^> sweep (elementwise-conjugate recurrences of recursive_green_cal.py:143-161), alone and
    next to the lesser sweep in the same launch; Sigma^out = Gamma (1 - f)."""
    from dpnegf_b200.recursive_green_cal import recursive_gf
    B = 3
    dev, seL, seR, E, s_in = _oracle_case(dims, B, seed=13, lesser=True)
    f = np.linspace(0.1, 0.9, B)
    s_out = rgf_oracle.s_in_from_se(seL.numpy(), seR.numpy(), 1 - f, f, dims)
    ans = recursive_gf(E.cuda(), _cu(dev.hl), _cu(dev.hd), _cu(dev.hu), _cu(dev.sd), _cu(dev.su),
                       _cu(dev.sl), seL.cuda(), seR.cuda(), eta=1e-5, need_lesser=lesser,
                       s_in=[torch.as_tensor(s).cuda() for s in s_in] if lesser else 0,
                       need_greater=True, s_out=[torch.as_tensor(s).cuda() for s in s_out])
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5, s_in=s_in if lesser else None, s_out=s_out,
                         need_lesser=lesser, need_greater=True)
    for t in ("gpd", "gpl", "gpu", "gip_left"):
        assert ref.get(t) is not None
    _compare(ans, lambda t: ref.get(t))


@pytest.mark.parametrize("dims", [[8, 6, 8], [128] * 5, [256] * 4])
def test_fused_transmission_and_dos(dims):
    """T(E) and per-orbital DOS reduced inside the sweep vs the oracle."""
    from dpnegf_b200 import rgf_plan
    B = 4
    dev, seL, seR, E, _ = _oracle_case(dims, B, seed=5)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    res = rgf_plan.run(geom, [E.cuda()], [seL.cuda()], [seR.cuda()], eta=1e-5, outputs=(),
                       trans=True, orb_dos=True, dos=True)
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5)
    T = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL.numpy()),
                                rgf_oracle.gamma_from_se(seR.numpy()))
    dos = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl])
    got_T = res.trans.cpu().numpy()
    got_dos = 2.0 * res.orb_dos.cpu().numpy().reshape(B, -1).sum(-1)
    np.testing.assert_allclose(got_T, T, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(got_dos, dos, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(res.dos.cpu().numpy(), dos, rtol=1e-10, atol=1e-12)


def test_transport_api_host_tensors():
    """Public fused API with host inputs returns host T/DOS equal to the oracle."""
    from dpnegf_b200 import transport
    dims = [48, 48, 48]
    B = 5
    dev, seL, seR, E, _ = _oracle_case(dims, B, seed=21)
    T, D, orb = transport.transmission_dos(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl, E, seL, seR,
                                           eta=1e-5, E_ref=0.02, orbital_dos=True)
    assert T.device.type == "cpu" and D.device.type == "cpu" and orb.shape == (B, sum(dims))
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5, E_ref=0.02)
    Tr = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL.numpy()),
                                 rgf_oracle.gamma_from_se(seR.numpy()))
    Dr = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], [x.numpy() for x in dev.sd],
                        [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl])
    np.testing.assert_allclose(T.numpy(), Tr, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(D.numpy(), Dr, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(2 * orb.numpy().sum(-1), Dr, rtol=1e-10, atol=1e-12)


def test_chain_transmission_is_one_in_band():
    """1-D chain, t=-1, leads from the oracle decimation: T(E)=1 for |E|<1.9."""
    from dpnegf_b200 import rgf_plan, workload
    chain = workload.chain_device(L=10)
    E = np.linspace(-3, 3, 61)
    seL, seR = [], []
    for e in E:
        for side, acc in ((chain.lead_L, seL), (chain.lead_R, seR)):
            s, _, st, _ = lead_oracle.self_energy(side.hL.numpy(), side.hLL.numpy(), side.sL.numpy(),
                                                  side.sLL.numpy(), e, side.hDL.numpy(), side.sDL.numpy(),
                                                  etaLead=1e-6)
            acc.append(s)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(chain.hd, chain.hu, chain.hl, chain.sd, chain.su, chain.sl)])
    res = rgf_plan.run(geom, [torch.as_tensor(E).to(torch.complex128).cuda()],
                       [torch.as_tensor(np.stack(seL)).cuda()], [torch.as_tensor(np.stack(seR)).cuda()],
                       eta=1e-6, outputs=(), trans=True, orb_dos=True)
    T = res.trans.cpu().numpy()
    inband = np.abs(E) < 1.9
    assert np.all(np.abs(T[inband] - 1.0) < 1e-4), T[inband]
    assert np.all(T[np.abs(E) > 2.1] < 1e-8)


@pytest.mark.parametrize("inv_ob", [32, 64, 128, 256, 512])
def test_inverse_outer_block_widths_agree(inv_ob):
    """Every Gauss-Jordan outer block width (the autotuned knob) gives the oracle's
    blocks to 1e-10, on sizes that use both panel layouts."""
    from dpnegf_b200 import rgf_plan
    dims = [200, 160, 300]
    dev, seL, seR, E, _ = _oracle_case(dims, 2, seed=29)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    res = rgf_plan.run(geom, [E.cuda()], [seL.cuda()], [seR.cuda()], eta=1e-5, outputs=("grd", "g_trans"),
                       inv_ob=inv_ob, inverse="gj")
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5)
    for q, w in enumerate(ref["grd"]):
        _assert_block_close(res.blocks[0]["grd"][q], w, f"grd[{q}] ob={inv_ob}")
    _assert_block_close(res.blocks[0]["g_trans"], ref["g_trans"], f"g_trans ob={inv_ob}")


@pytest.mark.parametrize("dims,B", [([64] * 4, 3), ([70, 33, 128, 65], 2), ([256] * 3, 2), ([300, 280], 1),
                                     ([17], 3), ([512, 96], 1)])
def test_block_inverse_matches_oracle(dims, B):
    """inverse="block" (recursive 2x2 blocks, pivoted 64-wide leaves) gives the oracle's blocks
    to 1e-10: ragged splits, a single leaf, three recursion levels (n = 512)."""
    from dpnegf_b200 import rgf_plan
    dev, seL, seR, E, _ = _oracle_case(dims, B, seed=len(dims) * 5 + dims[0])
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    res = rgf_plan.run(geom, [E.cuda()], [seL.cuda()], [seR.cuda()], eta=1e-5,
                       outputs=("g_trans", "grd", "grl", "gru"), trans=True, dos=True, inverse="block")
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=1e-5)
    blocks = res.blocks[0]
    for tag in ("g_trans", "grd", "grl", "gru"):
        want = ref[tag]
        if isinstance(want, list):
            for q, (g, w) in enumerate(zip(blocks[tag], want)):
                _assert_block_close(g, w, f"{tag}[{q}]")
        else:
            _assert_block_close(blocks[tag], want, tag)
    sd = [x.numpy() for x in dev.sd]
    T_ref = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL.numpy()),
                                    rgf_oracle.gamma_from_se(seR.numpy()))
    D_ref = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], sd, [x.numpy() for x in dev.su],
                           [x.numpy() for x in dev.sl])
    np.testing.assert_allclose(res.trans.cpu().numpy(), T_ref, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(res.dos.cpu().numpy(), D_ref, rtol=1e-10, atol=1e-12)


def test_empty_energy_batch_gives_empty_blocks():
    """An empty energy batch returns empty [0, n, m] blocks (the shapes the reference's
    recursive_gf returns for a [0] energy tensor) and launches nothing."""
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.recursive_green_cal import recursive_gf
    dims = [4, 5, 4]
    dev = workload.random_device(0, 0, seed=1, block_dims=dims)
    E = torch.zeros(0, dtype=torch.complex128, device="cuda")
    se = torch.zeros(0, 4, 4, dtype=torch.complex128, device="cuda")
    ans = recursive_gf(E, _cu(dev.hl), _cu(dev.hd), _cu(dev.hu), _cu(dev.sd), _cu(dev.su), _cu(dev.sl), se, se,
                       eta=1e-5, need_gr_lc=True)
    assert tuple(ans[0].shape) == (0, 4, 4)
    assert [tuple(x.shape) for x in ans[1]] == [(0, 4, 4), (0, 5, 4), (0, 4, 4)]
    assert [tuple(x.shape) for x in ans[2]] == [(0, 4, 4), (0, 5, 5), (0, 4, 4)]
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    res = rgf_plan.run(geom, [E], [se], [se], eta=1e-5, outputs=(), trans=True, dos=True)
    assert res.trans.numel() == 0 and res.dos.numel() == 0


def test_lesser_input_of_wrong_shape_is_refused():
    """An s_in block whose shape is not [B, n_q, n_q] raises ValueError before any launch (a
    wrong size would shift every later block of the packed lesser inputs)."""
    from dpnegf_b200 import rgf_plan, workload
    dims = [4, 5, 4]
    dev = workload.random_device(0, 0, seed=2, block_dims=dims)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    E = torch.linspace(-0.5, 0.5, 3, dtype=torch.float64).to(torch.complex128).cuda()
    se = workload.random_self_energy(3, 4, seed=3).cuda()
    s_in = [torch.zeros(3, n, n, dtype=torch.complex128, device="cuda") for n in dims]
    s_in[1] = torch.zeros(3, 4, 4, dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError, match=r"s_in\[1\] has shape"):
        rgf_plan.run(geom, [E], [se], [se], eta=1e-5, outputs=("gnd",), s_in=[s_in])
