"""Mixed-precision sweep (every block product on the tcgen05 3xTF32 GEMM,
FP32-accurate products; pivoting, panels and storage in FP64) against the FP64
oracle and the FP64 GPU path.

Accuracy stated per quantity, as checked here:
  T(E), refined (FP64-residual steps on G_{:,N}):     within 1e-6 absolute
                                                       (one step for the short chains here,
                                                       up to three at b=256, L=64)
  T(E) unrefined and DOS:                              within 1e-4 relative
  Green's-function blocks:                             within 1e-3 relative (max-norm)
  adjoint gradients:                                   within 1e-4 relative
(FP32-level products amplified by the conditioning of the sweep.)
"""
import numpy as np
import pytest
import torch

from oracle import rgf_oracle

pytestmark = pytest.mark.gpu
T_ATOL = 1e-6     # refined mixed T(E) vs FP64
FP32_RTOL = 1e-4  # unrefined mixed T, DOS, gradients vs FP64
BLOCK_RTOL = 1e-3  # mixed Green's-function blocks vs FP64 (max-norm)


def _case(dims, B, seed, emin=-2.0, emax=2.0):
    from dpnegf_b200 import workload
    dev = workload.random_device(0, 0, seed=seed, block_dims=dims)
    seL = workload.random_self_energy(B, dims[0], seed=seed + 1)
    seR = workload.random_self_energy(B, dims[-1], seed=seed + 2)
    E = torch.linspace(emin, emax, B, dtype=torch.float64).to(torch.complex128)
    return dev, seL, seR, E


def _oracle(dev, seL, seR, E, eta=1e-5):
    ref = rgf_oracle.rgf(E.numpy(), [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL.numpy(), seR.numpy(), eta=eta)
    T = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL.numpy()),
                                rgf_oracle.gamma_from_se(seR.numpy()))
    D = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], [x.numpy() for x in dev.sd],
                       [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl])
    return ref, T, D


def _run(dev, seL, seR, E, **kw):
    from dpnegf_b200 import rgf_plan
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    return rgf_plan.run(geom, [E.cuda()], [seL.cuda()], [seR.cuda()], eta=1e-5, **kw)


@pytest.mark.parametrize("dims,B", [([64] * 6, 6), ([200, 136, 200], 4), ([256] * 4, 3), ([40], 3),
                                     ([200, 48, 300], 2)])
def test_mixed_transmission_refined_within_1e6(dims, B):
    """Refined mixed T(E) within 1e-6 of the oracle; unrefined T and the DOS at
    FP32-product level.  Covers ragged tiles, K=1, and blocks above 128 (the
    inverse's tensor-core outer update) and above 256 (the NB=16 inverse)."""
    dev, seL, seR, E = _case(dims, B, seed=3 * len(dims) + dims[0])
    _, T, D = _oracle(dev, seL, seR, E)
    raw = _run(dev, seL, seR, E, outputs=(), trans=True, dos=True, precision="mixed")
    ref = _run(dev, seL, seR, E, outputs=(), trans=True, dos=True, precision="mixed", refine=True)
    t_raw, t_ref = raw.trans.cpu().numpy(), ref.trans.cpu().numpy()
    e_raw, e_ref = np.abs(t_raw - T).max(), np.abs(t_ref - T).max()
    print(f"mixed T error vs FP64 oracle: unrefined {e_raw:.2e}, refined {e_ref:.2e}")
    assert e_ref < T_ATOL, (e_raw, e_ref)
    scale = max(np.abs(T).max(), 1.0)
    assert np.abs(t_raw - T).max() < FP32_RTOL * scale
    np.testing.assert_allclose(raw.dos.cpu().numpy(), D, rtol=FP32_RTOL, atol=FP32_RTOL * np.abs(D).max())
    # the DOS is not refined: same value with and without refinement
    np.testing.assert_array_equal(ref.dos.cpu().numpy(), raw.dos.cpu().numpy())


def test_mixed_blocks_fp32_level():
    """Green's-function blocks of the mixed sweep within 1e-3 relative (max-norm) of the oracle."""
    dims = [72, 130, 72]
    dev, seL, seR, E = _case(dims, 3, seed=41)
    ref, _, _ = _oracle(dev, seL, seR, E)
    res = _run(dev, seL, seR, E, outputs=("g_trans", "grd", "grl", "gru"), precision="mixed")
    blk = res.blocks[0]
    for tag in ("grd", "grl", "gru"):
        for q, (g, w) in enumerate(zip(blk[tag], ref[tag])):
            g = g.cpu().numpy()
            err = np.abs(g - w).max() / np.abs(w).max()
            print(f"mixed {tag}[{q}] relative error {err:.2e}")
            assert err < BLOCK_RTOL, (tag, q, err)
    g = blk["g_trans"].cpu().numpy()
    assert np.abs(g - ref["g_trans"]).max() / np.abs(ref["g_trans"]).max() < BLOCK_RTOL


def test_mixed_refined_metric_size():
    """b=256, L=64 (the throughput workload's device and self-energies): refined
    mixed T(E) within 1e-6 of the FP64 GPU sweep, which the oracle tests pin.
    The contraction of one step worsens with the chain length; at 64 blocks one
    step leaves ~2e-4, two ~1e-6, three ~1e-8."""
    from dpnegf_b200 import rgf_plan, workload
    b, L, B = 256, 64, 8
    dev = workload.random_device(b, L, seed=0)
    seL = workload.random_self_energy(B, b, seed=1).cuda()
    seR = workload.random_self_energy(B, b, seed=2).cuda()
    E = workload.energy_grid(B).to(torch.complex128).cuda()
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    t64 = rgf_plan.run(geom, [E], [seL], [seR], eta=1e-5, outputs=(), trans=True).trans.cpu().numpy()
    tmx = rgf_plan.run(geom, [E], [seL], [seR], eta=1e-5, outputs=(), trans=True, precision="mixed",
                       refine=True, refine_steps=3).trans.cpu().numpy()
    print(f"b=256 L=64 refined mixed T error vs FP64: {np.abs(tmx - t64).max():.2e}")
    assert np.abs(tmx - t64).max() < T_ATOL, np.abs(tmx - t64).max()


def test_mixed_adjoint_close_to_fp64():
    """Mixed adjoint gradients within 1e-4 relative of the FP64 adjoint."""
    from dpnegf_b200 import adjoint
    dims = [48, 64, 48]
    dev, seL, seR, E = _case(dims, 4, seed=13)
    grads = {}
    for prec in ("fp64", "mixed"):
        hd = [x.cuda().requires_grad_() for x in dev.hd]
        hu = [x.cuda().requires_grad_() for x in dev.hu]
        sL = seL.cuda().requires_grad_()
        T = adjoint.transmission(hd, hu, [x.cuda() for x in dev.hl], [x.cuda() for x in dev.sd],
                                 [x.cuda() for x in dev.su], [x.cuda() for x in dev.sl], E.cuda(), sL,
                                 seR.cuda(), eta=1e-5, precision=prec)
        T.sum().backward()
        grads[prec] = [x.grad.cpu().numpy() for x in hd + hu] + [sL.grad.cpu().numpy()]
    for a, b in zip(grads["mixed"], grads["fp64"]):
        err = np.abs(a - b).max() / np.abs(b).max()
        print(f"mixed adjoint gradient relative error {err:.2e}")
        assert err < FP32_RTOL


@pytest.mark.parametrize("inv_ob", [32, 64, 128, 256])
def test_mixed_outer_block_widths(inv_ob):
    """The mixed sweep at every outer block width: refined T within 1e-6 of the oracle."""
    dims = [200, 136, 200]
    dev, seL, seR, E = _case(dims, 3, seed=51)
    _, T, _ = _oracle(dev, seL, seR, E)
    r = _run(dev, seL, seR, E, outputs=(), trans=True, precision="mixed", refine=True, inv_ob=inv_ob, inverse="gj")
    assert np.abs(r.trans.cpu().numpy() - T).max() < T_ATOL


@pytest.mark.parametrize("inverse", ["block", "gj"])
def test_mixed_with_each_inverse_scheme(inverse):
    """Both Schur-complement inverses in the mixed sweep (the autotuner picks the block scheme
    there from n = 384): refined T within 1e-6, unrefined T and DOS at FP32-product level."""
    dims, B = [384, 128, 384], 2
    dev, seL, seR, E = _case(dims, B, seed=77)
    _, T, D = _oracle(dev, seL, seR, E)
    raw = _run(dev, seL, seR, E, outputs=(), trans=True, dos=True, precision="mixed", inverse=inverse)
    ref = _run(dev, seL, seR, E, outputs=(), trans=True, precision="mixed", refine=True, refine_steps=3,
               inverse=inverse)
    assert np.abs(ref.trans.cpu().numpy() - T).max() < T_ATOL
    scale = max(np.abs(T).max(), 1.0)
    assert np.abs(raw.trans.cpu().numpy() - T).max() < FP32_RTOL * scale
    np.testing.assert_allclose(raw.dos.cpu().numpy(), D, rtol=FP32_RTOL, atol=FP32_RTOL * np.abs(D).max())
