"""The block inverse's safety net.  The recursive 2x2 block inverse pivots only
inside 64-wide leaves, so it needs nonsingular leading sub-blocks; eta > 0
guarantees them for physical inputs, eta = 0 does not.  The device below has
eta = 0 and a leading 64 x 64 sub-block of its first Schur complement that is
exactly singular while the whole block is not: the unpivoted block formula
fails on it (CPU check), and the sweep's residual probe must send the item
back to the pivoted Gauss-Jordan inverse (GPU check against the oracle)."""
import numpy as np
import pytest
import torch

from oracle import rgf_oracle

E0 = 0.3


def _device():
    rng = np.random.default_rng(5)
    c = lambda shape, s: rng.normal(size=shape) * s + 1j * rng.normal(size=shape) * s
    herm = lambda x: (x + x.conj().T) / 2
    n0, n1 = 128, 32
    H0 = herm(c((n0, n0), 0.3))
    q, _ = np.linalg.qr(c((56, 56), 1.0))
    lam = np.concatenate([[E0], rng.uniform(-2, 2, 55)])
    H0[8:64, 8:64] = (q * lam) @ q.conj().T          # eigenvalue E0 on orbitals 8..63
    H0[0:8, 8:64] = 0.0
    H0[8:64, 0:8] = 0.0                              # rows 0..63 split into an 8- and a 56-block
    H1 = herm(c((n1, n1), 0.3))
    hu = c((n0, n1), 0.4)
    hd = [H0, H1]
    sd = [np.eye(n0, dtype=complex), np.eye(n1, dtype=complex)]
    a, b = c((8, 8), 0.3), c((n1, n1), 0.3)
    seL = herm(a) - 1j * (a @ a.conj().T + 0.1 * np.eye(8))
    seR = herm(b) - 1j * (b @ b.conj().T + 0.1 * np.eye(n1))
    return hd, [hu], [hu.conj().T], sd, [np.zeros((n0, n1), complex)], [np.zeros((n1, n0), complex)], seL, seR


def _block_inverse_no_fallback(A, leaf=64):
    n = A.shape[0]
    if n <= leaf:
        return np.linalg.inv(A)
    h = n // 2
    X = _block_inverse_no_fallback(A[:h, :h], leaf)
    U = A[h:, :h] @ X
    Y = _block_inverse_no_fallback(A[h:, h:] - U @ A[:h, h:], leaf)
    TY = X @ A[:h, h:] @ Y
    return np.block([[X + TY @ U, -TY], [-Y @ U, Y]])


def test_unpivoted_block_formula_fails_on_this_device():
    hd, hu, hl, sd, su, sl, seL, seR = _device()
    A0 = E0 * sd[0] - hd[0]
    A0[:8, :8] -= seL
    G_blk = _block_inverse_no_fallback(A0)
    G_ref = np.linalg.inv(A0)
    assert np.linalg.norm(A0 @ G_ref - np.eye(128)) < 1e-10
    assert not (np.linalg.norm(A0 @ G_blk - np.eye(128)) < 1e-6)  # the fallback is what saves the GPU run


@pytest.mark.gpu
@pytest.mark.parametrize("inverse", ["block", "gj"])
def test_sweep_falls_back_to_pivoting(inverse):
    from dpnegf_b200 import rgf_plan
    hd, hu, hl, sd, su, sl, seL, seR = _device()
    t = lambda xs: [torch.as_tensor(x) for x in xs]
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(t(hd), t(hu), t(hl), t(sd), t(su), t(sl))])
    E = torch.tensor([E0, E0 + 0.2], dtype=torch.complex128).cuda()
    sL = torch.as_tensor(seL).expand(2, -1, -1).contiguous().cuda()
    sR = torch.as_tensor(seR).expand(2, -1, -1).contiguous().cuda()
    res = rgf_plan.run(geom, [E], [sL], [sR], eta=0.0, outputs=("g_trans", "grd"), trans=True,
                       inverse=inverse)
    ref = rgf_oracle.rgf(E.cpu().numpy(), hl, hd, hu, sd, su, sl, sL.cpu().numpy(), sR.cpu().numpy(), eta=0.0)
    for q, w in enumerate(ref["grd"]):
        got = res.blocks[0]["grd"][q].cpu().numpy()
        assert np.abs(got - w).max() / np.abs(w).max() < 1e-10, (q, inverse)
    g = res.blocks[0]["g_trans"].cpu().numpy()
    assert np.abs(g - ref["g_trans"]).max() / np.abs(ref["g_trans"]).max() < 1e-10
