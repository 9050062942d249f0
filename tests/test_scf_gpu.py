"""SCF loop around the captured sweep (the damped onsite-shift loop of the
b=512 SCF benchmark case, scaled down): 10 iterations with the iteration body
replayed as a CUDA graph equal the eager loop bit for bit, and the FP64 loop
matches an oracle SCF loop to 1e-9 relative; the mixed sweep to 1e-4."""
import numpy as np
import pytest
import torch

from oracle import rgf_oracle

pytestmark = pytest.mark.gpu


def _setup():
    from dpnegf_b200 import workload
    from dpnegf_b200.ozaki_res_cal import ozaki_residues
    from dpnegf_b200.scf import ozaki_weights
    dims = [24, 40, 24]
    dev = workload.random_device(0, 0, seed=17, block_dims=dims)
    kBT, mu_L, vL, vR = 0.025, 0.05, 0.1, -0.1
    fL = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vL)) / kBT))
    fR = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vR)) / kBT))
    poles, res = ozaki_residues(6)
    z, c, w = ozaki_weights(poles.numpy(), res.numpy(), 1e6, 6, kBT, mu_L, vL=vL, vR=vR, fermi_L=fL, fermi_R=fR)
    seL = workload.random_self_energy(len(z), dims[0], seed=18)
    seR = workload.random_self_energy(len(z), dims[-1], seed=19)
    return dev, z, c, w, seL, seR


def _loop(precision, use_graph, iters=10):
    from dpnegf_b200 import rgf_plan
    from dpnegf_b200.scf import ScfLoop
    dev, z, c, w, seL, seR = _setup()
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    loop = ScfLoop(geom, seL.cuda(), seR.cuda(), z, c, w, alpha=0.5, mix=0.3, eta=1e-5, precision=precision,
                   use_graph=use_graph)
    V, n = loop.run(iters)
    loop.restore()
    return V.cpu().numpy(), n.cpu().numpy(), loop


def _oracle_loop(iters=10):
    dev, z, c, w, seL, seR = _setup()
    hd0 = [x.numpy() for x in dev.hd]
    dims = [h.shape[0] for h in hd0]
    gam = rgf_oracle.gamma_from_se(seR.numpy())

    def density(V, eq_only=False):
        off = np.cumsum([0] + dims)
        hd = [hd0[q] + np.diag(V[off[q]:off[q + 1]]) for q in range(len(dims))]
        ref = rgf_oracle.rgf(z, [x.numpy() for x in dev.hl], hd, [x.numpy() for x in dev.hu],
                             [x.numpy() for x in dev.sd], [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                             seL.numpy(), seR.numpy(), eta=1e-5, need_gr_lc=True)
        g = np.concatenate([np.diagonal(b, axis1=1, axis2=2) for b in ref["grd"]], axis=1)
        a = np.concatenate([np.einsum("eij,ejk,eik->ei", x, gam, x.conj()).real for x in ref["gr_lc"]], axis=1)
        n_eq = (c.reshape(-1, 1) * g).real.sum(0)
        return n_eq if eq_only else n_eq + (w.reshape(-1, 1) * a).sum(0)

    V = np.zeros(sum(dims))
    n0 = density(V, eq_only=True)
    for _ in range(iters):
        n = density(V)
        V = V + 0.3 * (0.5 * (n - n0) - V)
    return V, n


def test_scf_graph_replay_equals_eager_and_oracle():
    Vg, ng, loop = _loop("fp64", True)
    assert loop.graph is not None and loop.iterations == 10
    Ve, ne, _ = _loop("fp64", False)
    np.testing.assert_array_equal(Vg, Ve)
    np.testing.assert_array_equal(ng, ne)
    Vo, no = _oracle_loop()
    assert np.abs(Vo).max() > 1e-6  # the bias moves the potential
    assert np.abs(Vg - Vo).max() <= 1e-9 * np.abs(Vo).max()
    assert np.abs(ng - no).max() <= 1e-9 * np.abs(no).max()


def test_scf_mixed_close_to_fp64():
    V64, n64, _ = _loop("fp64", True)
    Vm, nm, _ = _loop("mixed", True)
    assert np.abs(nm - n64).max() <= 1e-4 * np.abs(n64).max()
    assert np.abs(Vm - V64).max() <= 1e-4 * max(np.abs(V64).max(), 1e-3)


def _setup_k(nk=2):
    """The same orbitals at ``nk`` k-points: distinct H(k), S(k) realisations and self-energies."""
    from dpnegf_b200 import workload
    dev, z, c, w, _, _ = _setup()
    dims = dev.block_dims
    devs = [workload.random_device(0, 0, seed=40 + k, block_dims=dims) for k in range(nk)]
    seL = [workload.random_self_energy(len(z), dims[0], seed=50 + k) for k in range(nk)]
    seR = [workload.random_self_energy(len(z), dims[-1], seed=60 + k) for k in range(nk)]
    return devs, z, c, w, seL, seR


def _loop_k(use_graph, wk, iters=10):
    from dpnegf_b200 import rgf_plan
    from dpnegf_b200.scf import ScfLoop
    devs, z, c, w, seL, seR = _setup_k(len(wk))
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl) for d in devs])
    loop = ScfLoop(geom, [x.cuda() for x in seL], [x.cuda() for x in seR], z, c, w, alpha=0.5, mix=0.3, eta=1e-5,
                   use_graph=use_graph, wk=wk)
    V, n = loop.run(iters)
    loop.restore()
    return V.cpu().numpy(), n.cpu().numpy()


def _oracle_loop_k(wk, iters=10):
    devs, z, c, w, seL, seR = _setup_k(len(wk))
    dims = devs[0].block_dims
    off = np.cumsum([0] + dims)

    def density(V, eq_only=False):
        tot = 0.0
        for k, dev in enumerate(devs):
            hd = [dev.hd[q].numpy() + np.diag(V[off[q]:off[q + 1]]) for q in range(len(dims))]
            ref = rgf_oracle.rgf(z, [x.numpy() for x in dev.hl], hd, [x.numpy() for x in dev.hu],
                                 [x.numpy() for x in dev.sd], [x.numpy() for x in dev.su],
                                 [x.numpy() for x in dev.sl], seL[k].numpy(), seR[k].numpy(), eta=1e-5,
                                 need_gr_lc=True)
            gam = rgf_oracle.gamma_from_se(seR[k].numpy())
            g = np.concatenate([np.diagonal(b, axis1=1, axis2=2) for b in ref["grd"]], axis=1)
            a = np.concatenate([np.einsum("eij,ejk,eik->ei", x, gam, x.conj()).real for x in ref["gr_lc"]], axis=1)
            n = (c.reshape(-1, 1) * g).real.sum(0)
            tot = tot + wk[k] * (n if eq_only else n + (w.reshape(-1, 1) * a).sum(0))
        return tot

    V = np.zeros(sum(dims))
    n0 = density(V, eq_only=True)
    for _ in range(iters):
        n = density(V)
        V = V + 0.3 * (0.5 * (n - n0) - V)
    return V, n


def test_scf_over_k_points_matches_oracle():
    """Two k-points with weights 0.25 / 0.75 in one launch per iteration: graph replay equals the
    eager loop bit for bit, and both match the oracle's k-summed SCF loop to 1e-9 relative."""
    wk = [0.25, 0.75]
    Vg, ng = _loop_k(True, wk)
    Ve, ne = _loop_k(False, wk)
    np.testing.assert_array_equal(Vg, Ve)
    np.testing.assert_array_equal(ng, ne)
    Vo, no = _oracle_loop_k(wk)
    assert np.abs(Vo).max() > 1e-6
    assert np.abs(Vg - Vo).max() <= 1e-9 * np.abs(Vo).max()
    assert np.abs(ng - no).max() <= 1e-9 * np.abs(no).max()
