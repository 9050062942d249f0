"""Multi-rank host logic on CPU (gloo, world size 2): the item sharding covers
every item exactly once with balanced work, and the sharded run with its one
all-reduce gives every rank the single-process result.  The compute function
is the oracle's T(E) on a small ragged device (the GPU launch in production)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def test_shard_partitions_and_balances():
    from dpnegf_b200.multi import shard
    rng = np.random.default_rng(3)
    costs = rng.integers(1, 200, size=37).astype(float) ** 3
    for world in (1, 2, 3, 8):
        parts = [shard(costs, world, r) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max() + 1e-9
    with pytest.raises(ValueError):
        shard(costs, 2, 2)


def _case():
    from dpnegf_b200 import workload
    dims = [12, 20, 12]
    dev = workload.random_device(0, 0, seed=5, block_dims=dims)
    B = 9
    seL = workload.random_self_energy(B, dims[0], seed=6).numpy()
    seR = workload.random_self_energy(B, dims[-1], seed=7).numpy()
    E = np.linspace(-1.5, 1.5, B).astype(np.complex128)
    return dev, seL, seR, E


def _oracle_T(idx):
    from oracle import rgf_oracle
    dev, seL, seR, E = _case()
    ref = rgf_oracle.rgf(E[idx], [x.numpy() for x in dev.hl], [x.numpy() for x in dev.hd],
                         [x.numpy() for x in dev.hu], [x.numpy() for x in dev.sd],
                         [x.numpy() for x in dev.su], [x.numpy() for x in dev.sl],
                         seL[idx], seR[idx], eta=1e-5)
    T = rgf_oracle.transmission(ref["g_trans"], rgf_oracle.gamma_from_se(seL[idx]),
                                rgf_oracle.gamma_from_se(seR[idx]))
    return torch.as_tensor(T)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    from dpnegf_b200.multi import run_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        _, _, _, E = _case()
        costs = np.ones(len(E)) + np.arange(len(E)) % 3  # uneven item costs
        out = run_sharded(costs, _oracle_T, (len(E),))
        q.put((rank, out.numpy()))
    finally:
        dist.destroy_process_group()


def test_sharded_run_matches_single_process_gloo():
    from dpnegf_b200.multi import run_sharded
    _, _, _, E = _case()
    costs = np.ones(len(E)) + np.arange(len(E)) % 3
    single = run_sharded(costs, _oracle_T, (len(E),)).numpy()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        np.testing.assert_allclose(got[r], single, rtol=0, atol=1e-14)


class _DiagonalPlan:
    """Stands in for the deferred sweep on the CPU: a device without couplings, whose
    G_ii(z) = 1 / (z + i 1e-3 - H_ii) is read from the arena's current onsite values (so the
    potential feeds back) and A_R,ii = gamma_i |G_ii|^2."""

    def __init__(self, geom, z, gamma):
        from types import SimpleNamespace
        idx = []
        for d in geom.devs:
            row = []
            for q in range(int(d["blk0"]), int(d["blk0"]) + int(d["n_blocks"])):
                n = int(geom.blocks[q]["n"])
                row.append(int(geom.blocks[q]["hd"]) + np.arange(n) * (n + 1))
            idx.append(np.concatenate(row))
        self.idx = torch.as_tensor(np.array(idx))
        self.geom = geom
        self.z = torch.as_tensor(np.asarray(z), dtype=torch.complex128).reshape(1, -1, 1)
        self.gamma = torch.as_tensor(gamma, dtype=torch.float64)
        size = self.idx.numel() * self.z.shape[1]
        self.result = SimpleNamespace(orb_g=torch.zeros(size, dtype=torch.complex128),
                                      orb_ar=torch.zeros(size, dtype=torch.float64))

    def launch(self, stream=None):
        g = 1.0 / (self.z + 1e-3j - self.geom.hs[self.idx].unsqueeze(1))
        self.result.orb_g.copy_(g.reshape(-1))
        self.result.orb_ar.copy_((self.gamma * g.abs() ** 2).reshape(-1))

    def check(self):
        pass


def _scf_case():
    from dpnegf_b200 import workload
    from dpnegf_b200.ozaki_res_cal import ozaki_residues
    from dpnegf_b200.scf import ozaki_weights
    dims = [6, 8, 6]
    devs = [workload.random_device(0, 0, seed=70 + k, block_dims=dims) for k in range(2)]
    kBT, mu_L, vL, vR = 0.025, 0.05, 0.1, -0.1
    fL = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vL)) / kBT))
    fR = lambda x: 1.0 / (1.0 + torch.exp((x - (mu_L - vR)) / kBT))
    poles, res = ozaki_residues(4)
    z, c, w = ozaki_weights(poles.numpy(), res.numpy(), 1e6, 4, kBT, mu_L, vL=vL, vR=vR, fermi_L=fL, fermi_R=fR)
    gamma = np.linspace(0.05, 0.2, sum(dims))
    return devs, z, c, w, gamma


def _scf_run(ks, wk, iters=6):
    from dpnegf_b200 import rgf_plan
    from dpnegf_b200.scf import ScfLoop
    devs, z, c, w, gamma = _scf_case()
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl) for d in
                              (devs[k] for k in ks)], device="cpu")
    loop = ScfLoop(geom, [None] * len(ks), [None] * len(ks), z, c, w, alpha=0.5, mix=0.3, use_graph=False,
                   wk=wk, plan=_DiagonalPlan(geom, z, gamma))
    V, n = loop.run(iters)
    return V.numpy().copy(), n.numpy().copy()


def _scf_worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        q.put((rank, _scf_run([rank], [(0.25, 0.75)[rank]])))
    finally:
        dist.destroy_process_group()


def test_scf_k_points_over_ranks_match_single_process_gloo():
    """Two k-points (weights 0.25 / 0.75), one per gloo rank: the per-iteration all-reduce of the
    k-summed density gives every rank the single-process SCF trajectory (V and n after 6
    iterations), with the sweep replaced by a coupling-free device on the CPU."""
    V1, n1 = _scf_run([0, 1], [0.25, 0.75])
    assert np.abs(V1).max() > 1e-4  # the potential moves
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_scf_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        np.testing.assert_allclose(got[r][0], V1, rtol=0, atol=1e-13 * np.abs(V1).max())
        np.testing.assert_allclose(got[r][1], n1, rtol=0, atol=1e-13 * np.abs(n1).max())
