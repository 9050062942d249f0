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
