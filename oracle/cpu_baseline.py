"""Timed CPU baseline: the numpy oracle RGF on the host cores.

TEST/BASELINE INFRASTRUCTURE ONLY -- used by ``bench.py``'s ``cpu_baseline``
and ``--impl reference`` legs.  The reference's own CPU path is torch/MKL
Python (negf/recursive_green_cal.py); its restatement in ``rgf_oracle`` runs
the same complex128 algorithm through numpy's LAPACK/BLAS, so it stands in
for the reference on machines without the reference sources.

Work is split over a ``spawn`` process pool, one process per core with one
BLAS thread each (threaded batched LAPACK solves were seen to hang in this
image's torch/MKL, and one-thread-per-process is the reference's own
self-energy pool layout, negf/lead_property.py:878-893).
"""
import multiprocessing as mp
import os
import time

import numpy as np


def _worker_init():
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    try:
        from threadpoolctl import threadpool_limits
        threadpool_limits(1)
    except Exception:
        pass


_CACHE = {}


def _device(b, L, seed):
    key = (b, L, seed)
    if key not in _CACHE:
        import sys
        root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
        if root not in sys.path:
            sys.path.insert(0, root)
        from dpnegf_b200 import workload
        d = workload.random_device(b, L, seed=seed)
        np_ = lambda xs: [x.numpy() for x in xs]
        _CACHE.clear()
        _CACHE[key] = (np_(d.hd), np_(d.hu), np_(d.hl), np_(d.sd), np_(d.su), np_(d.sl))
    return _CACHE[key]


def _self_energies(b, B, seed):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    if root not in sys.path:
        sys.path.insert(0, root)
    from dpnegf_b200 import workload
    return (workload.random_self_energy(B, b, seed=seed + 1).numpy(),
            workload.random_self_energy(B, b, seed=seed + 2).numpy())


def transport_point(args):
    """T and DOS at one energy (oracle RGF + reductions); returns (T, DOS, seconds)."""
    b, L, seed, e, seL, seR, eta = args
    from oracle import rgf_oracle
    hd, hu, hl, sd, su, sl = _device(b, L, seed)
    t0 = time.perf_counter()
    out = rgf_oracle.rgf(np.array([e]), hl, hd, hu, sd, su, sl, seL[None], seR[None], eta=eta)
    T = rgf_oracle.transmission(out["g_trans"], rgf_oracle.gamma_from_se(seL[None]),
                                rgf_oracle.gamma_from_se(seR[None]))
    D = rgf_oracle.dos(out["grd"], out["grl"], out["gru"], sd, su, sl)
    return float(T[0]), float(D[0]), time.perf_counter() - t0


def run_sample(b, L, seed, energies, seL, seR, eta, procs):
    """Evaluate ``energies`` over ``procs`` single-thread processes; wall time excludes pool start."""
    ctx = mp.get_context("spawn")
    tasks = [(b, L, seed, float(e), seL[i], seR[i], eta) for i, e in enumerate(energies)]
    with ctx.Pool(procs, initializer=_worker_init) as pool:
        # warm the workers (imports, device generation) outside the timed region
        pool.map(_warm, [(b, L, seed)] * procs, chunksize=1)
        t0 = time.perf_counter()
        res = pool.map(transport_point, tasks, chunksize=1)
        wall = time.perf_counter() - t0
    return np.array([r[0] for r in res]), np.array([r[1] for r in res]), wall


def _warm(args):
    b, L, seed = args
    _device(b, L, seed)
    time.sleep(0.2)
    return os.getpid()
