"""Autotuner for the sweep's schedule knobs.

Two knobs of the in-kernel Schur-complement inverse are tuned together: the
inverse scheme (``inverse``: "block", recursive 2x2 blocks with every update on
the tile GEMM and pivoted Gauss-Jordan only on 64-wide leaves, or "gj", pivoted
Gauss-Jordan over the whole block) and the Gauss-Jordan outer block width
``inv_ob`` (64, 128, 256 or 512 columns; 32 is accepted too but never won),
which "gj" uses throughout and "block" uses when its residual probe sends an
item back to Gauss-Jordan.  Narrower outer blocks move work from the panels'
rank-32 updates (FP64 tensor cores, fed from shared memory) to the outer block
GEMM, which runs on the tile GEMM, or on the tcgen05 3xTF32 GEMM in the mixed
sweep; a width of at least n leaves no outer update.  Which choice is fastest
depends on block size and precision.  Results agree to rounding for every
choice.

``tune(n, precision)`` times each candidate on a short synthetic sweep of
block size ``n`` (one item per SM, four blocks) and stores the winner per
(GPU name, precision, block-size bucket) in the user cache
(``$DPNEGF_B200_AUTOTUNE`` or ``~/.cache/dpnegf_b200/autotune.json``).
``lookup`` reads the user cache first, then the table shipped with the
package (``autotune_b200.json``, written by ``python -m dpnegf_b200.autotune
--write-shipped`` on a B200), and returns ``{}`` when neither has an entry.
"""
import argparse
import json
import os
from typing import Callable, Dict, Optional

CANDIDATES = {"inv_ob": (64, 128, 256, 512), "inverse": ("block", "gj")}
BUCKETS = (32, 64, 96, 128, 192, 256, 384, 512)
SHIPPED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "autotune_b200.json")
_loaded: Dict[str, dict] = {}


def cache_path() -> str:
    p = os.environ.get("DPNEGF_B200_AUTOTUNE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "dpnegf_b200", "autotune.json")


def bucket(n: int) -> int:
    for b in BUCKETS:
        if n <= b:
            return b
    return BUCKETS[-1]


def gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"


def key(n: int, precision: str, gpu: Optional[str] = None) -> str:
    return f"{gpu or gpu_name()}|{precision}|n<={bucket(n)}"


def _read(path: str) -> dict:
    if path not in _loaded:
        try:
            with open(path) as f:
                _loaded[path] = json.load(f)
        except (OSError, ValueError):
            _loaded[path] = {}
    return _loaded[path]


def lookup(n: int, precision: str, gpu: Optional[str] = None) -> dict:
    """Tuned knobs for block size n (largest block of the batch) and precision; {} if untuned."""
    k = key(n, precision, gpu)
    for path in (cache_path(), SHIPPED):
        entry = _read(path).get(k)
        if entry:
            return dict(entry["best"])
    return {}


def store(n: int, precision: str, best: dict, times: dict, path: Optional[str] = None,
          gpu: Optional[str] = None) -> None:
    path = path or cache_path()
    table = dict(_read(path))
    table[key(n, precision, gpu)] = {"best": best, "ms": times}
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    _loaded[path] = table


def _time_sweep(n: int, precision: str, inv_ob: int, inverse: str = "gj", L: int = 4, repeats: int = 2) -> float:
    """Device time (ms) of one sweep (T + DOS) of a synthetic device, one item per SM."""
    import torch
    from . import _lib, rgf_plan, workload
    lib = _lib.load()
    B = max(1, lib.negf_sm_count())
    dev = workload.random_device(n, L, seed=11)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl)])
    seL = workload.random_self_energy(B, n, seed=12).cuda()
    seR = workload.random_self_energy(B, n, seed=13).cuda()
    E = workload.energy_grid(B).to(torch.complex128).cuda()
    ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    kw = dict(eta=1e-5, outputs=(), trans=True, dos=True, precision=precision, inv_ob=inv_ob, inverse=inverse)
    rgf_plan.run(geom, [E], [seL], [seR], **kw)
    best = float("inf")
    for _ in range(repeats):
        rgf_plan.run(geom, [E], [seL], [seR], events=ev, **kw)
        torch.cuda.synchronize()
        best = min(best, ev[0].elapsed_time(ev[1]))
    return best


def tune(n: int, precision: str = "fp64", write: bool = True, path: Optional[str] = None,
         timer: Optional[Callable[..., float]] = None) -> dict:
    """Time every Gauss-Jordan inv_ob candidate and the block inverse for block size n and keep
    the fastest scheme, with the fastest Gauss-Jordan width (the block scheme's fallback)."""
    timer = timer or _time_sweep
    cands = [ob for ob in CANDIDATES["inv_ob"] if ob < 2 * n] or [CANDIDATES["inv_ob"][0]]
    times = {str(ob): float(timer(n, precision, ob, inverse="gj")) for ob in cands}
    ob_best = int(min(times, key=lambda k: times[k]))
    times["block"] = float(timer(n, precision, ob_best, inverse="block"))
    scheme = "block" if times["block"] < times[str(ob_best)] else "gj"
    best = {"inverse": scheme, "inv_ob": ob_best}
    if write:
        store(n, precision, best, times, path=path)
    return best


def main(argv=None):
    ap = argparse.ArgumentParser(description="tune the sweep's schedule knobs on this GPU")
    ap.add_argument("--sizes", default="32,64,96,128,192,256,384,512")
    ap.add_argument("--precisions", default="fp64,mixed")
    ap.add_argument("--write-shipped", action="store_true", help="write the table shipped with the package")
    a = ap.parse_args(argv)
    path = SHIPPED if a.write_shipped else cache_path()
    for prec in a.precisions.split(","):
        for n in (int(x) for x in a.sizes.split(",")):
            best = tune(n, prec, path=path)
            entry = _read(path)[key(n, prec)]
            print(json.dumps({"n": n, "precision": prec, "best": best, "ms": entry["ms"]}), flush=True)


if __name__ == "__main__":
    main()
