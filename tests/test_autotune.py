"""Autotuner bookkeeping on CPU: buckets, the user cache over the shipped table,
and tune() keeping the fastest candidate (timer injected, no GPU)."""
import json

from dpnegf_b200 import autotune


def test_bucket_and_key():
    assert autotune.bucket(16) == 32 and autotune.bucket(130) == 192 and autotune.bucket(512) == 512
    assert autotune.key(200, "mixed", gpu="X") == "X|mixed|n<=256"


def test_tune_store_lookup(tmp_path, monkeypatch):
    user = tmp_path / "user.json"
    shipped = tmp_path / "shipped.json"
    monkeypatch.setenv("DPNEGF_B200_AUTOTUNE", str(user))
    monkeypatch.setattr(autotune, "SHIPPED", str(shipped))
    monkeypatch.setattr(autotune, "gpu_name", lambda: "FakeGPU")
    autotune._loaded.clear()
    shipped.write_text(json.dumps({"FakeGPU|fp64|n<=256": {"best": {"inv_ob": 128}, "ms": {}}}))
    assert autotune.lookup(250, "fp64") == {"inv_ob": 128}          # shipped table
    assert autotune.lookup(250, "mixed") == {}                       # untuned
    times = {64: 1.0, 128: 2.0, 256: 3.0, 512: 0.5}
    timer = lambda n, p, ob, inverse: times[ob] if inverse == "gj" else 0.8
    best = autotune.tune(250, "fp64", timer=timer)
    assert best == {"inverse": "block", "inv_ob": 64}  # 512 >= 2n is not a distinct candidate
    assert autotune.lookup(250, "fp64") == {"inverse": "block", "inv_ob": 64}  # user cache wins
    saved = json.loads(user.read_text())
    assert saved["FakeGPU|fp64|n<=256"]["ms"] == {"64": 1.0, "128": 2.0, "256": 3.0, "block": 0.8}
    slow = lambda n, p, ob, inverse: times[ob] if inverse == "gj" else 9.0
    assert autotune.tune(100, "mixed", timer=slow) == {"inverse": "gj", "inv_ob": 64}
    autotune._loaded.clear()
