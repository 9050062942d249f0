"""negf_rgf_run_static: the sweep with library-owned scratch, for callers that
cannot allocate device memory during the solve (e.g. a host transport code
that owns the GPU through its own memory pool).

Collected last on purpose.  Two calls in a row through the C ABI must match
the caller-scratch entry point negf_rgf_run within the suite's FP64 tolerance;
a problem whose single work slot exceeds the static array is rejected before
any launch.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def _case(b=64, L=6, B=50, seed=31):
    from dpnegf_b200 import rgf_plan, workload
    d = workload.random_device(b, L, seed=seed)
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl)])
    E = torch.linspace(-2.5, 2.5, B, dtype=torch.float64).to(torch.complex128)
    seL = workload.random_self_energy(B, b, seed=seed + 1).cuda()
    seR = workload.random_self_energy(B, b, seed=seed + 2).cuda()
    return geom, E, seL, seR


def test_static_scratch_matches_caller_scratch_twice():
    from dpnegf_b200 import noalloc, rgf_plan
    geom, E, seL, seR = _case()
    ref = rgf_plan.run(geom, [E.cuda()], [seL], [seR], eta=1e-5, outputs=(), trans=True, dos=True)
    T_ref, D_ref = ref.trans.cpu().numpy(), ref.dos.cpu().numpy()
    for _ in range(2):  # the second call reuses the array left over by the first
        T, D, st, code = noalloc.transmission_dos_static(geom, E, seL, seR, eta=1e-5)
        assert code == 0
        assert int((st != 0).sum()) == 0
        np.testing.assert_allclose(T.cpu().numpy(), T_ref, rtol=RTOL, atol=1e-12)
        np.testing.assert_allclose(D.cpu().numpy(), D_ref, rtol=RTOL, atol=1e-12)


def test_static_scratch_rejects_oversized_problem():
    from dpnegf_b200 import noalloc
    geom, E, seL, seR = _case(b=512, L=2, B=2, seed=5)
    assert noalloc.static_scratch_bytes() == 64 << 20
    T, D, st, code = noalloc.transmission_dos_static(geom, E, seL, seR, eta=1e-5)
    assert code == noalloc.NEGF_ERR_SCRATCH_LIMIT
