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


def test_static_scratch_on_a_side_stream():
    """The call waits for the stream it launched on, so results are complete on return."""
    from dpnegf_b200 import noalloc, rgf_plan
    geom, E, seL, seR = _case(b=48, L=5, B=40, seed=17)
    ref = rgf_plan.run(geom, [E.cuda()], [seL], [seR], eta=1e-5, outputs=(), trans=True, dos=True)
    T_ref, D_ref = ref.trans.cpu().numpy(), ref.dos.cpu().numpy()
    side = torch.cuda.Stream()
    for _ in range(2):
        T, D, st, code = noalloc.transmission_dos_static(geom, E, seL, seR, eta=1e-5, stream=side)
        assert code == 0
        assert int((st != 0).sum()) == 0
        np.testing.assert_allclose(T.cpu().numpy(), T_ref, rtol=RTOL, atol=1e-12)
        np.testing.assert_allclose(D.cpu().numpy(), D_ref, rtol=RTOL, atol=1e-12)


def test_static_scratch_lesser_and_orbital_outputs():
    """A deferred plan with block outputs, the lesser sweep and per-orbital DOS, run once on its
    own scratch and twice on the static array: the same numbers each time."""
    from dpnegf_b200 import noalloc, rgf_plan
    from oracle import rgf_oracle
    b, L, B = 40, 4, 6
    geom, E, seL, seR = _case(b=b, L=L, B=B, seed=23)
    f = np.linspace(0.2, 0.8, B)
    s_in = rgf_oracle.s_in_from_se(seL.cpu().numpy(), seR.cpu().numpy(), f, 1 - f, [b] * L)
    s_in = [[torch.as_tensor(s).cuda() for s in s_in]]
    kw = dict(eta=1e-5, outputs=("grd", "gnd"), trans=True, orb_dos=True, s_in=s_in, check=False, defer=True)
    plan = rgf_plan.run(geom, [E.cuda()], [seL], [seR], **kw)
    assert noalloc.static_slots(plan.prob) >= 1
    plan.launch()
    torch.cuda.synchronize()
    ref = plan.result
    want = {"trans": ref.trans.cpu().numpy(), "orb": ref.orb_dos.cpu().numpy(),
            "grd": [x.cpu().numpy() for x in ref.blocks[0]["grd"]],
            "gnd": [x.cpu().numpy() for x in ref.blocks[0]["gnd"]]}
    for _ in range(2):
        plan2 = rgf_plan.run(geom, [E.cuda()], [seL], [seR], **kw)
        res, code = noalloc.run_plan_static(plan2)
        assert code == 0
        assert int((res.status.cpu() != 0).sum()) == 0
        np.testing.assert_allclose(res.trans.cpu().numpy(), want["trans"], rtol=RTOL, atol=1e-12)
        np.testing.assert_allclose(res.orb_dos.cpu().numpy(), want["orb"], rtol=RTOL, atol=1e-12)
        for tag in ("grd", "gnd"):
            for g, w in zip(res.blocks[0][tag], want[tag]):
                scale = np.abs(w).max()
                assert np.abs(g.cpu().numpy() - w).max() <= RTOL * scale, tag
