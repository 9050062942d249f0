"""Host-side logic that needs no GPU: Fiori's quadrature set-up and errors (as the reference's
negf/density.py:236-265), its atom-to-block index against the oracle's restatement of
density.py:362-395 on random layouts, and the SCF loop's argument checks."""
import numpy as np
import pytest
import torch

from oracle import lead_oracle


def test_fiori_quadrature_and_errors():
    from dpnegf_b200.density import Fiori
    grid = torch.linspace(-0.5, 0.5, 11, dtype=torch.float64)
    f = Fiori(integrate_way="direct", e_grid=grid)
    assert f.pre_factor.dtype == torch.float32 and torch.allclose(f.pre_factor, torch.full((11,), 0.1))
    assert f.integrate_range is grid
    g = Fiori(n_gauss=8, integrate_way="gauss", e_grid=grid)
    x, w = lead_oracle.gauss_xw(-0.5, 0.5, 8)
    np.testing.assert_allclose(g.integrate_range.numpy(), x, atol=1e-7)
    np.testing.assert_allclose(g.pre_factor.numpy(), w, atol=1e-7)
    with pytest.raises(AssertionError, match="n_gauss must be set"):
        Fiori(integrate_way="gauss", e_grid=grid)
    with pytest.raises(ValueError, match="only supports 'gauss' and 'direct'"):
        Fiori(integrate_way="simpson", e_grid=grid)


def test_fiori_subblock_index_matches_oracle_on_random_layouts():
    from dpnegf_b200.density import Fiori
    f = Fiori(integrate_way="direct", e_grid=torch.linspace(0, 1, 3))
    rng = np.random.default_rng(11)
    for _ in range(200):
        norbs = list(rng.integers(1, 6, size=int(rng.integers(1, 12))))
        total = sum(norbs)
        cuts = sorted(set(rng.integers(1, total, size=int(rng.integers(0, 4))).tolist())) if total > 1 else []
        blocks = list(np.diff([0] + cuts + [total]))
        for a in range(len(norbs)):
            assert f.get_subblock_index(blocks, a, norbs) == lead_oracle.fiori_subblock_index(blocks, a, norbs)


def test_scf_loop_argument_checks():
    from dpnegf_b200 import rgf_plan, workload
    from dpnegf_b200.scf import ScfLoop
    devs = [workload.random_device(0, 0, seed=s, block_dims=[4, 6]) for s in (1, 2)]
    geom = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl) for d in devs],
                             device="cpu")
    z, c, w = np.array([1j]), np.array([1.0 + 0j]), np.zeros(1)
    with pytest.raises(ValueError, match="self-energy stack per k-point"):
        ScfLoop(geom, [None], [None], z, c, w, plan=object())
    with pytest.raises(ValueError, match="k weights"):
        ScfLoop(geom, [None] * 2, [None] * 2, z, c, w, wk=[1.0], plan=object())
    other = workload.random_device(0, 0, seed=3, block_dims=[4, 7])
    mixed = rgf_plan.Geometry([rgf_plan.DeviceBlocks(d.hd, d.hu, d.hl, d.sd, d.su, d.sl) for d in (devs[0], other)],
                              device="cpu")
    with pytest.raises(ValueError, match="same orbitals"):
        ScfLoop(mixed, [None] * 2, [None] * 2, z, c, w, plan=object())


def test_density_onsite_matches_reference():
    """Ozaki.get_density_onsite (per-atom sums of diag(DM) beside the positions) against the
    reference's own, for a matrix and a vector DM (plain torch, no GPU needed)."""
    from types import SimpleNamespace
    from dpnegf_b200.density import Ozaki
    from tests.goldens import Golden
    g = Golden("density_onsite")
    dp = SimpleNamespace(norbs_per_atom=[int(x) for x in g["norbs"]],
                         structure=SimpleNamespace(positions=g["positions"]))
    oz = Ozaki(R=1e6, M_cut=4, n_gauss=2)
    DM = torch.as_tensor(g["DM"])
    np.testing.assert_array_equal(oz.get_density_onsite(dp, DM).numpy(), g["out/matrix"])
    np.testing.assert_array_equal(oz.get_density_onsite(dp, DM.diag() * 2).numpy(), g["out/vector"])


def test_checkpointing_shrinks_the_rgf_slot():
    """With sqrt(K) checkpointing the g and z-tangent slabs of an adjoint slot shrink from
    sum n_q^2 to (ceil(K/s) + s) max_n^2 each (host-side sizing, no GPU)."""
    import ctypes
    from dpnegf_b200 import _lib
    K, n = 36, 32
    sizes = {}
    lib = ctypes.CDLL(_lib.LIB_PATH)
    lib.negf_rgf_scratch_bytes.restype = ctypes.c_size_t
    lib.negf_rgf_scratch_bytes.argtypes = [ctypes.POINTER(_lib.NegfRgfProblem)]
    for ck in (0, 6):
        p = _lib.NegfRgfProblem()
        p.max_n, p.max_g_slab, p.n_slots = n, K * n * n, 1
        p.flags = _lib.ADJOINT | _lib.ADJ_DOS | _lib.TRANS
        p.col_slab = K * n * n
        p.ckpt, p.ckpt_blocks = ck, K
        sizes[ck] = lib.negf_rgf_scratch_bytes(ctypes.byref(p))
    assert sizes[0] - sizes[6] == 2 * (K - 12) * n * n * 16
