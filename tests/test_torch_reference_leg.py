"""The torch restatement of the reference's GPU path that bench.py times
(``torch_reference_tdos``) gives the oracle's T(E) and DOS: it is checked here
on the CPU so the GPU timing it produces is the timing of a correct sweep."""
import numpy as np
import torch

import bench
from dpnegf_b200 import workload
from oracle import rgf_oracle


def test_torch_reference_path_matches_oracle():
    dims = [12] * 4
    dev = workload.random_device(0, 0, seed=21, block_dims=dims)
    B = 3
    seL = workload.random_self_energy(B, 12, seed=22)
    seR = workload.random_self_energy(B, 12, seed=23)
    E = torch.linspace(-1.5, 1.5, B, dtype=torch.float64)
    T, D = bench.torch_reference_tdos(dev.hd, dev.hu, dev.hl, dev.sd, dev.su, dev.sl, E, seL, seR, 1e-5)
    npy = lambda xs: [x.numpy() for x in xs]
    ref = rgf_oracle.rgf(E.numpy().astype(np.complex128), npy(dev.hl), npy(dev.hd), npy(dev.hu), npy(dev.sd),
                         npy(dev.su), npy(dev.sl), seL.numpy(), seR.numpy(), eta=1e-5)
    gL, gR = rgf_oracle.gamma_from_se(seL.numpy()), rgf_oracle.gamma_from_se(seR.numpy())
    T_ref = rgf_oracle.transmission(ref["g_trans"], gL, gR)
    D_ref = rgf_oracle.dos(ref["grd"], ref["grl"], ref["gru"], npy(dev.sd), npy(dev.su), npy(dev.sl))
    np.testing.assert_allclose(T.numpy(), T_ref, rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(D.numpy(), D_ref, rtol=1e-10, atol=1e-12)
