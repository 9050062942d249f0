"""Host-side argument checks of the product-chain wrappers (no GPU needed): malformed inputs
raise ValueError before any device work, and well-formed ones without a CUDA device raise
NegfError (there is no CPU fallback)."""
import numpy as np
import pytest
import torch

from dpnegf_b200 import _lib
from dpnegf_b200.products import coupling_sigma, gamma_sum, lead_adjoint

C = torch.complex128


def _z(*shape):
    return torch.zeros(*shape, dtype=C)


def test_gamma_sum_argument_checks():
    with pytest.raises(ValueError):
        gamma_sum(_z(3, 8, 8), _z(2, 4, 4), 0, torch.ones(3))      # batch mismatch
    with pytest.raises(ValueError):
        gamma_sum(_z(3, 8, 8), _z(3, 4, 4), 6, torch.ones(3))      # columns 6..10 outside G
    with pytest.raises(ValueError):
        gamma_sum(_z(3, 8, 8), _z(3, 4, 4), 4, torch.ones(2))      # one weight per energy
    if not torch.cuda.is_available():
        with pytest.raises(_lib.NegfError):
            gamma_sum(_z(3, 8, 8), _z(3, 4, 4), 4, torch.ones(3))


def test_coupling_sigma_argument_checks():
    with pytest.raises(ValueError):
        coupling_sigma(_z(2, 6, 6), _z(3, 8), None, [0.1, 0.2])     # H_DL wider than g
    with pytest.raises(ValueError):
        coupling_sigma(_z(2, 6, 6), _z(3, 4), _z(3, 5), [0.1, 0.2])  # S_DL shape differs
    with pytest.raises(ValueError):
        coupling_sigma(_z(2, 6, 6), _z(3, 4), None, [0.1])          # one energy per g
    if not torch.cuda.is_available():
        with pytest.raises(_lib.NegfError):
            coupling_sigma(_z(2, 6, 6), _z(3, 4), None, [0.1, 0.2])


def test_lead_adjoint_argument_checks():
    n, nc, B = 5, 3, 2
    blocks = [_z(n, n)] * 4
    E = np.array([0.1, 0.2])
    with pytest.raises(ValueError):
        lead_adjoint(*blocks, None, None, E, 1e-3, _z(B, n, n), _z(B, n, n), 3)      # unknown form
    with pytest.raises(ValueError):
        lead_adjoint(*blocks, None, None, E, 1e-3, _z(B, n, n), _z(B, nc, nc), 0)    # form 0 without H_DL
    with pytest.raises(ValueError):
        lead_adjoint(*blocks, _z(nc, n), None, E, 1e-3, _z(B, n, n), _z(B, n, n), 0)  # dL/dSigma not nc x nc
    with pytest.raises(ValueError):
        lead_adjoint(*blocks, _z(nc, n), None, E, 1e-3, _z(B, n, n), _z(1, nc, nc), 0)  # one per energy
    with pytest.raises(ValueError):
        lead_adjoint(*blocks, None, None, E[:1], 1e-3, _z(B, n, n), _z(B, n, n), 1)  # energies vs g_s
    if not torch.cuda.is_available():
        with pytest.raises(_lib.NegfError):
            lead_adjoint(*blocks, _z(nc, n), None, E, 1e-3, _z(B, n, n), _z(B, nc, nc), 0)
