"""Poles and residues of the Ozaki continued-fraction Fermi expansion.

Host-side set-up of the density integral (negf/ozaki_res_cal.py:8-37):
T. Ozaki, Phys. Rev. B 75, 035123 (2007); Karrasch, Meden, Schoenhammer,
Phys. Rev. B 82, 125114 (2010).  The 2M x 2M symmetric tridiagonal matrix has
zero diagonal and off-diagonal 1 / (2 sqrt((2n-1)(2n+1))), n = 1..2M-1.  Its
M positive eigenvalues lambda give the poles 1/lambda (ascending, in units of
kT) and the residues |v_0|^2 / (4 lambda^2).
"""
import numpy as np
import torch
from scipy.linalg import eigh_tridiagonal


def ozaki_residues(M_cut: int = 1000):
    M = int(M_cut)
    N = 2 * M
    k = np.arange(1, N, dtype=np.float64)
    off = 0.5 / np.sqrt((2.0 * k - 1.0) * (2.0 * k + 1.0))
    lam, vec = eigh_tridiagonal(np.zeros(N), off, select="i", select_range=(M, N - 1))
    poles = (1.0 / lam)[::-1]
    res = (np.abs(vec[0, :]) ** 2 / (4.0 * lam ** 2))[::-1]
    return torch.from_numpy(poles.copy()), torch.from_numpy(res.copy())
