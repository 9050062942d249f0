"""Bloch unfolding of lead k-points (negf/bloch.py:5-56).

A lead whose transverse cell is a (B0, B1, B2) supercell of a smaller cell is
solved on the small cell at the B0*B1*B2 unfolded k-points (k + m)/B.
"""
import numpy as np


class Bloch:
    def __init__(self, bloch_factor):
        f = np.asarray(bloch_factor, dtype=np.int64).reshape(-1)
        assert f.shape[0] == 3, "kpoint should be a 3D vector"
        self.bloch_factor = f

    def unfold_points(self, k):
        k = np.asarray(k, dtype=np.float64).reshape(-1)
        assert k.shape[0] == 3, "kpoint should be a 3D vector"
        B = self.bloch_factor
        # ordering: the first factor varies fastest (reference :48-56)
        m2, m1, m0 = np.meshgrid(np.arange(B[2]), np.arange(B[1]), np.arange(B[0]), indexing="ij")
        out = np.stack([(m0 + k[0]) / B[0], (m1 + k[1]) / B[1], (m2 + k[2]) / B[2]], axis=-1)
        return out.reshape(-1, 3)
