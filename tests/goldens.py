"""Loader for the committed reference fixtures in ``tests/golden``."""
import os

import numpy as np

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


class Golden:
    def __init__(self, name):
        self.path = os.path.join(GOLDEN_DIR, name if name.endswith(".npz") else name + ".npz")
        self._z = dict(np.load(self.path))

    def has(self, key):
        return key in self._z or f"{key}#len" in self._z

    def __getitem__(self, key):
        if key in self._z:
            return self._z[key]
        n = int(self._z[f"{key}#len"])
        return [self[f"{key}/{i}"] for i in range(n)]

    def get(self, key, default=None):
        return self[key] if self.has(key) else default


def rgf_cases():
    return sorted(f[:-4] for f in os.listdir(GOLDEN_DIR) if f.startswith("rgf_") and f.endswith(".npz"))
