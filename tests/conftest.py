import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "cylinder-fem-amr_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def golden(name):
    import numpy as np
    path = os.path.join(GOLDEN, name)
    if not os.path.exists(path):
        pytest.skip(f"golden file {name} not generated yet")
    return np.load(path)


class MeshFromGolden:
    """A fixtures.Mesh-like view of the mesh stored in a golden file."""

    def __init__(self, g):
        import numpy as np
        self.x = np.ascontiguousarray(g["x"])
        self.y = np.ascontiguousarray(g["y"])
        self.tag = np.ascontiguousarray(g["tag"], dtype=np.int32)
        self.tri = np.ascontiguousarray(g["elem_v"], dtype=np.int32).reshape(-1, 3)
        self.gen = np.zeros(self.tri.shape[0], np.int32)

    @property
    def n(self):
        return self.x.size

    @property
    def ne(self):
        return self.tri.shape[0]

    @property
    def elem_v(self):
        return self.tri.reshape(-1)
