"""The synthetic meshes are conforming NVB triangulations of the domain (CPU)."""
import numpy as np
import pytest

import fixtures as F


@pytest.mark.parametrize("name", ["tiny", "small", "medium", "c0"])
def test_mesh_conforming(name):
    m = F.make_mesh(name)
    q = F.validate(m)
    assert q["min_area"] > 0.0
    assert q["max_count"] <= 2
    assert q["bad_boundary_edges"] == 0
    assert q["min_angle"] > 10.0
    assert abs(q["area"] - (4.0 - np.pi * 0.01)) < 2e-3


def test_mesh_deterministic():
    a, b = F.make_mesh("small"), F.make_mesh("small")
    assert np.array_equal(a.tri, b.tri) and np.array_equal(a.x, b.x)


def test_boundary_tags():
    m = F.make_mesh("small")
    r = np.hypot(m.x - F.XC, m.y - F.YC)
    cyl = m.tag == F.BC_CYLINDER
    assert cyl.any() and np.allclose(r[cyl], F.RC, atol=1e-12)
    assert np.all(m.x[m.tag == F.BC_INLET] == 0.0)
    assert np.all(m.x[m.tag == F.BC_OUTLET] == F.LX)
    w = m.tag == F.BC_WALL
    assert np.all((m.y[w] == 0.0) | (m.y[w] == F.LY))


def test_uniform_bisection_doubles_elements():
    m = F.make_mesh("tiny")
    r = F.refine_uniform(m, 2)
    assert r.ne >= 4 * m.ne
    assert F.validate(r)["max_count"] <= 2
