"""The --dump-systems files (src/cylinder_fem_amr.cu:332-352, :426-438): byte layout, round trip,
and on a GPU a dumped step solved through the device solvers against the oracle."""
import os

import numpy as np
import pytest

import dumps as D
import fixtures as F
from oracle import oracle as O


def _momentum_system(m):
    rp, ci = O.csr_build(m.n, m.elem_v)
    u, v, p = F.fourier_field(m.x, m.y, 1), F.fourier_field(m.x, m.y, 2), 0.3 * F.fourier_field(m.x, m.y, 3)
    A, ru, rv, mass = O.assemble_momentum(m, rp, ci, u, v, u, v, p, O.bdf2_params())
    uu, vv = u.copy(), v.copy()
    O.apply_bc_momentum(m, rp, ci, A, ru, rv, uu, vv)
    return rp, ci, A, ru, rv, uu, vv


def test_momentum_dump_layout_and_round_trip(tmp_path):
    m = F.make_mesh("tiny")
    rp, ci, A, ru, rv, u0, v0 = _momentum_system(m)
    path = os.path.join(tmp_path, "case_momentum.bin")
    D.write_momentum(path, rp, ci, A, ru, rv, u0, v0, m.x, m.y, m.tag)
    n, nnz = m.n, ci.size
    assert os.path.getsize(path) == 8 + 4 * (n + 1) + 4 * nnz + 8 * nnz + 6 * 8 * n + 4 * n
    raw = np.fromfile(path, "<i4", 2)
    assert raw.tolist() == [n, nnz]
    d = D.read_momentum(path)
    assert "u" not in d
    for k, want in (("row_ptr", rp), ("col_ind", ci), ("val", A), ("rhs_u", ru), ("rhs_v", rv), ("u0", u0),
                    ("v0", v0), ("x", m.x), ("y", m.y), ("bc_tag", m.tag)):
        assert np.array_equal(d[k], want), k
    # the solutions appended after the solves
    D.write_momentum(path, rp, ci, A, ru, rv, u0, v0, m.x, m.y, m.tag, u=2 * u0, v=3 * v0)
    d = D.read_momentum(path)
    assert np.array_equal(d["u"], 2 * u0) and np.array_equal(d["v"], 3 * v0)


def test_pressure_dump_layout_and_round_trip(tmp_path):
    m = F.make_mesh("tiny")
    rp, ci = O.csr_build(m.n, m.elem_v)
    val = np.random.default_rng(1).uniform(size=ci.size)
    rhs, x0 = np.arange(m.n, dtype=float), np.ones(m.n)
    path = os.path.join(tmp_path, "case_pressure.bin")
    D.write_pressure(path, rp, ci, val, rhs, x0)
    assert os.path.getsize(path) == 8 + 4 * (m.n + 1) + 12 * ci.size + 16 * m.n
    d = D.read_pressure(path)
    assert d["n"] == m.n and d["nnz"] == ci.size
    assert np.array_equal(d["val"], val) and np.array_equal(d["rhs"], rhs) and np.array_equal(d["x0"], x0)
    with open(path, "r+b") as f:
        f.truncate(os.path.getsize(path) - 8)
    with pytest.raises(ValueError):
        D.read_pressure(path)


@pytest.mark.gpu
def test_dumped_systems_solve_on_the_device(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    m = F.make_mesh("small")
    rp, ci, A, ru, rv, u0, v0 = _momentum_system(m)
    path = os.path.join(tmp_path, "s_momentum.bin")
    D.write_momentum(path, rp, ci, A, ru, rv, u0, v0, m.x, m.y, m.tag)
    u, v, its = D.solve_momentum(D.read_momentum(path), tol=1e-10, max_iter=400)
    ilu = O.Ilu(rp, ci)
    ilu.factor(A)
    uo, vo, reps = O.bicgstab2(rp, ci, A, ru, rv, u0, v0, ilu, 400, 1e-10)
    assert np.abs(u - uo).max() <= 1e-8 * np.abs(uo).max() and np.abs(v - vo).max() <= 1e-8 * np.abs(vo).max()
    from tests.golden.make_golden import shifted_laplacian
    K = shifted_laplacian(rp, ci)
    b = np.cos(0.11 * np.arange(m.n))
    path = os.path.join(tmp_path, "s_pressure.bin")
    D.write_pressure(path, rp, ci, K, b, np.zeros(m.n))
    x, it = D.solve_pressure(D.read_pressure(path), tol=1e-10)
    xo, rep = O.pcg(rp, ci, K, b, np.zeros(m.n), 4000, 1e-10, amg=O.Amg(rp, ci, K))
    assert np.abs(x - xo).max() <= 1e-8 * np.abs(xo).max()
