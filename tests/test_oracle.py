"""The oracle (CPU restatement, oracle/cfa_oracle.c) pinned against the reference's own code.

* Golden vectors from the reference's host code (tests/golden/ref_host_*.npz, made by
  tests/golden/make_golden.py host): CSR pattern, SA-AMG hierarchies, SpGEMM and transpose --
  bit-exact.
* Golden vectors from the reference's CUDA build (tests/golden/ref_gpu_*.npz, made on a GPU by
  make_golden.py gpu): colouring (bit-exact), ILU factor and apply, BiCGSTAB2 solutions,
  assembled step systems -- to 1e-12 / the solver tolerance.
* The reference's own unit tests on the hot path (tests/test_cfa.cu: test_momentum_ilu,
  test_oss_assembled, test_amg_remap part 1) restated on the oracle.
"""
import numpy as np
import pytest

import fixtures as F
from tests.conftest import MeshFromGolden, golden
from oracle import oracle as O


def rows_rel_err(a, b, rp):
    """max over rows of |a - b| / max(|row of b|), the assembled-value metric (1e-12)."""
    err = 0.0
    for i in range(rp.size - 1):
        s, e = rp[i], rp[i + 1]
        scale = max(np.abs(b[s:e]).max(), 1e-300)
        err = max(err, np.abs(a[s:e] - b[s:e]).max() / scale)
    return err


@pytest.mark.parametrize("name", ["tiny", "small"])
def test_csr_matches_reference(name):
    g = golden(f"ref_host_{name}.npz")
    m = MeshFromGolden(g)
    rp, ci = O.csr_build(m.n, m.elem_v)
    assert np.array_equal(rp, g["rp"]) and np.array_equal(ci, g["ci"])


@pytest.mark.parametrize("name", ["tiny", "small"])
@pytest.mark.parametrize("which", ["ppe", "lap"])
def test_amg_hierarchy_matches_reference(name, which):
    g = golden(f"ref_host_{name}.npz")
    rp, ci = g["rp"], g["ci"]
    amg = O.Amg(rp, ci, g[f"{which}_val"])
    assert amg.nlev == int(g[f"{which}_levels"][0])
    for l in range(amg.nlev):
        L = amg.level(l)
        assert L["omega"] == g[f"{which}_L{l}_omega"][0]
        for name_ in ("A", "P", "R"):
            _, _, r_, c_, v_ = L[name_]
            assert np.array_equal(r_, g[f"{which}_L{l}_{name_}_rp"])
            assert np.array_equal(c_, g[f"{which}_L{l}_{name_}_ci"])
            assert np.array_equal(v_, g[f"{which}_L{l}_{name_}_v"])
    Ac, inv = amg.coarse()
    assert amg.coarse_n == int(g[f"{which}_coarse_n"][0])
    assert np.array_equal(inv.ravel(), g[f"{which}_coarse_inv"])


def test_spgemm_and_transpose_match_reference():
    g = golden("ref_host_spgemm.npz")
    for t in range(3):
        ar, ac, bc = (int(v) for v in g[f"t{t}_dims"])
        A = (ar, ac, g[f"t{t}_A_rp"], g[f"t{t}_A_ci"], g[f"t{t}_A_v"])
        B = (ac, bc, g[f"t{t}_B_rp"], g[f"t{t}_B_ci"], g[f"t{t}_B_v"])
        Cm = O.csr_multiply(A, B)
        assert np.array_equal(Cm[2], g[f"t{t}_C_rp"]) and np.array_equal(Cm[3], g[f"t{t}_C_ci"])
        assert np.array_equal(Cm[4], g[f"t{t}_C_v"])
        T = O.csr_transpose(A)
        assert np.array_equal(T[2], g[f"t{t}_T_rp"]) and np.array_equal(T[3], g[f"t{t}_T_ci"])
        assert np.array_equal(T[4], g[f"t{t}_T_v"])


# ------------------------------------------------------------------------------------------------
# restated reference unit tests (tests/test_cfa.cu)
# ------------------------------------------------------------------------------------------------
def ilu_identity_error(rp, ci, a, colour, lu):
    """max |(LU)_ij - a_ij| / |a_ii| over the pattern, order (colour, index) (test_cfa.cu:253-271)."""
    n = rp.size - 1
    pos = {}
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            pos[(i, ci[k])] = k

    def before(p, q):
        return colour[p] < colour[q] or (colour[p] == colour[q] and p < q)

    err = 0.0
    for i in range(n):
        for e in range(rp[i], rp[i + 1]):
            j = ci[e]
            s = 0.0
            for q in range(rp[i], rp[i + 1]):
                k = ci[q]
                if not (k == i or before(k, i)) or not (k == j or before(k, j)):
                    continue
                kj = pos.get((k, j))
                if kj is None:
                    continue
                s += (1.0 if k == i else lu[q]) * lu[kj]
            err = max(err, abs(s - a[e]) / abs(a[pos[(i, i)]]))
    return err


def test_momentum_ilu_restated():
    """test_momentum_ilu (tests/test_cfa.cu:205-293) on the oracle."""
    from tests.golden.make_golden import momentum_ilu_matrix
    g = golden("ref_host_tiny.npz")
    rp, ci = g["rp"], g["ci"]
    n = rp.size - 1
    a, b = momentum_ilu_matrix(rp, ci)
    ilu = O.Ilu(rp, ci)
    lu, _, _, _ = ilu.factor(a)
    col = ilu.colour
    bad = sum(1 for i in range(n) for k in range(rp[i], rp[i + 1]) if ci[k] != i and col[ci[k]] == col[i])
    assert bad == 0
    assert ilu_identity_error(rp, ci, a, col, lu) < 1e-12
    xu, xv, reps = O.bicgstab2(rp, ci, a, b[:n], b[n:], np.zeros(n), np.zeros(n), ilu, 200, 1e-10)
    xj0, r0 = O.bicgstab(rp, ci, a, b[:n], np.zeros(n), 400, 1e-10)
    xj1, r1 = O.bicgstab(rp, ci, a, b[n:], np.zeros(n), 400, 1e-10)
    x, xj = np.concatenate([xu, xv]), np.concatenate([xj0, xj1])
    assert reps[0].converged and reps[1].converged
    assert np.abs(x - xj).max() < 1e-8 * np.abs(xj).max()


def test_oss_assembled_restated():
    """test_oss_assembled (tests/test_cfa.cu:296-329) on the oracle."""
    m = F.make_mesh("small")
    rp, ci = O.csr_build(m.n, m.elem_v)
    rng = np.random.default_rng(11)
    xin = rng.uniform(size=m.n) - 0.5
    s = 0.1 + rng.uniform(size=m.ne)
    mass = O.lumped_mass(m)
    a, b = np.zeros(m.n), np.zeros(m.n)
    O.oss_matrix_free(m, s, mass, xin, a)
    oss, inv_m = O.assemble_oss(m, rp, ci, s, mass)
    O.oss_apply(m, rp, ci, oss, inv_m, xin, b)
    scale = np.abs(a).max()
    assert scale > 0 and np.abs(a - b).max() < 1e-12 * scale


def test_amg_setup_and_pcg_restated():
    """test_amg_remap part 1 (tests/test_cfa.cu:333-371): a multi-level hierarchy of the shifted
    graph Laplacian, and PCG with it converging to 1e-10."""
    m = F.make_mesh("medium")
    rp, ci = O.csr_build(m.n, m.elem_v)
    from tests.golden.make_golden import shifted_laplacian
    a = shifted_laplacian(rp, ci)
    amg = O.Amg(rp, ci, a)
    assert amg.nlev + 1 > 2
    b = np.cos(0.11 * np.arange(m.n))
    x, rep = O.pcg(rp, ci, a, b, np.zeros(m.n), 400, 1e-10, amg=amg)
    assert rep.converged
    r = b - O.spmv(rp, ci, a, x)
    assert np.linalg.norm(r) < 1.01e-10 * np.linalg.norm(b)


def test_amg_remap_restated():
    """test_amg_remap (tests/test_cfa.cu:372-437): remapping onto an unchanged mesh gives the
    setup's V-cycle; after a local refinement (new nodes) the remapped hierarchy reaches 1e-10
    with at most 3x + 5 the iterations of a fresh setup."""
    from tests.golden.make_golden import shifted_laplacian
    m = F.make_mesh("medium")
    rp, ci = O.csr_build(m.n, m.elem_v)
    a = shifted_laplacian(rp, ci)
    amg = O.Amg(rp, ci, a)
    assert amg.nlev + 1 > 2
    r = np.sin(0.37 * np.arange(m.n)) + 0.2
    z_setup = amg.apply(r)
    assert amg.remap(rp, ci, a, np.arange(m.n)) and amg.remaps == 1
    z_remap = amg.apply(r)
    assert np.abs(z_remap - z_setup).max() <= 1e-14 * np.abs(z_setup).max()
    m2, n2o = F.refine_blob(m, radius=0.08, rounds=3)
    assert m2.n > m.n and (n2o < 0).any() and (n2o >= 0).sum() == m.n
    rp2, ci2 = O.csr_build(m2.n, m2.elem_v)
    a2 = shifted_laplacian(rp2, ci2)
    assert amg.remap(rp2, ci2, a2, n2o) and amg.remaps == 2
    b = np.cos(0.11 * np.arange(m2.n))
    x, rep = O.pcg(rp2, ci2, a2, b, np.zeros(m2.n), 400, 1e-10, amg=amg)
    x2, rep2 = O.pcg(rp2, ci2, a2, b, np.zeros(m2.n), 400, 1e-10, amg=O.Amg(rp2, ci2, a2))
    assert rep.converged and rep2.converged
    assert rep.iterations <= 3 * rep2.iterations + 5
    # a hierarchy without levels has nothing to reuse: remap sets it up anew
    t = F.make_mesh("tiny")
    trp, tci = O.csr_build(t.n, t.elem_v)
    small = O.Amg(trp, tci, shifted_laplacian(trp, tci), coarse_target=t.n)
    assert small.nlev == 0 and not small.remap(trp, tci, shifted_laplacian(trp, tci), np.arange(t.n))
    assert small.remaps == 0


def test_post_solve_known_answers():
    """The kernels after the solves on exact cases: K f = 0 on interior rows for a linear f
    (k_stiffness_apply), the lumped gradient of a linear dp is its slope on interior nodes and
    the vorticity of a linear shear is constant (k_accumulate_grad_dp_and_vorticity), and the
    volume forces of the fluid at rest are zero (test_force_at_rest, tests/test_cfa.cu:171-185)."""
    m = F.make_mesh("small")
    inner = m.tag == 0
    f = 0.7 * m.x - 1.3 * m.y + 0.2
    out = np.zeros(m.n)
    O.stiffness_apply(m, f, 1.0, out)
    assert np.abs(out[inner]).max() < 1e-12 * np.abs(f).max()
    mass = O.lumped_mass(m)
    u, v = 0.5 * m.y, -0.25 * m.x
    gdx, gdy, vn = O.grad_dp_vorticity(m, f, u, v)
    assert np.abs(gdx[inner] / mass[inner] - 0.7).max() < 1e-12
    assert np.abs(gdy[inner] / mass[inner] + 1.3).max() < 1e-12
    assert np.abs(vn / mass - (-0.25 - 0.5)).max() < 1e-12
    z = np.zeros(m.n)
    assert np.abs(O.volume_forces(m, z, z, z, z, z, z, z, 1.5e3, -2e3, 0.5e3, 1e-3, 1.0)).max() == 0.0


def test_amr_indicators_vanish_for_channel_flow():
    """k_accumulate_recovered_gradient + k_compute_amr_error_indicator: the undisturbed inflow
    profile gives exactly zero (the reference's design statement, fem_kernels.cuh:911-918), a
    disturbed field does not."""
    m = F.make_mesh("small")
    mass = O.lumped_mass(m)
    up = 4 * 1.5 * m.y * (1 - m.y)
    g, err = O.amr_indicators(m, up, np.zeros(m.n), 1.5, 1.0, mass)
    assert np.abs(err).max() == 0.0 and np.abs(g).max() == 0.0
    g, err = O.amr_indicators(m, up + 0.01 * F.fourier_field(m.x, m.y, 4), np.zeros(m.n), 1.5, 1.0, mass)
    assert err[:m.ne].max() > 0 and err[m.ne:].max() > 0


def test_reprojection_reduces_the_discrete_divergence():
    """project_divergence_free (src/cfa/device.cuh:413-461) on a non-solenoidal field: the discrete
    divergence on interior nodes drops, the pressure is untouched."""
    m = F.make_mesh("small")
    rp, ci = O.csr_build(m.n, m.elem_v)
    u, v = F.fourier_field(m.x, m.y, 1), F.fourier_field(m.x, m.y, 2)
    mass = O.lumped_mass(m)
    z = np.zeros(m.n)
    inner = m.tag == 0

    def div_norm(a, b):
        _, _, div = O.assemble_ppe(m, rp, ci, a, b, z, z, z, mass, np.zeros(m.ne), 1e-3, 1.0, 0.0)
        return np.linalg.norm(div[inner])

    before = div_norm(u, v)
    O.project_divergence_free(m, rp, ci, 1e-3, u, v, tol=1e-12)
    assert div_norm(u, v) < 0.5 * before


def test_oracle_stepper_reaches_a_steady_drag():
    """The CPU time loop (the oracle of the device stepper) from rest: the solves converge every
    step and the drag settles; the lift stays small by symmetry of the inflow."""
    m = F.make_mesh("small")
    z = np.zeros(m.n)
    st = O.Stepper(m, z, z, z, dt=5e-3)
    hist = [st.step() for _ in range(12)]
    cd = np.array([h[0] for h in hist])
    assert all(it[2] > 0 for it in st.iters)
    assert abs(cd[-1] - cd[-2]) < 0.05 * abs(cd[-1]) and 0.5 < cd[-1] < 5.0
    assert abs(hist[-1][1]) < 0.05


def test_pcg_oss_amg_step():
    """The pressure solve of a synthetic step: PCG + OSS + AMG reaches 1e-10 with far fewer
    iterations than Jacobi, and both agree."""
    m = F.make_mesh("small")
    rp, ci = O.csr_build(m.n, m.elem_v)
    u, v, p = F.fourier_field(m.x, m.y, 1), F.fourier_field(m.x, m.y, 2), 0.3 * F.fourier_field(m.x, m.y, 3)
    A, ru, rv, mass = O.assemble_momentum(m, rp, ci, u, v, u, v, p, O.bdf2_params())
    dt_proj = 2e-3 / 3
    s = O.oss_weights(m, u, v, dt_proj, 1.0, 1e-3, 0.3)
    gx, gy = O.scalar_gradient(m, p, s)
    Kp, rhs, div = O.assemble_ppe(m, rp, ci, u, v, p, gx, gy, mass, s, dt_proj, 1.0, 0.3)
    dp = np.zeros(m.n)
    O.apply_bc_pressure(m, rp, ci, Kp, rhs, dp, mass)
    oss, inv_m = O.assemble_oss(m, rp, ci, s, mass)
    amg = O.Amg(rp, ci, Kp)
    x, rep = O.pcg(rp, ci, Kp, rhs, dp, 4000, 1e-10, oss, inv_m, m.tag, amg)
    xj, repj = O.pcg(rp, ci, Kp, rhs, dp, 4000, 1e-10, oss, inv_m, m.tag, None)
    assert rep.converged and repj.converged and rep.iterations < repj.iterations / 5
    assert np.abs(x - xj).max() < 1e-8 * np.abs(x).max()


# ------------------------------------------------------------------------------------------------
# against the reference's CUDA build (golden files made on a GPU)
# ------------------------------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["tiny", "small"])
def test_oracle_matches_reference_gpu(name):
    g = golden(f"ref_gpu_{name}.npz")
    h = golden(f"ref_host_{name}.npz")
    rp, ci = h["rp"], h["ci"]
    n = rp.size - 1
    m = MeshFromGolden(h)
    # colouring bit-exact, factor and apply to 1e-12
    ilu = O.Ilu(rp, ci)
    assert np.array_equal(ilu.colour, g["ilu_colour"])
    assert np.array_equal(ilu.colour_start, g["ilu_colour_start"])
    assert np.array_equal(ilu.rows, g["ilu_rows"])
    lu, _, _, _ = ilu.factor(g["ilu_val"])
    assert rows_rel_err(lu, g["ilu_lu"], rp) < 1e-12
    z = ilu.apply(g["ilu_b"], nrhs=2)
    assert np.abs(z - g["ilu_z"]).max() < 1e-12 * np.abs(g["ilu_z"]).max()
    # BiCGSTAB2 to the reference's tolerance
    b = g["ilu_b"]
    xu, xv, reps = O.bicgstab2(rp, ci, g["ilu_val"], b[:n], b[n:], np.zeros(n), np.zeros(n), ilu, 200, 1e-10)
    x = np.concatenate([xu, xv])
    assert np.abs(x - g["b2_x"]).max() < 1e-8 * np.abs(g["b2_x"]).max()
    assert abs(reps[0].iterations - g["b2_info"][0]) <= 2 and abs(reps[1].iterations - g["b2_info"][2]) <= 2
    # assembled step systems (the reference assembles with FP64 atomics: 1e-12 per row)
    u, v, p = h["u"], h["v"], h["p"]
    A, ru, rv, mass = O.assemble_momentum(m, rp, ci, u, v, u, v, p, O.bdf2_params())
    uu, vv = u.copy(), v.copy()
    O.apply_bc_momentum(m, rp, ci, A, ru, rv, uu, vv)
    assert rows_rel_err(A, g["step_A_val"], rp) < 1e-12
    for k, val in (("rhs_u", ru), ("rhs_v", rv), ("mass", mass)):
        assert np.abs(val - g["step_" + k]).max() <= 1e-12 * np.abs(g["step_" + k]).max()
    us, vs = g["step_u"], g["step_v"]   # the reference's momentum solution enters the PPE
    dt_proj = 2e-3 / 3
    s = O.oss_weights(m, us, vs, dt_proj, 1.0, 1e-3, 0.3)
    assert np.abs(s - g["step_elem_s"]).max() <= 1e-12 * np.abs(g["step_elem_s"]).max()
    gx, gy = O.scalar_gradient(m, p, s)
    assert np.abs(gx - g["step_gpx"]).max() <= 1e-12 * np.abs(g["step_gpx"]).max()
    Kp, rhs, div = O.assemble_ppe(m, rp, ci, us, vs, p, gx, gy, mass, s, dt_proj, 1.0, 0.3)
    dp = np.zeros(n)
    O.apply_bc_pressure(m, rp, ci, Kp, rhs, dp, mass)
    assert rows_rel_err(Kp, g["step_Kp_val"], rp) < 1e-12
    assert np.abs(rhs - g["step_rhs_p"]).max() <= 1e-12 * np.abs(g["step_rhs_p"]).max()
    oss, inv_m = O.assemble_oss(m, rp, ci, s, mass)
    nnz = ci.size
    for q in range(4):
        assert rows_rel_err(oss[q * nnz:(q + 1) * nnz], g["step_oss_val"][q * nnz:(q + 1) * nnz], rp) < 1e-11
    # solutions of the step (tol 1e-10 relative)
    ilu2 = O.Ilu(rp, ci)
    ilu2.factor(A)
    xu, xv, reps = O.bicgstab2(rp, ci, A, ru, rv, uu, vv, ilu2, 1000, 1e-10)
    assert reps[0].converged and reps[1].converged and g["step_conv"][0] and g["step_conv"][1]
    assert np.abs(xu - us).max() < 1e-8 * np.abs(us).max()
    assert np.abs(xv - vs).max() < 1e-8 * np.abs(vs).max()
    amg = O.Amg(rp, ci, Kp)
    x, rep = O.pcg(rp, ci, Kp, rhs, dp, 4000, 1e-10, oss, inv_m, m.tag, amg)
    assert rep.converged and g["step_conv"][2]
    assert np.abs(x - g["step_dp"]).max() < 1e-7 * np.abs(g["step_dp"]).max()
    assert abs(rep.iterations - g["step_its"][2]) <= 2
    # Laplacian PCG + AMG, one V-cycle (bit-exact hierarchy -> V-cycle to round-off)
    amgl = O.Amg(rp, ci, h["lap_val"])
    zl = amgl.apply(np.sin(0.37 * np.arange(n)) + 0.2)
    assert np.abs(zl - g["lap_vcycle_z"]).max() < 1e-12 * np.abs(g["lap_vcycle_z"]).max()
    xl, repl = O.pcg(rp, ci, h["lap_val"], np.cos(0.11 * np.arange(n)), np.zeros(n), 400, 1e-10, amg=amgl)
    assert repl.converged and abs(repl.iterations - g["lap_pcg_info"][0]) <= 1
    assert np.abs(xl - g["lap_pcg_x"]).max() < 1e-8 * np.abs(g["lap_pcg_x"]).max()


def test_fp64_first_phase_keeps_the_fp64_iteration_count():
    """The CPU emulation of the V-cycle per precision (oracle/vcycle_precision.py) on the c0
    pressure system: the V-cycle in FP32 throughout takes more PCG iterations to 1e-10 than in
    FP64, and FP64 V-cycles down to 1e-2 of the initial residual followed by FP32 ones take the
    FP64 count: the schedule of the mixed-precision solves."""
    from oracle import vcycle_precision as VP
    m = F.make_mesh("c0")
    rp, ci, Kp, rhs, oss, inv_m = VP.pressure_system(m)

    def op(x):
        y = O.spmv(rp, ci, Kp, x)
        O.oss_apply(m, rp, ci, oss, inv_m, x, y)
        return y

    h = VP.Hierarchy(rp, ci, Kp)
    nl = len(h.levels)
    all64, all32 = h.cast([np.float64] * nl), h.cast([np.float32] * nl)
    it64 = VP.pcg_iterations(h, op, rhs, all64)
    it32 = VP.pcg_iterations(h, op, rhs, all32)
    itph = VP.pcg_iterations(h, op, rhs, all64, all32, 1e-2)
    assert 0 < it64 < it32
    assert itph == it64
