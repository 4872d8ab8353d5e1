"""Generates the golden vectors of tests/golden/ from the REFERENCE'S OWN CODE.

  python tests/golden/make_golden.py host        # here: the reference's host code (no GPU)
  python tests/golden/make_golden.py gpu OUTDIR  # on a GPU machine: the reference's CUDA build

Both parts call oracle/_ref/libcfa_ref.so (built by oracle/build.py from the reference source
tree; see oracle/ref_harness.cu) on seeded fixture meshes, and store inputs and outputs, so the
tests never regenerate inputs: they read them from the files.

host: CSR pattern (build_csr_and_boundary_topology), the full SA-AMG hierarchy of two matrices
      (the pressure operator of a synthetic step, and the shifted graph Laplacian of the
      reference's test_amg_remap), csr_multiply/csr_transpose on random sparse matrices.
gpu:  MulticolourIlu0 colouring, factor and apply; GpuBicgstab2 and Jacobi BiCGSTAB solutions on
      the test_momentum_ilu matrix; the assembled step systems and solutions of one synthetic step
      (momentum + pressure with OSS and AMG, tol 1e-10); PCG + AMG on the Laplacian.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cylinder-fem-amr_b200"))

import fixtures as F  # noqa: E402
from oracle import oracle as O  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
MESHES = ("tiny", "small")


def _p(a):
    return O._p(a)


def step_inputs(mesh, seed=0):
    u = F.fourier_field(mesh.x, mesh.y, 1 + 10 * seed)
    v = F.fourier_field(mesh.x, mesh.y, 2 + 10 * seed)
    p = 0.3 * F.fourier_field(mesh.x, mesh.y, 3 + 10 * seed)
    return u, v, p


def oracle_pressure_matrix(mesh, rp, ci, u, v, p):
    """The PPE operator of the synthetic step (oracle assembly: the input of the AMG golden)."""
    A, ru, rv, mass = O.assemble_momentum(mesh, rp, ci, u, v, u, v, p, O.bdf2_params())
    dt_proj = 2e-3 / 3
    s = O.oss_weights(mesh, u, v, dt_proj, 1.0, 1e-3, 0.3)
    gx, gy = O.scalar_gradient(mesh, p, s)
    Kp, rhs, div = O.assemble_ppe(mesh, rp, ci, u, v, p, gx, gy, mass, s, dt_proj, 1.0, 0.3)
    dp = np.zeros(mesh.n)
    O.apply_bc_pressure(mesh, rp, ci, Kp, rhs, dp, mass)
    return Kp


def shifted_laplacian(rp, ci):
    """The SPD matrix of test_amg_remap (tests/test_cfa.cu:335-346)."""
    n = rp.size - 1
    a = np.zeros(ci.size)
    for i in range(n):
        deg = 0
        d = -1
        for k in range(rp[i], rp[i + 1]):
            if ci[k] == i:
                d = k
                continue
            a[k] = -1.0
            deg += 1
        a[d] = deg * (1.0 + 1.0e-4)
    return a


def momentum_ilu_matrix(rp, ci, seed=7):
    """Non-symmetric diagonally dominant matrix in the manner of test_momentum_ilu
    (tests/test_cfa.cu:216-231), drawn with numpy's seeded generator."""
    rng = np.random.default_rng(seed)
    n = rp.size - 1
    a = np.zeros(ci.size)
    b = np.zeros(2 * n)
    for i in range(n):
        off = 0.0
        d = -1
        for k in range(rp[i], rp[i + 1]):
            if ci[k] == i:
                d = k
                continue
            a[k] = -(0.2 + rng.uniform()) * (1.6 if ci[k] > i else 0.6)
            off += abs(a[k])
        a[d] = 1.05 * off + 0.1
        b[i] = rng.uniform() - 0.5
        b[n + i] = np.sin(0.01 * i)
    return a, b


def amg_host(R, rp, ci, v, prefix, out):
    n = rp.size - 1
    h = C.c_void_p(R.ref_amg_host_setup(n, _p(rp), _p(ci), _p(v)))
    nl = R.ref_amg_host_levels(h)
    out[prefix + "levels"] = np.array([nl])
    for l in range(nl):
        for which, name in ((0, "A"), (1, "P"), (2, "R")):
            info = np.zeros(3, np.int32)
            R.ref_amg_host_level(h, l, which, _p(info), None, None, None)
            r_ = np.zeros(info[0] + 1, np.int32)
            c_ = np.zeros(info[2], np.int32)
            v_ = np.zeros(info[2])
            R.ref_amg_host_level(h, l, which, None, _p(r_), _p(c_), _p(v_))
            out[f"{prefix}L{l}_{name}_rp"], out[f"{prefix}L{l}_{name}_ci"], out[f"{prefix}L{l}_{name}_v"] = r_, c_, v_
            out[f"{prefix}L{l}_{name}_shape"] = info[:2].copy()
        out[f"{prefix}L{l}_omega"] = np.array([R.ref_amg_host_omega(h, l)])
    info = np.zeros(3, np.int32)
    R.ref_amg_host_level(h, 0, 3, _p(info), None, None, None)
    cn = int(info[0])
    inv = np.zeros(cn * cn)
    ok = R.ref_amg_host_coarse_inv(h, _p(inv))
    out[prefix + "coarse_n"] = np.array([cn])
    out[prefix + "coarse_inv"] = inv if ok else np.zeros(0)
    R.ref_amg_host_free(h)


def random_csr(rng, rows, cols, per_row):
    rp = [0]
    ci, v = [], []
    for _ in range(rows):
        k = int(rng.integers(0, per_row + 1))
        cs = np.sort(rng.choice(cols, size=min(k, cols), replace=False)).astype(np.int32)
        ci.extend(cs.tolist())
        v.extend(rng.normal(size=len(cs)).tolist())
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v)


def mesh_arrays(mesh, out):
    out["elem_v"] = mesh.elem_v
    out["x"], out["y"], out["tag"] = mesh.x, mesh.y, mesh.tag.astype(np.int32)


def host_part():
    R = O.ref()
    for name in MESHES:
        mesh = F.make_mesh(name)
        out = {}
        mesh_arrays(mesh, out)
        n, ne = mesh.n, mesh.ne
        rp = np.zeros(n + 1, np.int32)
        nnz = R.ref_csr_build(n, ne, _p(mesh.elem_v), _p(mesh.x), _p(mesh.y), _p(mesh.tag), _p(rp), None)
        ci = np.zeros(nnz, np.int32)
        R.ref_csr_build(n, ne, _p(mesh.elem_v), _p(mesh.x), _p(mesh.y), _p(mesh.tag), _p(rp), _p(ci))
        out["rp"], out["ci"] = rp, ci
        u, v, p = step_inputs(mesh)
        out["u"], out["v"], out["p"] = u, v, p
        Kp = oracle_pressure_matrix(mesh, rp, ci, u, v, p)
        out["ppe_val"] = Kp
        amg_host(R, rp, ci, Kp, "ppe_", out)
        lap = shifted_laplacian(rp, ci)
        out["lap_val"] = lap
        amg_host(R, rp, ci, lap, "lap_", out)
        path = os.path.join(HERE, f"ref_host_{name}.npz")
        np.savez_compressed(path, **out)
        print(path, n, nnz, "levels", out["ppe_levels"][0], out["lap_levels"][0])
    # SpGEMM / transpose on random matrices
    rng = np.random.default_rng(5)
    out = {}
    for t in range(3):
        ar, ac, bc = int(rng.integers(20, 200)), int(rng.integers(20, 200)), int(rng.integers(5, 150))
        A = random_csr(rng, ar, ac, 9)
        B = random_csr(rng, ac, bc, 7)
        crp = np.zeros(ar + 1, np.int32)
        nnz = R.ref_csr_multiply(ar, ac, _p(A[0]), _p(A[1]), _p(A[2]), bc, _p(B[0]), _p(B[1]), _p(B[2]), _p(crp), None, None)
        cci, cv = np.zeros(nnz, np.int32), np.zeros(nnz)
        R.ref_csr_multiply(ar, ac, _p(A[0]), _p(A[1]), _p(A[2]), bc, _p(B[0]), _p(B[1]), _p(B[2]), _p(crp), _p(cci), _p(cv))
        trp, tci, tv = np.zeros(ac + 1, np.int32), np.zeros(A[1].size, np.int32), np.zeros(A[1].size)
        R.ref_csr_transpose(ar, ac, _p(A[0]), _p(A[1]), _p(A[2]), _p(trp), _p(tci), _p(tv))
        out[f"t{t}_dims"] = np.array([ar, ac, bc])
        for k, a in zip(("A_rp", "A_ci", "A_v", "B_rp", "B_ci", "B_v", "C_rp", "C_ci", "C_v", "T_rp", "T_ci", "T_v"),
                        (*A, *B, crp, cci, cv, trp, tci, tv)):
            out[f"t{t}_{k}"] = a
    path = os.path.join(HERE, "ref_host_spgemm.npz")
    np.savez_compressed(path, **out)
    print(path)


def gpu_part(outdir):
    R = O.ref()
    if not R.ref_gpu_available():
        raise SystemExit("no GPU")
    os.makedirs(outdir, exist_ok=True)
    for name in MESHES:
        host = np.load(os.path.join(HERE, f"ref_host_{name}.npz"))
        rp, ci = host["rp"], host["ci"]
        n, nnz = rp.size - 1, ci.size
        out = {}
        # MulticolourIlu0 on the test_momentum_ilu matrix; GpuBicgstab2 vs Jacobi BiCGSTAB
        a, b = momentum_ilu_matrix(rp, ci)
        out["ilu_val"], out["ilu_b"] = a, b
        colour = np.zeros(n, np.int32)
        cstart = np.zeros(65, np.int32)
        rows = np.zeros(n, np.int32)
        lu = np.zeros(nnz)
        z = np.zeros(2 * n)
        nc = R.ref_ilu(n, _p(rp), _p(ci), _p(a), _p(colour), _p(cstart), _p(rows), _p(lu), _p(b), _p(z), 2)
        out["ilu_colour"], out["ilu_colour_start"], out["ilu_rows"], out["ilu_lu"], out["ilu_z"] = \
            colour, cstart[: nc + 1].copy(), rows, lu, z
        xu, xv = np.zeros(n), np.zeros(n)
        info, rel = np.zeros(4, np.int32), np.zeros(2)
        R.ref_bicgstab2(n, _p(rp), _p(ci), _p(a), _p(b), _p(b[n:].copy()), _p(xu), _p(xv), 200, C.c_double(1e-10),
                        _p(info), _p(rel))
        out["b2_x"], out["b2_info"], out["b2_rel"] = np.concatenate([xu, xv]), info, rel
        xj = np.zeros(n)
        conv, relj = C.c_int(), C.c_double()
        it = R.ref_bicgstab(n, _p(rp), _p(ci), _p(a), _p(b), _p(xj), 400, C.c_double(1e-10), C.byref(conv), C.byref(relj))
        out["bj_x"], out["bj_info"] = xj, np.array([it, conv.value])
        # PCG + AMG on the shifted Laplacian; one V-cycle of sin(0.37 i) + 0.2 (test_amg_remap)
        lap = host["lap_val"]
        bl = np.cos(0.11 * np.arange(n))
        xl = np.zeros(n)
        r_v = np.sin(0.37 * np.arange(n)) + 0.2
        z_v = np.zeros(n)
        levels = C.c_int()
        it = R.ref_pcg(n, _p(rp), _p(ci), _p(lap), _p(bl), _p(xl), 400, C.c_double(1e-10), None, None, None, 1,
                       C.byref(conv), C.byref(relj), C.byref(levels), _p(r_v), _p(z_v))
        out["lap_pcg_x"], out["lap_pcg_info"], out["lap_vcycle_z"] = xl, np.array([it, conv.value, levels.value]), z_v
        # one step of the solve path (tol 1e-10)
        mesh_ev, x, y, tag = host["elem_v"], host["x"], host["y"], host["tag"]
        ne = mesh_ev.size // 3
        u, v, p = host["u"], host["v"], host["p"]
        h = C.c_void_p(R.ref_step_create(n, ne, _p(mesh_ev), _p(x), _p(y), _p(tag), _p(u), _p(v), _p(p),
                                         C.c_double(1e-3), C.c_double(1e-3), C.c_double(1.0), C.c_double(1.5),
                                         C.c_double(1.0), C.c_double(1e-3), C.c_double(0.3), C.c_double(1e-10),
                                         1000, 4000))
        R.ref_step_amg_setup(h)
        its, convs, rels = np.zeros(3, np.int32), np.zeros(3, np.int32), np.zeros(3)
        su, sv, sdp = np.zeros(n), np.zeros(n), np.zeros(n)
        R.ref_step_run(h, _p(its), _p(convs), _p(rels), _p(su), _p(sv), _p(sdp))
        sys_arrays = {k: np.zeros(sz) for k, sz in (("A_val", nnz), ("rhs_u", n), ("rhs_v", n), ("mass", n),
                                                     ("Kp_val", nnz), ("rhs_p", n), ("div_num", n), ("elem_s", ne),
                                                     ("gpx", n), ("gpy", n), ("oss_val", 4 * nnz), ("inv_m", n))}
        R.ref_step_systems(h, *[_p(sys_arrays[k]) for k in ("A_val", "rhs_u", "rhs_v", "mass", "Kp_val", "rhs_p",
                                                            "div_num", "elem_s", "gpx", "gpy", "oss_val", "inv_m")])
        R.ref_step_free(h)
        for k, val in sys_arrays.items():
            out["step_" + k] = val
        out["step_u"], out["step_v"], out["step_dp"] = su, sv, sdp
        out["step_its"], out["step_conv"], out["step_rel"] = its, convs, rels
        path = os.path.join(outdir, f"ref_gpu_{name}.npz")
        np.savez_compressed(path, **out)
        print(path, "colours", nc, "b2", info, "pcg", it, "step its", its)


if __name__ == "__main__":
    if sys.argv[1] == "host":
        host_part()
    else:
        gpu_part(sys.argv[2] if len(sys.argv) > 2 else HERE)
