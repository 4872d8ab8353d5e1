"""CPU emulation of the SA-AMG V-cycle with each level in FP64 or FP32, inside a flexible PCG.

TEST INFRASTRUCTURE ONLY (an analysis tool next to the oracle; never imported by the product).
It takes the oracle's hierarchy of a pressure system (the same one the parity tests build), runs
the V(2,2) cycle of the tiled kernels (pre-smoothing from a zero start, residual, restriction,
the levels below, the dense coarse inverse in FP64, prolongation, two post-smoothing sweeps) with
scipy in the chosen precision per level, and counts the PCG iterations to 1e-10 relative residual
for a precision schedule: all FP64, all FP32, one level in the other precision, and a switch from
one precision to the other at a relative residual. It is how the FP64 phase of mixed-precision
solves was chosen (the FP32 V-cycle's rounding costs iterations when it is made while the
residual is large, not when the residual is small).

    python -m oracle.vcycle_precision [mesh name, default c1]
"""
import sys

import numpy as np
import scipy.sparse as sp

from oracle import oracle as O


def pressure_system(m):
    """The pressure system of the parity tests: PPE with the OSS term, BCs applied."""
    import fixtures as F
    rp, ci = O.csr_build(m.n, m.elem_v)
    u, v, p = (F.fourier_field(m.x, m.y, 1), F.fourier_field(m.x, m.y, 2), 0.3 * F.fourier_field(m.x, m.y, 3))
    _, _, _, mass = O.assemble_momentum(m, rp, ci, u, v, u, v, p, O.bdf2_params())
    dt_proj = 2e-3 / 3
    s = O.oss_weights(m, u, v, dt_proj, 1.0, 1e-3, 0.3)
    gx, gy = O.scalar_gradient(m, p, s)
    Kp, rhs, _ = O.assemble_ppe(m, rp, ci, u, v, p, gx, gy, mass, s, dt_proj, 1.0, 0.3)
    O.apply_bc_pressure(m, rp, ci, Kp, rhs, np.zeros(m.n), mass)
    oss, inv_m = O.assemble_oss(m, rp, ci, s, mass)
    return rp, ci, Kp, rhs, oss, inv_m


class Hierarchy:
    """The oracle's SA-AMG levels as scipy matrices, castable per level."""

    def __init__(self, rp, ci, val):
        amg = O.Amg(rp, ci, val)
        self.levels = []
        for lv in range(amg.nlev):
            d = amg.level(lv)
            mats = {}
            for name in ("A", "P", "R"):
                r, c, mrp, mci, mv = d[name]
                mats[name] = sp.csr_matrix((mv, mci, mrp), shape=(r, c))
            self.levels.append(dict(mats, dinv=d["dinv"], omega=d["omega"]))
        _, self.coarse_inv = amg.coarse()

    def cast(self, dtypes):
        """Level dicts with values, D^-1 and omega in dtypes[l]."""
        out = []
        for lv, dt in zip(self.levels, dtypes):
            out.append(dict(A=lv["A"].astype(dt), P=lv["P"].astype(dt), R=lv["R"].astype(dt),
                            dinv=lv["dinv"].astype(dt), omega=dt(lv["omega"]), dt=dt))
        return out

    def vcycle(self, levels, l, b):
        lv = levels[l]
        b = b.astype(lv["dt"])
        A, dinv, om = lv["A"], lv["dinv"], lv["omega"]
        x = om * dinv * b
        x = x + om * dinv * (b - A @ x)
        r = b - A @ x
        bc = lv["R"] @ r
        if l + 1 < len(levels):
            xc = self.vcycle(levels, l + 1, bc)
        else:
            xc = self.coarse_inv @ bc.astype(np.float64)
        x = x + lv["P"] @ xc.astype(lv["dt"])
        for _ in range(2):
            x = x + om * dinv * (b - A @ x)
        return x


def pcg_iterations(h, op, b, first, second=None, switch=0.0, tol=1e-10, max_iter=500):
    """Flexible (Polak-Ribiere) PCG iterations with the V-cycle levels `first`, replaced by
    `second` once the relative residual is below `switch`; -1 when not converged."""
    x = np.zeros_like(b)
    r = b.copy()
    bn = np.linalg.norm(b)
    levels = first
    z = h.vcycle(levels, 0, r).astype(np.float64)
    p = z.copy()
    rz = r @ z
    for it in range(1, max_iter + 1):
        q = op(p)
        alpha = rz / (p @ q)
        x += alpha * p
        r -= alpha * q
        rn = np.linalg.norm(r)
        if rn < tol * bn:
            return it
        if second is not None and rn < switch * bn:
            levels, second = second, None
        zn = h.vcycle(levels, 0, r).astype(np.float64)
        beta = -alpha * (zn @ q) / rz
        rz = r @ zn
        p = zn + beta * p
    return -1


def main(name="c1"):
    import fixtures as F
    m = F.make_mesh(name)
    rp, ci, Kp, rhs, oss, inv_m = pressure_system(m)

    def op(x):
        y = O.spmv(rp, ci, Kp, x)
        O.oss_apply(m, rp, ci, oss, inv_m, x, y)
        return y

    h = Hierarchy(rp, ci, Kp)
    nl = len(h.levels)
    f64, f32 = np.float64, np.float32
    all64, all32 = h.cast([f64] * nl), h.cast([f32] * nl)
    rows = [("all FP64", all64, None, 0.0), ("all FP32", all32, None, 0.0),
            ("level 0 FP32", h.cast([f32] + [f64] * (nl - 1)), None, 0.0),
            ("coarsest level FP32", h.cast([f64] * (nl - 1) + [f32]), None, 0.0)]
    rows += [(f"FP32, FP64 below {sw:g}", all32, all64, sw) for sw in (1e-6, 1e-7, 1e-8)]
    rows += [(f"FP64, FP32 below {sw:g}", all64, all32, sw) for sw in (1e-1, 1e-2, 1e-3, 1e-4)]
    for label, first, second, sw in rows:
        print(f"{label}: {pcg_iterations(h, op, rhs, first, second, sw)} iterations", flush=True)


if __name__ == "__main__":
    import os
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "cylinder-fem-amr_b200"))
    main(sys.argv[1] if len(sys.argv) > 1 else "c1")
