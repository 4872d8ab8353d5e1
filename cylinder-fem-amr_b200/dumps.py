"""The reference driver's ``--dump-systems`` files (src/cylinder_fem_amr.cu:332-352, :426-438): the
momentum and pressure systems of one step, as the reference's solver benches read them
(scripts/momentum_study/mb.cu:42-47). Little-endian, no padding:

  <prefix>_momentum.bin: int32 n, nnz; row_ptr int32[n+1]; col_ind int32[nnz]; val f64[nnz];
                         rhs_u, rhs_v, u0, v0, x, y f64[n] each; bc_tag int32[n];
                         then the solutions u, v f64[n] each (appended after the solves)
  <prefix>_pressure.bin: int32 n, nnz; row_ptr int32[n+1]; col_ind int32[nnz]; val f64[nnz];
                         rhs f64[n]; initial guess f64[n]   (the OSS term is not included)
"""
from __future__ import annotations

import numpy as np

_MOM_VECS = ("rhs_u", "rhs_v", "u0", "v0", "x", "y")


def _csr(f, n, nnz):
    rp = np.fromfile(f, "<i4", n + 1)
    ci = np.fromfile(f, "<i4", nnz)
    val = np.fromfile(f, "<f8", nnz)
    if rp.size != n + 1 or ci.size != nnz or val.size != nnz:
        raise ValueError("truncated system dump")
    return rp, ci, val


def read_momentum(path: str) -> dict:
    with open(path, "rb") as f:
        n, nnz = (int(v) for v in np.fromfile(f, "<i4", 2))
        rp, ci, val = _csr(f, n, nnz)
        out = dict(n=n, nnz=nnz, row_ptr=rp, col_ind=ci, val=val)
        for k in _MOM_VECS:
            out[k] = np.fromfile(f, "<f8", n)
            if out[k].size != n:
                raise ValueError("truncated momentum dump")
        out["bc_tag"] = np.fromfile(f, "<i4", n)
        sol = np.fromfile(f, "<f8", 2 * n)
        if sol.size == 2 * n:
            out["u"], out["v"] = sol[:n], sol[n:]
    return out


def write_momentum(path: str, row_ptr, col_ind, val, rhs_u, rhs_v, u0, v0, x, y, bc_tag, u=None, v=None) -> None:
    n, nnz = len(row_ptr) - 1, len(col_ind)
    with open(path, "wb") as f:
        np.asarray([n, nnz], "<i4").tofile(f)
        np.asarray(row_ptr, "<i4").tofile(f)
        np.asarray(col_ind, "<i4").tofile(f)
        np.asarray(val, "<f8").tofile(f)
        for a in (rhs_u, rhs_v, u0, v0, x, y):
            np.asarray(a, "<f8").tofile(f)
        np.asarray(bc_tag, "<i4").tofile(f)
        if u is not None:
            np.asarray(u, "<f8").tofile(f)
            np.asarray(v, "<f8").tofile(f)


def read_pressure(path: str) -> dict:
    with open(path, "rb") as f:
        n, nnz = (int(v) for v in np.fromfile(f, "<i4", 2))
        rp, ci, val = _csr(f, n, nnz)
        rhs = np.fromfile(f, "<f8", n)
        x0 = np.fromfile(f, "<f8", n)
        if rhs.size != n or x0.size != n:
            raise ValueError("truncated pressure dump")
    return dict(n=n, nnz=nnz, row_ptr=rp, col_ind=ci, val=val, rhs=rhs, x0=x0)


def write_pressure(path: str, row_ptr, col_ind, val, rhs, x0) -> None:
    n, nnz = len(row_ptr) - 1, len(col_ind)
    with open(path, "wb") as f:
        np.asarray([n, nnz], "<i4").tofile(f)
        np.asarray(row_ptr, "<i4").tofile(f)
        np.asarray(col_ind, "<i4").tofile(f)
        np.asarray(val, "<f8").tofile(f)
        np.asarray(rhs, "<f8").tofile(f)
        np.asarray(x0, "<f8").tofile(f)


def solve_momentum(d: dict, precision=None, tol: float = 1e-7, max_iter: int = 150, ctx=None):
    """The dumped momentum system through the device BiCGSTAB2 + MC-ILU(0) (what mb.cu times):
    returns (u, v, iterations)."""
    import torch
    import cfa_b200 as cfa
    ctx = ctx or cfa.default_context()
    precision = cfa.FP64 if precision is None else precision
    t = lambda a, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    rp, ci = t(d["row_ptr"], torch.int32), t(d["col_ind"], torch.int32)
    ilu = cfa.MulticolourIlu0(ctx, precision)
    ilu.set_pattern(d["n"], d["row_ptr"], d["col_ind"], rp, ci)
    A = t(d["val"])
    ilu.factor(A)
    u, v = t(d["u0"]), t(d["v0"])
    s = cfa.GpuBicgstab2(ctx)
    s.solve(d["n"], rp, ci, A, t(d["rhs_u"]), t(d["rhs_v"]), u, v, max_iter, tol, ilu)
    return u.cpu().numpy(), v.cpu().numpy(), (s.iters[0], s.iters[1])


def solve_pressure(d: dict, tol: float = 1e-7, max_iter: int = 4000, precision=None, ctx=None):
    """The dumped pressure system (without its OSS term, which the dump does not hold) through the
    device SA-AMG PCG: returns (x, iterations)."""
    import torch
    import cfa_b200 as cfa
    ctx = ctx or cfa.default_context()
    precision = cfa.FP64 if precision is None else precision
    t = lambda a, dt=torch.float64: torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dt)
    rp, ci, A = t(d["row_ptr"], torch.int32), t(d["col_ind"], torch.int32), t(d["val"])
    amg = cfa.AmgPreconditioner(ctx, precision)
    amg.setup(d["n"], d["nnz"], rp, ci, A)
    x = t(d["x0"])
    s = cfa.GpuLinearSolver(ctx)
    it = s.solve_pcg(d["n"], rp, ci, A, t(d["rhs"]), x, max_iter, tol, None, amg)
    return x.cpu().numpy(), it
