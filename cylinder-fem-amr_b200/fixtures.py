"""Seeded synthetic meshes and fields for the solve path (inputs only, not the solver).

Domain: the rectangle [0, 4] x [0, 1] minus the disc of radius 0.1 centred at (0.5, 0.5).
The base mesh is a Delaunay triangulation (scipy) of seeded jittered points, graded from a
spacing of 0.01 on the circle to ``h`` away from it. It is then refined by newest-vertex
bisection (NVB) with edge-marking closure, which keeps the mesh conforming without hanging
nodes. Element storage follows the reference's ``Triangle`` (``src/cfa/mesh.cuh:8-12``):
``v[0]`` is the newest vertex, ``(v[1], v[2])`` the refinement edge, counter-clockwise.
One refinement "level" is two bisections, as in the reference (``src/cfa/amr.cuh:10``).

Nodes are numbered like the reference's ``AdaptiveMesh::extract`` (``src/cfa/amr.cuh:144-215``):
elements sorted along a Morton curve of their centroids, vertices by first use, so neighbouring
unknowns stay close in memory.

Boundary tags are the reference's ``BoundaryTag`` (``src/cfa/common.cuh:68-74``): inlet x = 0,
walls y = 0 and y = 1, outlet x = 4, cylinder on the circle (midpoints snapped to the arc).
"""
from __future__ import annotations

import dataclasses

import numpy as np

BC_INTERIOR, BC_INLET, BC_OUTLET, BC_WALL, BC_CYLINDER = 0, 1, 2, 3, 4
LX, LY = 4.0, 1.0
XC, YC, RC = 0.5, 0.5, 0.1
_KEY = np.int64(1) << np.int64(32)


@dataclasses.dataclass
class Mesh:
    x: np.ndarray        # float64 [n]
    y: np.ndarray        # float64 [n]
    tag: np.ndarray      # int32 [n]
    tri: np.ndarray      # int32 [ne, 3]; v0 newest vertex, (v1, v2) refinement edge, CCW
    gen: np.ndarray      # int32 [ne]; bisections since the base mesh

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def ne(self) -> int:
        return int(self.tri.shape[0])

    @property
    def elem_v(self) -> np.ndarray:
        return np.ascontiguousarray(self.tri.reshape(-1), dtype=np.int32)


# ----------------------------------------------------------------------------------------------
# base mesh
# ----------------------------------------------------------------------------------------------
def _classify(px: np.ndarray, py: np.ndarray) -> np.ndarray:
    """Tag of boundary points by exact position (same precedence as ``classify_boundary_node``,
    ``src/cfa/mesh.cuh:62-70``: cylinder, wall, inlet, outlet)."""
    t = np.full(px.shape, BC_INTERIOR, np.int32)
    t[px == LX] = BC_OUTLET
    t[px == 0.0] = BC_INLET
    t[(py == 0.0) | (py == LY)] = BC_WALL
    return t


def base_mesh(h: float = 0.05, h_circle: float = 0.01, grade: float = 0.3, seed: int = 0) -> Mesh:
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    nx, ny = int(round(LX / h)), int(round(LY / h))
    xs, ys = np.linspace(0.0, LX, nx + 1), np.linspace(0.0, LY, ny + 1)
    bpts = np.concatenate([
        np.stack([xs, np.zeros_like(xs)], 1),
        np.stack([xs, np.full_like(xs, LY)], 1),
        np.stack([np.zeros(ny - 1), ys[1:-1]], 1),
        np.stack([np.full(ny - 1, LX), ys[1:-1]], 1),
    ])
    btag = _classify(bpts[:, 0], bpts[:, 1])

    def spacing(r):
        return h_circle + (h - h_circle) * np.clip((r - RC) / grade, 0.0, 1.0)

    # circle and graded rings around it
    ring_pts = []
    r, k = RC, 0
    while True:
        s = spacing(r)
        m = max(8, int(round(2.0 * np.pi * r / s)))
        off = 0.5 * (k % 2)
        th = 2.0 * np.pi * (np.arange(m) + off) / m
        ring_pts.append(np.stack([XC + r * np.cos(th), YC + r * np.sin(th)], 1))
        if s >= 0.98 * h or r + 0.866 * s + s > 0.5 - 0.5 * h:
            break
        r += 0.866 * s
        k += 1
    r_last = r
    cpts = ring_pts[0]
    rpts = np.concatenate(ring_pts[1:]) if len(ring_pts) > 1 else np.zeros((0, 2))

    # jittered interior grid outside the rings
    gx, gy = np.meshgrid(np.arange(h, LX - 0.5 * h, h), np.arange(h, LY - 0.5 * h, h))
    g = np.stack([gx.ravel(), gy.ravel()], 1)
    g += rng.uniform(-0.15 * h, 0.15 * h, size=g.shape)
    d = np.hypot(g[:, 0] - XC, g[:, 1] - YC)
    g = g[d > r_last + 0.7 * h]
    inside = (g[:, 0] > 0.5 * h) & (g[:, 0] < LX - 0.5 * h) & (g[:, 1] > 0.5 * h) & (g[:, 1] < LY - 0.5 * h)
    g = g[inside]

    pts = np.concatenate([bpts, cpts, rpts, g])
    tag = np.concatenate([btag, np.full(len(cpts), BC_CYLINDER, np.int32),
                          np.zeros(len(rpts) + len(g), np.int32)])
    tri = Delaunay(pts).simplices.astype(np.int64)
    cx = pts[tri, 0].mean(1)
    cy = pts[tri, 1].mean(1)
    tri = tri[np.hypot(cx - XC, cy - YC) > RC]
    x0, y0 = pts[tri[:, 0], 0], pts[tri[:, 0], 1]
    x1, y1 = pts[tri[:, 1], 0], pts[tri[:, 1], 1]
    x2, y2 = pts[tri[:, 2], 0], pts[tri[:, 2], 1]
    det = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0)
    tri = tri[np.abs(det) > 1e-14]
    det = det[np.abs(det) > 1e-14]
    neg = det < 0
    tri[neg] = tri[neg][:, [0, 2, 1]]
    # NVB label: newest vertex opposite the longest edge
    p = pts[tri]
    l0 = np.sum((p[:, 1] - p[:, 2]) ** 2, 1)
    l1 = np.sum((p[:, 2] - p[:, 0]) ** 2, 1)
    l2 = np.sum((p[:, 0] - p[:, 1]) ** 2, 1)
    lm = np.argmax(np.stack([l0, l1, l2], 1), 1)
    rot = np.stack([lm, (lm + 1) % 3, (lm + 2) % 3], 1)
    tri = np.take_along_axis(tri, rot, 1)
    used = np.zeros(len(pts), bool)
    used[tri.ravel()] = True
    remap = np.cumsum(used) - 1
    mesh = Mesh(pts[used, 0].copy(), pts[used, 1].copy(), tag[used].copy(),
                remap[tri].astype(np.int32), np.zeros(len(tri), np.int32))
    return renumber(mesh)


# ----------------------------------------------------------------------------------------------
# newest-vertex bisection
# ----------------------------------------------------------------------------------------------
def _edge_keys(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    lo = np.minimum(a, b).astype(np.int64)
    hi = np.maximum(a, b).astype(np.int64)
    return lo * _KEY + hi


def nvb_round(mesh: Mesh, mark: np.ndarray) -> Mesh:
    """One bisection round: the refinement edges of the marked elements are marked, the marks
    are closed (an element with any marked edge gets its refinement edge marked), and every
    element is bisected along its marked edges (at most twice per round)."""
    tri = mesh.tri.astype(np.int64)
    ne, n = tri.shape[0], mesh.n
    key = _edge_keys(tri[:, [1, 2, 0]], tri[:, [2, 0, 1]])      # e0 = (v1, v2): refinement edge
    ukey, inv, cnt = np.unique(key.ravel(), return_inverse=True, return_counts=True)
    eid = inv.reshape(ne, 3)
    emark = np.zeros(len(ukey), bool)
    emark[eid[mark, 0]] = True
    while True:
        need = emark[eid].any(1) & ~emark[eid[:, 0]]
        if not need.any():
            break
        emark[eid[need, 0]] = True
    me = np.nonzero(emark)[0]
    a = (ukey[me] // _KEY).astype(np.int64)
    b = (ukey[me] % _KEY).astype(np.int64)
    mx = 0.5 * (mesh.x[a] + mesh.x[b])
    my = 0.5 * (mesh.y[a] + mesh.y[b])
    bnd = cnt[me] == 1
    cyl = bnd & (mesh.tag[a] == BC_CYLINDER) & (mesh.tag[b] == BC_CYLINDER)
    if cyl.any():
        dx, dy = mx[cyl] - XC, my[cyl] - YC
        rr = np.hypot(dx, dy)
        mx[cyl] = XC + RC * dx / rr
        my[cyl] = YC + RC * dy / rr
    mtag = np.where(bnd, _classify(mx, my), BC_INTERIOR).astype(np.int32)
    mtag[cyl] = BC_CYLINDER
    newid = np.full(len(ukey), -1, np.int64)
    newid[me] = n + np.arange(len(me))

    out_t, out_g = [], []
    cur, cg = tri, mesh.gen.astype(np.int32)
    for _ in range(3):
        k0 = _edge_keys(cur[:, 1], cur[:, 2])
        pos = np.minimum(np.searchsorted(ukey, k0), len(ukey) - 1)
        sel = (ukey[pos] == k0) & emark[pos]
        out_t.append(cur[~sel])
        out_g.append(cg[~sel])
        s, sg = cur[sel], cg[sel]
        if len(s) == 0:
            cur = s
            break
        m = newid[pos[sel]]
        c1 = np.stack([m, s[:, 0], s[:, 1]], 1)
        c2 = np.stack([m, s[:, 2], s[:, 0]], 1)
        cur = np.concatenate([c1, c2])
        cg = np.concatenate([sg + 1, sg + 1])
    assert len(cur) == 0, "NVB round left marked edges"
    return Mesh(np.concatenate([mesh.x, mx]), np.concatenate([mesh.y, my]),
                np.concatenate([mesh.tag, mtag]), np.concatenate(out_t).astype(np.int32),
                np.concatenate(out_g).astype(np.int32))


def _spread_bits(v: np.ndarray) -> np.ndarray:
    v = v.astype(np.uint32)
    v = (v | (v << 8)) & np.uint32(0x00FF00FF)
    v = (v | (v << 4)) & np.uint32(0x0F0F0F0F)
    v = (v | (v << 2)) & np.uint32(0x33333333)
    v = (v | (v << 1)) & np.uint32(0x55555555)
    return v


def renumber(mesh: Mesh) -> Mesh:
    """Elements along a Morton curve of their centroids (ties by index), vertices by first use."""
    t = mesh.tri
    cx = (mesh.x[t[:, 0]] + mesh.x[t[:, 1]] + mesh.x[t[:, 2]]) / 3.0
    cy = (mesh.y[t[:, 0]] + mesh.y[t[:, 1]] + mesh.y[t[:, 2]]) / 3.0
    qx = np.clip(cx / LX * 65535.0, 0, 65535).astype(np.uint32)
    qy = np.clip(cy / LY * 65535.0, 0, 65535).astype(np.uint32)
    code = _spread_bits(qx) | (_spread_bits(qy) << np.uint32(1))
    order = np.lexsort((np.arange(len(t)), code))
    t = t[order]
    flat = t.ravel()
    first = np.full(mesh.n, np.iinfo(np.int64).max, np.int64)
    np.minimum.at(first, flat, np.arange(len(flat)))
    vorder = np.argsort(first, kind="stable")
    vorder = vorder[first[vorder] < np.iinfo(np.int64).max]
    compact = np.full(mesh.n, -1, np.int64)
    compact[vorder] = np.arange(len(vorder))
    return Mesh(mesh.x[vorder].copy(), mesh.y[vorder].copy(), mesh.tag[vorder].copy(),
                compact[t].astype(np.int32), mesh.gen[order].copy())


def refine_uniform(mesh: Mesh, bisections: int) -> Mesh:
    for _ in range(bisections):
        mesh = nvb_round(mesh, np.ones(mesh.ne, bool))
    return mesh


def refine_region(mesh: Mesh, max_gen: int, radius: float = 0.3, band=(0.4, 0.6), x_min: float = 0.5) -> Mesh:
    """NVB up to ``max_gen`` bisections inside ``radius`` of the disc centre and in the wake band."""
    while True:
        t = mesh.tri
        cx = (mesh.x[t[:, 0]] + mesh.x[t[:, 1]] + mesh.x[t[:, 2]]) / 3.0
        cy = (mesh.y[t[:, 0]] + mesh.y[t[:, 1]] + mesh.y[t[:, 2]]) / 3.0
        region = (np.hypot(cx - XC, cy - YC) < radius) | ((cy > band[0]) & (cy < band[1]) & (cx > x_min))
        mark = region & (mesh.gen < max_gen)
        if not mark.any():
            return mesh
        mesh = nvb_round(mesh, mark)


def refine_blob(mesh: Mesh, centre=(1.0, 0.3), radius: float = 0.05, rounds: int = 2):
    """One remesh of an adaptive run: ``rounds`` NVB rounds on the elements whose centroid lies
    within ``radius`` of ``centre``, then renumbered. Returns the new mesh and new_to_old, the old
    index of every kept node (-1 for a new node), matched by exact coordinates as the reference's
    remap test does (tests/test_cfa.cu:395-401)."""
    old = mesh
    for _ in range(rounds):
        t = mesh.tri
        cx = (mesh.x[t[:, 0]] + mesh.x[t[:, 1]] + mesh.x[t[:, 2]]) / 3.0
        cy = (mesh.y[t[:, 0]] + mesh.y[t[:, 1]] + mesh.y[t[:, 2]]) / 3.0
        mesh = nvb_round(mesh, np.hypot(cx - centre[0], cy - centre[1]) < radius)
    mesh = renumber(mesh)
    index = {xy: i for i, xy in enumerate(zip(old.x.tolist(), old.y.tolist()))}
    new_to_old = np.array([index.get(xy, -1) for xy in zip(mesh.x.tolist(), mesh.y.tolist())], np.int32)
    return mesh, new_to_old


# ----------------------------------------------------------------------------------------------
# named workloads
# ----------------------------------------------------------------------------------------------
CONFIGS = {
    # ~25k vertices, uniform
    "c0": dict(h=0.05, uniform=3, region_gen=0),
    # ~400k vertices, adaptive: uniform 2 levels, then up to 4.5 levels near the disc and in the wake
    "c1": dict(h=0.06, uniform=4, region_gen=9),
    # ~4M vertices, uniform
    "c2": dict(h=0.045, uniform=10, region_gen=0),
    # small cases for CPU tests
    "tiny": dict(h=0.2, uniform=0, region_gen=0),
    "small": dict(h=0.1, uniform=2, region_gen=0),
    "medium": dict(h=0.08, uniform=4, region_gen=6),
}


def make_mesh(name: str = "c0", seed: int = 0) -> Mesh:
    cfg = CONFIGS[name]
    m = base_mesh(h=cfg["h"], seed=seed)
    m = refine_uniform(m, cfg["uniform"])
    if cfg["region_gen"] > cfg["uniform"]:
        m = refine_region(m, cfg["region_gen"])
    return renumber(m)


def fourier_field(x: np.ndarray, y: np.ndarray, seed: int, modes: int = 8, kmax: float = 2 * np.pi * 4,
                  amplitude: float = 1.0) -> np.ndarray:
    """Sum of ``modes`` random Fourier modes a_k sin(k . x + phi_k), |k| <= kmax, seeded."""
    rng = np.random.default_rng(seed)
    k = rng.uniform(-kmax, kmax, size=(modes, 2))
    nk = np.hypot(k[:, 0], k[:, 1])
    k = k * np.minimum(1.0, kmax / np.maximum(nk, 1e-30))[:, None]
    ph = rng.uniform(0.0, 2 * np.pi, size=modes)
    a = rng.uniform(-1.0, 1.0, size=modes)
    a *= amplitude / np.sum(np.abs(a))
    return (a[None, :] * np.sin(x[:, None] * k[None, :, 0] + y[:, None] * k[None, :, 1] + ph[None, :])).sum(1)


def validate(mesh: Mesh) -> dict:
    """Conformity checks (cf. ``validate_mesh``, ``src/cfa/mesh.cuh:302-376``): positive areas,
    every edge in at most two elements, single-element edges on the physical boundary."""
    t = mesh.tri.astype(np.int64)
    x, y = mesh.x, mesh.y
    det = (x[t[:, 1]] - x[t[:, 0]]) * (y[t[:, 2]] - y[t[:, 0]]) - (x[t[:, 2]] - x[t[:, 0]]) * (y[t[:, 1]] - y[t[:, 0]])
    key = _edge_keys(t[:, [1, 2, 0]], t[:, [2, 0, 1]]).ravel()
    ukey, cnt = np.unique(key, return_counts=True)
    a, b = ukey // _KEY, ukey % _KEY
    single = cnt == 1
    bad_bnd = single & ((mesh.tag[a] == BC_INTERIOR) | (mesh.tag[b] == BC_INTERIOR))
    # minimum angle
    p = np.stack([x[t], y[t]], -1)
    ang = []
    for k in range(3):
        u = p[:, (k + 1) % 3] - p[:, k]
        w = p[:, (k + 2) % 3] - p[:, k]
        c = (u * w).sum(1) / np.sqrt((u * u).sum(1) * (w * w).sum(1))
        ang.append(np.degrees(np.arccos(np.clip(c, -1, 1))))
    return dict(n=mesh.n, ne=mesh.ne, min_area=float(0.5 * det.min()), max_count=int(cnt.max()),
                bad_boundary_edges=int(bad_bnd.sum()), min_angle=float(np.min(ang)),
                area=float(0.5 * det.sum()))
