"""Seeded synthetic FETD models in the reference's input format.

Graded tensor-product hexahedral grids split into six Kuhn tetrahedra per hex
(conforming, all tets positively oriented in the reference's convention
V = det[1 x y z]/6 > 0, src/FETD_UTILITY.f90:105-112).  The reference's
coordinate convention is kept: z > 0 is earth (physical tags 12, 13, ...),
z < 0 is air (tag 11), as in LINUX/mod_big_sig_0.001.geo.  Transmitter loops
follow grid edges (a staircase for circles) and are written as ``Edges`` with
physical tag 51, vertices renumbered so that the loop runs through
increasing vertex numbers and closes on the first one -- exactly the
orientation the reference's ``src_drc`` convention assumes
(src/FETD_FWD.f90:446-448).  Receivers are nudged off the Kuhn-tet faces so
point location is unambiguous.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

from .meshio import Control, Mesh

AIR, EARTH = 11, 12


def graded_axis(required: Sequence[float], core: Tuple[float, float], h_core: float, half: float,
                ratio: float, h_min: Optional[float] = None) -> np.ndarray:
    """Grid lines on [-half, half]: all `required` lines, spacing <= h_core
    inside `core`, geometric growth by `ratio` outside it."""
    lo, hi = core
    pts = set(float(x) for x in required)
    pts.update([lo, hi, -half, half])
    # core: fill gaps larger than h_core
    core_pts = sorted(p for p in pts if lo <= p <= hi)
    fill = []
    for a, b in zip(core_pts[:-1], core_pts[1:]):
        k = int(np.ceil((b - a) / h_core - 1e-9))
        fill.extend(a + (b - a) * np.arange(1, k) / k)
    pts.update(fill)
    # growth outside the core
    h = h_core
    x = hi
    while True:
        h *= ratio
        x += h
        if x >= half - 0.5 * h:
            break
        pts.add(x)
    h = h_core
    x = lo
    while True:
        h *= ratio
        x -= h
        if x <= -half + 0.5 * h:
            break
        pts.add(x)
    out = np.array(sorted(p for p in pts if -half <= p <= half))
    # merge lines closer than h_min (keep required ones)
    if h_min:
        keep = [out[0]]
        req = set(float(r) for r in required)
        for p in out[1:]:
            if p - keep[-1] < h_min and p not in req and p != half:
                continue
            keep.append(p)
        out = np.array(keep)
    return out


# Kuhn subdivision of the unit cube: tets p -> p+e_a -> p+e_a+e_b -> p+1
_KUHN = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]


@dataclass
class Grid:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray

    @property
    def shape(self):
        return len(self.x), len(self.y), len(self.z)

    def node(self, i, j, k):
        nx, ny, nz = self.shape
        return (np.asarray(k) * ny + np.asarray(j)) * nx + np.asarray(i)


def hex_to_tets(g: Grid, cell_phys) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Nodes (0-based ids), tets (T,4) 0-based, per-tet physical tag.
    ``cell_phys(xc, yc, zc)`` gives the tag of each hex from its centre."""
    nx, ny, nz = g.shape
    X, Y, Z = np.meshgrid(g.x, g.y, g.z, indexing="ij")
    nod = np.stack([X.transpose(2, 1, 0).ravel(), Y.transpose(2, 1, 0).ravel(), Z.transpose(2, 1, 0).ravel()], axis=1)
    I, J, K = np.meshgrid(np.arange(nx - 1), np.arange(ny - 1), np.arange(nz - 1), indexing="ij")
    I, J, K = I.ravel(), J.ravel(), K.ravel()
    xc = 0.5 * (g.x[I] + g.x[I + 1]); yc = 0.5 * (g.y[J] + g.y[J + 1]); zc = 0.5 * (g.z[K] + g.z[K + 1])
    phys = np.asarray(cell_phys(xc, yc, zc))
    tets, tph = [], []
    for perm in _KUHN:
        off = np.zeros((len(I), 3), dtype=np.int64)
        verts = [g.node(I, J, K)]
        for ax in perm:
            off[:, ax] += 1
            verts.append(g.node(I + off[:, 0], J + off[:, 1], K + off[:, 2]))
        t = np.stack(verts, axis=1)
        tets.append(t)
        tph.append(phys)
    tets = np.concatenate(tets)
    tph = np.concatenate(tph)
    # orientation: make det[1 x y z] > 0
    P = nod[tets]
    d = np.einsum("ti,ti->t", P[:, 1] - P[:, 0], np.cross(P[:, 2] - P[:, 0], P[:, 3] - P[:, 0]))
    neg = d < 0
    tets[neg, 0], tets[neg, 1] = tets[neg, 1].copy(), tets[neg, 0].copy()
    return nod, tets, tph


def staircase_loop(g: Grid, z_index: int, inside) -> List[int]:
    """Closed loop of grid nodes (0-based) bounding the union of surface cells
    (i,j) whose centre satisfies inside(xc, yc); counter-clockwise in (x,y)."""
    nx, ny, _ = g.shape
    xc = 0.5 * (g.x[:-1] + g.x[1:]); yc = 0.5 * (g.y[:-1] + g.y[1:])
    M = inside(xc[:, None], yc[None, :])
    # directed boundary edges of the marked region (counter-clockwise)
    nxt = {}
    for i in range(nx - 1):
        for j in range(ny - 1):
            if not M[i, j]:
                continue
            if j == 0 or not M[i, j - 1]:
                nxt[(i, j)] = (i + 1, j)          # bottom edge, left->right
            if i == nx - 2 or not M[i + 1, j]:
                nxt[(i + 1, j)] = (i + 1, j + 1)  # right edge, up
            if j == ny - 2 or not M[i, j + 1]:
                nxt[(i + 1, j + 1)] = (i, j + 1)  # top edge, right->left
            if i == 0 or not M[i - 1, j]:
                nxt[(i, j + 1)] = (i, j)          # left edge, down
    if not nxt:
        raise ValueError("empty loop")
    start = min(nxt)
    loop = [start]
    cur = nxt[start]
    while cur != start:
        loop.append(cur)
        cur = nxt[cur]
        if len(loop) > len(nxt) + 1:
            raise ValueError("loop region is not simply connected")
    if len(loop) != len(nxt):
        raise ValueError("loop region is not simply connected")
    return [int(g.node(i, j, z_index)) for (i, j) in loop]


@dataclass
class Model:
    mesh: Mesh
    ctl: Control
    loops: List[List[int]]          # per RHS column: loop vertices (1-based, traversal order)
    receivers: np.ndarray           # (R,3)
    rec_rhs: np.ndarray             # RHS column of each receiver
    info: dict = field(default_factory=dict)

    def source_columns(self, edg_vex: np.ndarray):
        """(src_edg, src_drc) per RHS column from the loop vertex lists, with
        +1 when the traversal runs from the lower to the higher vertex number."""
        key = edg_vex[:, 0].astype(np.int64) * (1 << 32) + edg_vex[:, 1]
        cols = []
        for lp in self.loops:
            a = np.asarray(lp, dtype=np.int64)
            b = np.roll(a, -1)
            lo, hi = np.minimum(a, b), np.maximum(a, b)
            pos = np.searchsorted(key, lo * (1 << 32) + hi)
            cols.append(((pos + 1).astype(np.int32), np.where(a < b, 1, -1).astype(np.int32)))
        return cols


def _renumber_loop_first(nod, tets, loop0):
    """Renumber nodes so loop vertices come first in traversal order (1-based ids returned)."""
    N = len(nod)
    on_loop = set(loop0)
    order = list(loop0) + [v for v in range(N) if v not in on_loop]
    new = np.empty(N, dtype=np.int64)
    new[np.asarray(order)] = np.arange(N)
    return nod[np.asarray(order)], new[tets] + 1, new


def _nudge(p, g: Grid):
    """Move a receiver (by at most a few percent of its cell) off the grid planes
    and off the Kuhn planes u_a = u_b of its cell, so that exactly one tet holds it."""
    p = np.array(p, dtype=float)
    lo, hs, us = [], [], []
    for ax, lines in enumerate((g.x, g.y, g.z)):
        k = int(np.clip(np.searchsorted(lines, p[ax], side="right") - 1, 0, len(lines) - 2))
        h = lines[k + 1] - lines[k]
        lo.append(lines[k]); hs.append(h)
        us.append(float(np.clip((p[ax] - lines[k]) / h, 0.08, 0.92)))
    for _ in range(3):
        for a in range(3):
            for b in range(a + 1, 3):
                if abs(us[a] - us[b]) < 0.04:
                    us[b] = us[b] + 0.05 if us[b] < 0.85 else us[b] - 0.05
    return np.array([lo[a] + hs[a] * us[a] for a in range(3)])


def build_model(kind: str = "halfspace", seed: int = 0, scale: float = 1.0, **kw) -> Model:
    """Seeded synthetic models.

    kind:
      "halfspace" -- homogeneous earth under air, circular (staircase) loop on
                     the surface, one central receiver (the plain single-RHS case);
      "block"     -- conductive block in a host, square loop, receivers on a line;
      "multiloop" -- the block model with an nx*ny grid of small square loops,
                     one RHS column and one central receiver each;
      "ellipsoids" -- a 0.005 S/m host with 4 random ellipsoidal conductors
                     (0.05-1 S/m, semi-axes 50-300 m, centres 50-400 m deep)
                     under a 16 x 16 grid of 50 m loops at 40 m spacing, one
                     RHS column and one central receiver each;
      "layered"   -- a 1-D layered earth (3-6 layers, conductivities
                     log-uniform in [1e-4, 1e-1] S/m, thicknesses log-uniform
                     in [10, 300] m, all drawn from the seed) under air, a
                     square loop on the surface and one central receiver.
    ``scale`` multiplies the number of grid lines in the core (mesh size).
    """
    rng = np.random.default_rng(seed)
    half = kw.get("half", 50000.0)
    sig_air = kw.get("sig_air", 1e-12)
    if kind == "halfspace":
        R = kw.get("radius", 500.0)
        h = kw.get("h_core", 100.0) / scale
        sig = kw.get("sigma", 1e-3)
        xs = graded_axis([-R, R], (-R - h, R + h), h, half, kw.get("ratio", 1.6))
        ys = xs.copy()
        hz = kw.get("h_z", 20.0) / scale
        zs = graded_axis([0.0], (-2 * hz, kw.get("z_core", 200.0)), hz, half, kw.get("ratio", 1.6))
        g = Grid(xs, ys, zs)
        nod, tets, tph = hex_to_tets(g, lambda x, y, z: np.where(z > 0, EARTH, AIR))
        kz = int(np.searchsorted(zs, 0.0))
        loop = staircase_loop(g, kz, lambda x, y: x * x + y * y <= R * R)
        rec = [_nudge(kw.get("receiver", (0.0, 0.0, 3.0)), g)]
        domains = [(AIR, sig_air, 1.0, 1.0), (EARTH, sig, 1.0, 1.0)]
        loops0 = [loop]
        rec_rhs = [0]
    elif kind in ("block", "multiloop"):
        host, blk = kw.get("sigma", 0.01), kw.get("sigma_block", 0.1)
        bx, bz = kw.get("block_xy", 100.0), (kw.get("block_top", 100.0), kw.get("block_top", 100.0) + kw.get("block_h", 100.0))
        h = kw.get("h_core", 40.0) / scale
        req = [-bx, bx]
        # the large square loop (block) and the grid of small loops (multiloop);
        # with shared_grid both kinds carry the lines of both, so that they
        # build the same mesh and differ only in sources and receivers
        shared = kw.get("shared_grid", False)
        a_big = kw.get("big_loop_half", 500.0) if shared else kw.get("loop_half", 500.0)
        n_l = kw.get("n_loops", 8)
        sp_ = kw.get("loop_spacing", 40.0)
        a_small = kw.get("small_loop_half", 25.0) if shared else kw.get("loop_half", 25.0)
        centers = (np.arange(n_l) - (n_l - 1) / 2.0) * sp_
        if kind == "block" or shared:
            req += [-a_big, a_big]
            core = (-a_big - 2 * h, a_big + 2 * h)
        if kind == "multiloop" or shared:
            req += list(centers - a_small) + list(centers + a_small)
            if not shared:
                core = (min(centers) - a_small - 2 * h, max(centers) + a_small + 2 * h)
        xs = graded_axis(req, core, h, half, kw.get("ratio", 1.5), h_min=kw.get("h_min", 4.0))
        ys = xs.copy()
        hz = kw.get("h_z", 20.0) / scale
        zs = graded_axis([0.0, bz[0], bz[1]], (-2 * hz, bz[1] + 2 * hz), hz, half, kw.get("ratio", 1.5))
        g = Grid(xs, ys, zs)

        def phys(x, y, z):
            p = np.where(z > 0, EARTH, AIR)
            inb = (np.abs(x) < bx) & (np.abs(y) < bx) & (z > bz[0]) & (z < bz[1])
            return np.where(inb, EARTH + 1, p)

        nod, tets, tph = hex_to_tets(g, phys)
        kz = int(np.searchsorted(zs, 0.0))
        domains = [(AIR, sig_air, 1.0, 1.0), (EARTH, host, 1.0, 1.0), (EARTH + 1, blk, 1.0, 1.0)]
        mesh_loop = None
        if kind == "block" or shared:
            mesh_loop = staircase_loop(g, kz, lambda x, y: (np.abs(x) < a_big) & (np.abs(y) < a_big))
        if kind == "block":
            loops0 = [mesh_loop]
            nrec = kw.get("n_receivers", 64)
            xr = (np.arange(nrec) - (nrec - 1) / 2.0) * kw.get("rec_spacing", 20.0)
            rec = [_nudge((x, 0.0, kw.get("rec_z", 2.5)), g) for x in xr]
            rec_rhs = [0] * nrec
        else:
            loops0, rec, rec_rhs = [], [], []
            a = a_small
            for iy, cy in enumerate(centers):
                for ix, cx in enumerate(centers):
                    loops0.append(staircase_loop(g, kz, lambda x, y, cx=cx, cy=cy:
                                                 (np.abs(x - cx) < a) & (np.abs(y - cy) < a)))
                    rec.append(_nudge((cx, cy, kw.get("rec_z", 2.5)), g))
                    rec_rhs.append(len(loops0) - 1)
    elif kind == "ellipsoids":
        # host with random ellipsoidal conductors under an n x n grid of small
        # square loops (one RHS column and one central receiver each)
        host = kw.get("sigma", 0.005)
        n_ell = kw.get("n_ellipsoids", 4)
        ell_sig = 10.0 ** rng.uniform(np.log10(0.05), 0.0, n_ell)          # 0.05 .. 1 S/m
        ell_ax = rng.uniform(50.0, 300.0, (n_ell, 3))                      # semi-axes (m)
        ell_ctr = np.column_stack([rng.uniform(-300.0, 300.0, n_ell), rng.uniform(-300.0, 300.0, n_ell),
                                   rng.uniform(50.0, 400.0, n_ell)])       # centre depth 50 .. 400 m
        h = kw.get("h_core", 20.0) / scale
        n_l = kw.get("n_loops", 16)
        sp_, a = kw.get("loop_spacing", 40.0), kw.get("loop_half", 25.0)
        centers = (np.arange(n_l) - (n_l - 1) / 2.0) * sp_
        req = list(centers - a) + list(centers + a)
        core = (min(centers) - a - 2 * h, max(centers) + a + 2 * h)
        xs = graded_axis(req, core, h, half, kw.get("ratio", 1.5), h_min=kw.get("h_min", 4.0))
        ys = xs.copy()
        hz = kw.get("h_z", 20.0) / scale
        deepest = float(np.max(ell_ctr[:, 2] + ell_ax[:, 2]))
        zs = graded_axis([0.0], (-2 * hz, min(deepest, kw.get("z_core", 700.0))), hz, half, kw.get("ratio", 1.5))
        g = Grid(xs, ys, zs)

        def phys(x, y, z):
            p = np.where(z > 0, EARTH, AIR)
            for k in range(n_ell):
                d = ((x - ell_ctr[k, 0]) / ell_ax[k, 0]) ** 2 + ((y - ell_ctr[k, 1]) / ell_ax[k, 1]) ** 2 + \
                    ((z - ell_ctr[k, 2]) / ell_ax[k, 2]) ** 2
                p = np.where((d <= 1.0) & (z > 0), EARTH + 1 + k, p)
            return p

        nod, tets, tph = hex_to_tets(g, phys)
        kz = int(np.searchsorted(zs, 0.0))
        domains = [(AIR, sig_air, 1.0, 1.0), (EARTH, host, 1.0, 1.0)] + \
                  [(EARTH + 1 + k, float(ell_sig[k]), 1.0, 1.0) for k in range(n_ell)]
        loops0, rec, rec_rhs = [], [], []
        for cy in centers:
            for cx in centers:
                loops0.append(staircase_loop(g, kz, lambda x, y, cx=cx, cy=cy:
                                             (np.abs(x - cx) < a) & (np.abs(y - cy) < a)))
                rec.append(_nudge((cx, cy, kw.get("rec_z", 2.5)), g))
                rec_rhs.append(len(loops0) - 1)
    elif kind == "layered":
        nlay = int(kw.get("n_layers", rng.integers(3, 7)))
        sig_l = 10.0 ** rng.uniform(-4.0, -1.0, nlay)
        thick = 10.0 ** rng.uniform(1.0, np.log10(300.0), nlay - 1)
        tops = np.concatenate([[0.0], np.cumsum(thick)])          # top of each layer (z down)
        a = kw.get("loop_half", 100.0)
        h = kw.get("h_core", 25.0) / scale
        xs = graded_axis([-a, a], (-a - 2 * h, a + 2 * h), h, half, kw.get("ratio", 1.5))
        ys = xs.copy()
        hz = kw.get("h_z", 10.0) / scale
        zs = graded_axis(list(tops), (-2 * hz, tops[-1] + 2 * hz), hz, half, kw.get("ratio", 1.5), h_min=2.0)
        g = Grid(xs, ys, zs)

        def phys(x, y, z):
            lay = np.clip(np.searchsorted(tops, z, side="right") - 1, 0, nlay - 1)
            return np.where(z > 0, EARTH + lay, AIR)

        nod, tets, tph = hex_to_tets(g, phys)
        kz = int(np.searchsorted(zs, 0.0))
        loops0 = [staircase_loop(g, kz, lambda x, y: (np.abs(x) < a) & (np.abs(y) < a))]
        rec = [_nudge(kw.get("receiver", (0.0, 0.0, 2.0)), g)]
        rec_rhs = [0]
        domains = [(AIR, sig_air, 1.0, 1.0)] + [(EARTH + i, float(sig_l[i]), 1.0, 1.0) for i in range(nlay)]
    else:
        raise ValueError("unknown model kind %r" % kind)
    if kind not in ("block", "multiloop") or mesh_loop is None:
        mesh_loop = loops0[0]
    # the .mesh source (physical 51) is the large loop on a shared grid, so the
    # block and multiloop kinds then write identical mesh files
    nod2, tets1, new = _renumber_loop_first(nod, tets, mesh_loop)
    loops = [[int(new[v]) + 1 for v in lp] for lp in loops0]
    l0 = [int(new[v]) + 1 for v in mesh_loop]
    src = np.array([[l0[i], l0[(i + 1) % len(l0)]] for i in range(len(l0))])
    mesh = Mesh(nod2, tets1, tph, src.astype(np.int64), np.full(len(src), 51, dtype=np.int64))
    ctl = Control()
    ctl.rec_cor = np.array(rec)
    ctl.rec_charac = kw.get("rec_charac", 1e5)
    ctl.domains = domains
    ctl.source_type = 1
    ctl.pulse_type = kw.get("pulse_type", 1)
    ctl.t0 = kw.get("t0", 1e-6)
    ctl.current = 1.0
    ctl.sp_mthd = 2
    ctl.sp_division = kw.get("sp_division", 10)
    ctl.time_maximum = kw.get("time_maximum", 1e-2)
    ctl.sp_double = kw.get("sp_double", 100)
    ctl.sp_dblesize = 2
    out = np.zeros(9, dtype=bool); out[5] = True
    ctl.output = out
    ctl.time_points = kw.get("time_points", np.logspace(-6, -2, 40))
    info = dict(kind=kind, seed=seed, n_nodes=len(nod2), n_tets=len(tets1), grid=g.shape, rng=int(rng.integers(1 << 30)))
    return Model(mesh, ctl, loops, np.array(rec), np.array(rec_rhs, dtype=np.int32), info)
