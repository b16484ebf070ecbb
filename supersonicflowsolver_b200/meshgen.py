"""Seeded synthetic wedge/ramp meshes in Fluent ASCII layout.

The reference ships hand-made GAMBIT meshes of a compression ramp in a channel
(x in [0, 3], y in [0, 1], ramp from x = 0.5, e.g. wedge40_120.msh). This module
builds the same family of domains for any ramp angle and resolution:

* ``wedge2d``: nx x ny quads; optional seeded jitter of interior nodes
  (fraction of the local spacing) and seeded shuffling of cells and faces
  inside their zones;
* ``wedge3d``: the 2D profile extruded in z, as hexahedra or split into six
  tetrahedra per hex along the main diagonal (Kuhn/Freudenthal split, which
  is conforming between neighbouring hexes);
* ``refine2d`` / ``wedge2d_adapted``: one level of hanging-node refinement of
  chosen quads, in the layout Fluent gives adapted meshes (the reference's
  wedge_adaptation.msh): children in the fluid zone, parent cells in a
  parent zone (bc 32), split faces kept in parent face zones (bc 31), and
  the 58/59 cell and face trees;
* ``write_fluent``: writes the mesh so that both the reference reader
  (psstAnsysDirector::build_step, psstAnsysGridReader.cpp:1138-1306) and this
  package's reader accept it.

Zone layout follows the reference meshes: cells in zone 2 ("fluid"), boundary
face zones 3 symm (bottom before the ramp), 4 wedge (ramp face), 5 wall (flat
part after the ramp), 6 out, 7 up, 8 in, 9 side (z planes, 3D only) and the
interior faces in zone 10. Face nodes are ordered so that the face normal the
reference computes (psstFiniteVolumeGridTools.cpp:423-424 in 2D, the last fan
triangle in 3D) points from neighbour 1 into neighbour 0; boundary faces have
the interior cell as neighbour 0 and no neighbour 1.
"""
import dataclasses
import math

import numpy as np

ZONE_NAMES = {3: "symm", 4: "wedge", 5: "wall", 6: "out", 7: "up", 8: "in", 9: "side"}
INTERIOR_ZONE = 10
CELL_ZONE = 2
PARENT_CELL_ZONE = 11
PARENT_FACE_ZONE_OFFSET = 100  # parent faces of zone z live in zone z + 100


@dataclasses.dataclass
class FaceZone:
    zone_id: int
    bc_type: int  # Fluent boundary type (2 = interior, 3 = wall)
    name: str
    nodes: np.ndarray  # (nf, k) 0-based vertex ids
    c0: np.ndarray  # 0-based cell ids
    c1: np.ndarray  # 0-based cell ids, -1 = none (boundary)


@dataclasses.dataclass
class Mesh:
    dim: int
    verts: np.ndarray  # (nv, dim)
    cell_type: int  # Fluent cell type: 3 quad, 2 tet, 4 hex
    ncells: int  # active cells (the fluid zone)
    face_zones: list  # list[FaceZone], in file order
    # adapted meshes: parent cells (ids ncells .. ncells + nparents - 1, zone
    # PARENT_CELL_ZONE) with their children (0-based active ids), and for each
    # parent face zone (bc 31) its child zone and, per parent face, the local
    # indices of its two halves in that child zone
    nparents: int = 0
    cell_children: np.ndarray = None  # (nparents, 4)
    face_children: dict = dataclasses.field(default_factory=dict)  # parent zone id -> (child zone id, (n, 2))

    @property
    def nfaces(self):
        return sum(len(z.c0) for z in self.face_zones)


def _profile_y(x, angle_deg, ramp_x0, ramp_top):
    """Bottom wall of the channel: flat, then a ramp of the given angle up to ramp_top."""
    t = math.tan(math.radians(angle_deg))
    return np.clip((x - ramp_x0) * t, 0.0, ramp_top)


def _x_lines(nx, length, angle_deg, ramp_x0, ramp_top):
    """x positions of the vertical grid lines; the ramp start and end are snapped
    onto grid lines when a line lies within half a spacing of them."""
    x = np.linspace(0.0, length, nx + 1)
    dx = length / nx
    ramp_x1 = ramp_x0 + ramp_top / math.tan(math.radians(angle_deg)) if angle_deg > 0 else ramp_x0
    for xs in (ramp_x0, ramp_x1):
        i = int(round(xs / dx))
        if 0 < i < nx and abs(x[i] - xs) < 0.5 * dx:
            x[i] = xs
    return x, ramp_x1


def _structured_nodes(nx, ny, angle_deg, length, height, ramp_x0, ramp_top):
    x, ramp_x1 = _x_lines(nx, length, angle_deg, ramp_x0, ramp_top)
    yb = _profile_y(x, angle_deg, ramp_x0, ramp_top)
    s = np.linspace(0.0, 1.0, ny + 1)
    X = np.repeat(x[:, None], ny + 1, axis=1)  # (nx+1, ny+1)
    Y = yb[:, None] + (height - yb[:, None]) * s[None, :]
    return X, Y, x, ramp_x1


def _bottom_zone(xm, ramp_x0, ramp_x1):
    return np.where(xm < ramp_x0 - 1e-12, 3, np.where(xm < ramp_x1 - 1e-12, 4, 5))


def wedge2d(nx=120, ny=40, angle_deg=15.0, length=3.0, height=1.0, ramp_x0=0.5, ramp_top=0.2,
            jitter=0.0, seed=0, shuffle_seed=None, interior_first=False):
    """nx x ny quad mesh of the ramp channel (nx along x)."""
    X, Y, x, ramp_x1 = _structured_nodes(nx, ny, angle_deg, length, height, ramp_x0, ramp_top)
    if jitter > 0.0:
        rng = np.random.default_rng(seed)
        dxl = np.minimum(np.diff(x)[:-1], np.diff(x)[1:])  # local x spacing at interior lines
        dy = np.diff(Y, axis=1)
        dyl = np.minimum(dy[1:-1, :-1], dy[1:-1, 1:])  # (nx-1, ny-1)
        jx = rng.uniform(-jitter, jitter, size=(nx - 1, ny - 1)) * dxl[:, None]
        jy = rng.uniform(-jitter, jitter, size=(nx - 1, ny - 1)) * dyl
        X = X.copy()
        Y = Y.copy()
        X[1:-1, 1:-1] += jx
        Y[1:-1, 1:-1] += jy
    vid = np.arange((nx + 1) * (ny + 1)).reshape(nx + 1, ny + 1)
    verts = np.stack([X.ravel(), Y.ravel()], axis=1)
    cid = np.arange(nx * ny).reshape(nx, ny)  # cell (i, j)

    zones = {}
    # interior vertical faces between (i-1, j) and (i, j): nodes (i,j)->(i,j+1), c0 = left cell
    i, j = np.meshgrid(np.arange(1, nx), np.arange(ny), indexing="ij")
    iv_nodes = np.stack([vid[i, j], vid[i, j + 1]], -1).reshape(-1, 2)
    iv_c0, iv_c1 = cid[i - 1, j].ravel(), cid[i, j].ravel()
    # interior horizontal faces between (i, j-1) and (i, j): nodes (i,j)->(i+1,j), c0 = upper cell
    i, j = np.meshgrid(np.arange(nx), np.arange(1, ny), indexing="ij")
    ih_nodes = np.stack([vid[i, j], vid[i + 1, j]], -1).reshape(-1, 2)
    ih_c0, ih_c1 = cid[i, j].ravel(), cid[i, j - 1].ravel()
    zones[INTERIOR_ZONE] = (np.concatenate([iv_nodes, ih_nodes]), np.concatenate([iv_c0, ih_c0]),
                            np.concatenate([iv_c1, ih_c1]))
    jj = np.arange(ny)
    zones[8] = (np.stack([vid[0, jj + 1], vid[0, jj]], -1), cid[0, jj], None)  # in
    zones[6] = (np.stack([vid[nx, jj], vid[nx, jj + 1]], -1), cid[nx - 1, jj], None)  # out
    ii = np.arange(nx)
    zones[7] = (np.stack([vid[ii + 1, ny], vid[ii, ny]], -1), cid[ii, ny - 1], None)  # up
    xm = 0.5 * (x[:-1] + x[1:])
    bz = _bottom_zone(xm, ramp_x0, ramp_x1)
    for z in (3, 4, 5):
        sel = ii[bz == z]
        if len(sel):
            zones[z] = (np.stack([vid[sel, 0], vid[sel + 1, 0]], -1), cid[sel, 0], None)
    mesh = _assemble(2, verts, 3, nx * ny, zones, interior_first)
    if shuffle_seed is not None:
        mesh = shuffle(mesh, shuffle_seed)
    return mesh


def _assemble(dim, verts, cell_type, ncells, zones, interior_first):
    order = sorted(k for k in zones if k != INTERIOR_ZONE)
    order = ([INTERIOR_ZONE] + order) if interior_first else (order + [INTERIOR_ZONE])
    fz = []
    for z in order:
        nodes, c0, c1 = zones[z]
        if c1 is None:
            c1 = -np.ones_like(c0)
        bc = 2 if z == INTERIOR_ZONE else 3
        name = "default-interior" if z == INTERIOR_ZONE else ZONE_NAMES[z]
        fz.append(FaceZone(z, bc, name, np.ascontiguousarray(nodes, dtype=np.int64),
                           np.asarray(c0, dtype=np.int64), np.asarray(c1, dtype=np.int64)))
    return Mesh(dim, np.ascontiguousarray(verts, dtype=np.float64), cell_type, ncells, fz)


def shuffle(mesh, seed):
    """Permutes cells and, inside every face zone, faces (seeded)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(mesh.ncells)  # new id of old cell
    newz = []
    for z in mesh.face_zones:
        fp = rng.permutation(len(z.c0))
        c1 = z.c1[fp]
        newz.append(FaceZone(z.zone_id, z.bc_type, z.name, z.nodes[fp], perm[z.c0[fp]],
                             np.where(c1 >= 0, perm[np.maximum(c1, 0)], -1)))
    return Mesh(mesh.dim, mesh.verts, mesh.cell_type, mesh.ncells, newz)


def refine2d(mesh, refine):
    """One level of hanging-node refinement of the quads selected by the
    boolean mask ``refine`` (ncells,): each becomes four children joined at its
    centre, each face next to a refined cell is split at its midpoint. The
    split face stays in the file as a parent face (bc 31, zone id + 100) with
    its original neighbours; its halves replace it in its own zone, so a quad
    next to a refined one has five faces (a hanging node). Active cells are
    the unrefined cells in their order, then the children of each refined
    cell; parents follow as zone PARENT_CELL_ZONE (bc 32)."""
    assert mesh.dim == 2 and mesh.cell_type == 3 and mesh.nparents == 0
    refine = np.asarray(refine, dtype=bool)
    nc = mesh.ncells
    # each cell's edges oriented with the cell on the left (c0 is left of n0->n1)
    edges = [[] for _ in range(nc)]
    for z in mesh.face_zones:
        for i in range(len(z.c0)):
            a, b = int(z.nodes[i, 0]), int(z.nodes[i, 1])
            edges[z.c0[i]].append((a, b))
            if z.c1[i] >= 0:
                edges[z.c1[i]].append((b, a))
    verts = [tuple(v) for v in mesh.verts]

    def add_vert(x):
        verts.append(tuple(x))
        return len(verts) - 1

    ref_ids = np.flatnonzero(refine)
    unref = np.flatnonzero(~refine)
    new_id = np.full(nc, -1, dtype=np.int64)
    new_id[unref] = np.arange(len(unref))
    corners, child_of = {}, {}  # refined cell -> CCW corners; -> 4 child ids
    for r, c in enumerate(ref_ids):
        nxt = {a: b for a, b in edges[c]}
        assert len(nxt) == 4, "refine2d needs plain quads"
        v = [edges[c][0][0]]
        for _ in range(3):
            v.append(nxt[v[-1]])
        corners[c] = v
        child_of[c] = len(unref) + 4 * r + np.arange(4)
    mid = {}  # undirected edge -> midpoint vertex

    def midpoint(a, b):
        k = (min(a, b), max(a, b))
        if k not in mid:
            mid[k] = add_vert(0.5 * (np.asarray(verts[a]) + np.asarray(verts[b])))
        return mid[k]

    def half_cell(c, a, b, first):
        """Active cell on the left of the half of edge a->b (cell c on its left)
        that touches a (first) or b."""
        if not refine[c]:
            return new_id[c]
        v = corners[c]
        k = v.index(a)
        return child_of[c][k] if first else child_of[c][(k + 1) % 4]

    pid = np.full(nc, -1, dtype=np.int64)
    ntot_active = len(unref) + 4 * len(ref_ids)
    pid[ref_ids] = ntot_active + np.arange(len(ref_ids))

    def cell_ref(c):  # a cell as a parent face's neighbour
        return pid[c] if refine[c] else new_id[c]

    zones, parents = [], []
    for z in mesh.face_zones:
        nodes, c0, c1 = [], [], []
        pn, p0, p1, kids = [], [], [], []
        for i in range(len(z.c0)):
            a, b = int(z.nodes[i, 0]), int(z.nodes[i, 1])
            l, r = int(z.c0[i]), int(z.c1[i])
            if not (refine[l] or (r >= 0 and refine[r])):
                nodes.append((a, b))
                c0.append(new_id[l])
                c1.append(new_id[r] if r >= 0 else -1)
                continue
            m = midpoint(a, b)
            pn.append((a, b))
            p0.append(cell_ref(l))
            p1.append(cell_ref(r) if r >= 0 else -1)
            kids.append((len(nodes), len(nodes) + 1))
            for (s, e), first in (((a, m), True), ((m, b), False)):
                nodes.append((s, e))
                c0.append(half_cell(l, a, b, first))
                c1.append(half_cell(r, b, a, not first) if r >= 0 else -1)
        if z.zone_id == INTERIOR_ZONE:
            for c in ref_ids:
                v = corners[c]
                ctr = add_vert(np.mean([verts[q] for q in v], axis=0))
                ms = [midpoint(v[k], v[(k + 1) % 4]) for k in range(4)]
                for k in range(4):  # child k left of m_k -> centre, child k+1 right of it
                    nodes.append((ms[k], ctr))
                    c0.append(child_of[c][k])
                    c1.append(child_of[c][(k + 1) % 4])
        zones.append(FaceZone(z.zone_id, z.bc_type, z.name, np.asarray(nodes, dtype=np.int64).reshape(-1, 2),
                              np.asarray(c0, dtype=np.int64), np.asarray(c1, dtype=np.int64)))
        if pn:
            parents.append((FaceZone(z.zone_id + PARENT_FACE_ZONE_OFFSET, 31, "", np.asarray(pn, dtype=np.int64),
                                     np.asarray(p0, dtype=np.int64), np.asarray(p1, dtype=np.int64)),
                            z.zone_id, np.asarray(kids, dtype=np.int64)))
    face_children = {pz.zone_id: (cz, k) for pz, cz, k in parents}
    cell_children = np.stack([child_of[c] for c in ref_ids]) if len(ref_ids) else np.zeros((0, 4), np.int64)
    return Mesh(2, np.asarray(verts, dtype=np.float64), 3, ntot_active, zones + [p[0] for p in parents],
                len(ref_ids), cell_children, face_children)


def wedge2d_adapted(nx=40, ny=12, angle_deg=15.0, refine_frac=0.25, seed=0, **kw):
    """wedge2d with a seeded random fraction of its quads refined once, plus
    every quad in the band x in [0.4, 1.2] next to the ramp foot and the
    oblique shock (where an adaptation would put cells)."""
    base = wedge2d(nx, ny, angle_deg, **kw)
    rng = np.random.default_rng(seed)
    refine = rng.random(base.ncells) < refine_frac
    xc = np.zeros(base.ncells)
    cnt = np.zeros(base.ncells)
    for z in base.face_zones:
        xm = base.verts[z.nodes].mean(axis=1)[:, 0]
        np.add.at(xc, z.c0, xm)
        np.add.at(cnt, z.c0, 1)
        inner = z.c1 >= 0
        np.add.at(xc, z.c1[inner], xm[inner])
        np.add.at(cnt, z.c1[inner], 1)
    xc /= cnt
    refine |= (xc > 0.4) & (xc < 1.2)
    return refine2d(base, refine)


def wedge3d(nx=200, ny=100, nz=50, angle_deg=12.0, length=3.0, height=1.0, depth=1.0, ramp_x0=0.5,
            ramp_top=0.2, tets=True, interior_first=False):
    """The 2D profile extruded over z in [0, depth]: hexahedra or 6 Kuhn tets per hex."""
    X, Y, x, ramp_x1 = _structured_nodes(nx, ny, angle_deg, length, height, ramp_x0, ramp_top)
    zc = np.linspace(0.0, depth, nz + 1)
    NX, NY, NZ = nx + 1, ny + 1, nz + 1
    verts = np.empty((NX * NY * NZ, 3))
    verts[:, 0] = np.repeat(X.ravel(), NZ)
    verts[:, 1] = np.repeat(Y.ravel(), NZ)
    verts[:, 2] = np.tile(zc, NX * NY)

    def vid(i, j, k):
        return (i * NY + j) * NZ + k

    gi, gj, gk = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    gi, gj, gk = gi.ravel(), gj.ravel(), gk.ravel()
    corner = np.stack([vid(gi + a, gj + b, gk + c) for a in (0, 1) for b in (0, 1) for c in (0, 1)], -1)
    # corner index bits: a*4 + b*2 + c
    if tets:
        cells = []
        for p in ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)):
            bits = [0]
            cur = 0
            for ax in p:
                cur |= (4, 2, 1)[ax]
                bits.append(cur)
            cells.append(corner[:, bits])
        cell_nodes = np.stack(cells, 1).reshape(-1, 4)  # hex-major, 6 tets each
        face_local = np.array([[1, 2, 3], [0, 3, 2], [0, 1, 3], [0, 2, 1]])
        opp = np.array([0, 1, 2, 3])
        cell_type = 2
    else:
        cell_nodes = corner
        # quad faces of a hex (corner bits a*4+b*2+c), each listed cyclically
        face_local = np.array([[0, 1, 3, 2], [4, 6, 7, 5], [0, 4, 5, 1], [2, 3, 7, 6], [0, 2, 6, 4],
                               [1, 5, 7, 3]])
        opp = None
        cell_type = 4
    ncell = len(cell_nodes)
    nfl = face_local.shape[0]
    k = face_local.shape[1]
    fn = cell_nodes[:, face_local].reshape(-1, k)  # (ncell*nfl, k)
    fcell = np.repeat(np.arange(ncell), nfl)
    # orient every face outward from its cell
    P = verts[fn]  # (n, k, 3)
    nrm = np.cross(P[:, 1] - P[:, 0], P[:, 2] - P[:, 0])
    cc = verts[cell_nodes].mean(axis=1)[fcell]
    out = np.einsum("ij,ij->i", nrm, P.mean(axis=1) - cc) > 0
    fn = np.where(out[:, None], fn, fn[:, ::-1])
    key_nodes = np.sort(fn, axis=1)
    if k == 3:
        key = (key_nodes[:, 0] << 42) | (key_nodes[:, 1] << 21) | key_nodes[:, 2]
    else:
        key = (key_nodes[:, 0] << 42) | (key_nodes[:, 1] << 21) | key_nodes[:, 3]
    order = np.argsort(key, kind="stable")
    ks = key[order]
    first = np.ones(len(ks), dtype=bool)
    first[1:] = ks[1:] != ks[:-1]
    starts = np.flatnonzero(first)
    counts = np.diff(np.append(starts, len(ks)))
    a = order[starts]
    inter = counts == 2
    b = np.where(inter, order[np.minimum(starts + 1, len(order) - 1)], -1)
    # interior: nodes outward from cell A -> normal points into cell B: c0 = B, c1 = A
    ia, ib = a[inter], b[inter]
    zones = {INTERIOR_ZONE: (fn[ia], fcell[ib], fcell[ia])}
    # boundary: normal must point into the interior cell (neighbour 0): reverse
    ba = a[~inter]
    bn = fn[ba][:, ::-1]
    bc_cell = fcell[ba]
    cen = verts[bn].mean(axis=1)
    tol = 1e-9
    zid = np.full(len(ba), -1)
    zid[np.abs(cen[:, 0]) < tol] = 8
    zid[np.abs(cen[:, 0] - length) < tol] = 6
    zid[(zid < 0) & ((np.abs(cen[:, 2]) < tol) | (np.abs(cen[:, 2] - depth) < tol))] = 9
    zid[(zid < 0) & (np.abs(cen[:, 1] - height) < tol)] = 7
    rest = zid < 0
    zid[rest] = _bottom_zone(cen[rest, 0], ramp_x0, ramp_x1)
    for z in (3, 4, 5, 6, 7, 8, 9):
        sel = zid == z
        if sel.any():
            zones[z] = (bn[sel], bc_cell[sel], None)
    return _assemble(3, verts, cell_type, ncell, zones, interior_first)


def write_fluent(mesh, path):
    """Writes the mesh as a Fluent ASCII .msh (hex indices, 1-based)."""
    dim = mesh.dim
    nv = len(mesh.verts)
    with open(path, "w") as f:
        f.write('(0 "supersonicflowsolver_b200 synthetic mesh")\n\n')
        f.write("(0 \"Dimension:\")\n(2 %d)\n\n" % dim)
        f.write("(10 (0 1 %x 0 %d))\n" % (nv, dim))
        f.write("(10 (1 1 %x 1 %d)(\n" % (nv, dim))
        np.savetxt(f, mesh.verts, fmt="%.17g")
        f.write("))\n\n")
        nf = mesh.nfaces
        f.write("(13 (0 1 %x 0))\n" % nf)
        first = 1
        for z in mesh.face_zones:
            n = len(z.c0)
            k = z.nodes.shape[1]
            ftype = {2: 2, 3: 3, 4: 4}[k]
            f.write("(13 (%x %x %x %x %x)(\n" % (z.zone_id, first, first + n - 1, z.bc_type, ftype))
            cols = np.concatenate([z.nodes + 1, (z.c0 + 1)[:, None], (z.c1 + 1)[:, None]], axis=1)
            np.savetxt(f, cols, fmt="%x")
            f.write("))\n")
            first += n
        zfirst, first = {}, 1
        for z in mesh.face_zones:
            zfirst[z.zone_id] = first
            first += len(z.c0)
        for z in mesh.face_zones:  # face trees of adapted meshes
            if z.bc_type != 31:
                continue
            cz, kids = mesh.face_children[z.zone_id]
            f.write("(59 (%x %x %x %x)(\n" % (zfirst[z.zone_id], zfirst[z.zone_id] + len(z.c0) - 1, z.zone_id, cz))
            np.savetxt(f, np.concatenate([np.full((len(kids), 1), 2), kids + zfirst[cz]], axis=1), fmt="%x")
            f.write("))\n")
        total = mesh.ncells + mesh.nparents
        f.write("\n(12 (0 1 %x 0))\n" % total)
        f.write("(12 (%x 1 %x 1 %x))\n\n" % (CELL_ZONE, mesh.ncells, mesh.cell_type))
        if mesh.nparents:
            f.write("(12 (%x %x %x 20 %x))\n" % (PARENT_CELL_ZONE, mesh.ncells + 1, total, mesh.cell_type))
            f.write("(58 (%x %x %x %x)(\n" % (mesh.ncells + 1, total, PARENT_CELL_ZONE, CELL_ZONE))
            np.savetxt(f, np.concatenate([np.full((mesh.nparents, 1), 4), mesh.cell_children + 1], axis=1),
                       fmt="%x")
            f.write("))\n\n")
        f.write('(0 "Zones:")\n')
        f.write("(39 (%d fluid fluid)())\n" % CELL_ZONE)
        for z in mesh.face_zones:
            if z.bc_type == 31:
                continue  # parent face zones carry no name, as in Fluent's adapted meshes
            kind = "interior" if z.bc_type == 2 else "wall"
            f.write("(39 (%d %s %s)())\n" % (z.zone_id, kind, z.name))


def write_case(dirpath, case, *, mach=2.5, T=300.0, p=101325.0, angle_deg=0.0, cfl=0.5, lc=1,
               max_iter=10, save_step=1000000, rk_level=4, rk_custom=None, flux=3, order=2, grad=1,
               limiter=3, R=287.0, gamma=1.4, dim=2, init_mode=0, zones=("symm", "wedge", "wall", "up")):
    """Writes <case>.inp/.prop/.par/.bvp/.btq in the reference's formats
    (psstFiniteVolumeGrid.cpp:36-194, 403-557, 641-717; Description.md:179-195).

    The gas is given through M = 8.31/R and cp = gamma R/(gamma-1), the only
    inputs the reference accepts (R = 8.31/M at psstFiniteVolumeGrid.cpp:651).
    Files end without a newline: the reference's eof() loops re-read the last
    record otherwise (psstFiniteVolumeGrid.cpp:418, 495).
    """
    import os

    os.makedirs(dirpath, exist_ok=True)
    M = 8.31 / R
    cp = gamma * R / (gamma - 1.0)
    a = math.sqrt(gamma * R * T)
    speed = mach * a
    vel = [speed * math.cos(math.radians(angle_deg)), speed * math.sin(math.radians(angle_deg))]
    if dim == 3:
        vel.append(0.0)
    coeff = " ".join("%.17g" % c for c in (rk_custom or [0.1, 0.2, 0.5, 1.0]))
    lines = ["%d\t//init" % init_mode, "%.17g\t//CFL" % cfl, "%d\t//lc" % lc, "%d\t//maxIter" % max_iter,
             "%d\t//save" % save_step, "%d\t//RK level" % (len(rk_custom) if rk_custom else rk_level),
             "%d\t//RK mode" % (1 if rk_custom else 0), coeff + "\t//custom", "%d\t//flux" % flux,
             "%d\t//order" % order, "%d\t//grad" % grad, "%d\t//limiter" % limiter]
    w = lambda ext, text: open(os.path.join(dirpath, case + ext), "w").write(text)
    w(".inp", "\n".join(lines))
    w(".prop", "%.17g\t//M\n%.17g\t//cp" % (M, cp))
    w(".par", " ".join("%.17g" % v for v in vel) + "\t//velocity\n%.17g\t//T\n%.17g\t//p" % (T, p))
    walls = list(zones) + (["side"] if dim == 3 else [])
    bvp = ["in\t23\t" + "\t".join("%.17g" % v for v in vel) + "\t%.17g" % p]
    bvp += ["%s\t15" % z for z in walls] + ["out\t26"]
    btq = ["in\t27\t%.17g" % T] + ["%s\t18" % z for z in walls] + ["out\t25"]
    w(".bvp", "\n".join(bvp))
    w(".btq", "\n".join(btq))
    return {"M": M, "cp": cp, "velocity": vel, "T": T, "p": p}
