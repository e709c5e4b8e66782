"""Seeded synthetic meshes written in the reference's own input formats.

The reference reads a JSON config (``src/io/Config.cpp:6-82``), a text mesh with
``#node`` / ``#element`` sections (``src/io/MeshParser.h:22-100``; element lines
are 1-based node indices, optionally followed by a material id,
``src/model/Body.cpp:49-90``) and constraint files holding 1-based node indices
(fix, force) or one face per line (pressure) (``src/io/IO.cpp:67-96``,
``src/fe/ExternalConstraint.cpp:50-247``).  Everything here produces exactly
those files, so a generated case runs unchanged through the reference, the
oracle and this library.

Node orderings follow the reference's element classes:

* C3D4  -- any corner order (the residual does not depend on orientation).
* C3D10 -- corners 0..3, then mid-edge nodes on edges (0,1) (1,2) (2,0) (0,3)
  (1,3) (2,3) (``src/fe/element/TetrahedraElement.cpp:62-79``).
* C3D8  -- corners in two loops, 0-1-2-3 then 4-5-6-7 above them
  (``src/fe/element/HexahedraElement.cpp:15-28``).
* C3D20 -- the same 8 corners, then mid-edge nodes on (0,1) (1,2) (2,3) (3,0)
  (4,5) (5,6) (6,7) (7,4) (0,4) (1,5) (2,6) (3,7)
  (``src/fe/element/HexahedraElement.cpp:147-170``).

Units are SI (metres, pascals, newtons).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field

import numpy as np

HEX_EDGES = [(0, 1), (1, 2), (2, 3), (3, 0), (4, 5), (5, 6), (6, 7), (7, 4),
             (0, 4), (1, 5), (2, 6), (3, 7)]
TET10_EDGES = [(0, 1), (1, 2), (2, 0), (0, 3), (1, 3), (2, 3)]
# faces by corner index, as cyclic loops
HEX_FACES = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (1, 2, 6, 5), (2, 3, 7, 6), (3, 0, 4, 7)]
TET_FACES = [(0, 1, 2), (0, 1, 3), (1, 2, 3), (0, 2, 3)]
# Kuhn split of a hexahedron into 6 tetrahedra around the 0-6 diagonal
KUHN = [(0, 1, 2, 6), (0, 2, 3, 6), (0, 3, 7, 6), (0, 7, 4, 6), (0, 4, 5, 6), (0, 5, 1, 6)]


@dataclass
class Mesh:
    X: np.ndarray                  # (n_nodes, 3) float64
    conn: np.ndarray               # (n_elem, n_en) int64, 0-based
    mat: np.ndarray | None = None  # (n_elem,) material ids or None (-> -1)

    @property
    def n_en(self) -> int:
        return self.conn.shape[1]


@dataclass
class Case:
    """A whole reference input: mesh, materials, constraints, analysis keys."""
    mesh: Mesh
    materials: list
    fix: np.ndarray                                   # 0-based node ids
    pressure: list = field(default_factory=list)      # [(value or [vx,vy,vz], faces (list of 0-based tuples))]
    force: list = field(default_factory=list)         # [([fx,fy,fz], 0-based node ids)]
    analysis: dict = field(default_factory=dict)
    integration: str = "full"                         # "full" | "reduced" (library key; the reference ignores it)

    def write(self, directory: str, name: str = "case") -> str:
        """Write mesh/constraint/config files; return the config path."""
        os.makedirs(directory, exist_ok=True)
        write_mesh(os.path.join(directory, "mesh.txt"), self.mesh)
        cons = []
        write_nodes(os.path.join(directory, "fix.txt"), self.fix)
        cons.append({"id": 1, "type": "fix", "constraint_file": "fix.txt"})
        for k, (value, faces) in enumerate(self.pressure):
            fn = f"pressure{k}.txt"
            write_faces(os.path.join(directory, fn), faces)
            cons.append({"id": 2 + k, "type": "pressure", "value": value, "constraint_file": fn})
        for k, (value, nodes) in enumerate(self.force):
            fn = f"force{k}.txt"
            write_nodes(os.path.join(directory, fn), nodes)
            cons.append({"id": 100 + k, "type": "force", "value": list(value), "constraint_file": fn})
        analysis = {"max_solver_iters": 0, "max_line_search": 20, "residual_criterion": 1e-6,
                    "dx_criterion": 1e-8}
        analysis.update(self.analysis)
        if self.integration != "full":
            analysis["integration"] = self.integration
        cfg = {
            "analysis": analysis,
            "model": [{"type": "soft", "mesh_file": "mesh.txt"}],
            "constraint": cons,
            "material": self.materials,
            "output": {"save_frame": False, "show_log": False, "disk_log": False},
        }
        path = os.path.join(directory, name + ".json")
        with open(path, "w") as f:
            json.dump(cfg, f, indent=1)
        return path


# --------------------------------------------------------------------------- writers

def write_mesh(path: str, mesh: Mesh) -> None:
    with open(path, "w") as f:
        f.write("#node\n")
        np.savetxt(f, mesh.X, fmt="%.17g", delimiter="    ")
        f.write("#element\n")
        c = mesh.conn + 1
        if mesh.mat is not None:
            c = np.concatenate([c, mesh.mat.reshape(-1, 1)], axis=1)
        np.savetxt(f, c, fmt="%d", delimiter="    ")


def write_nodes(path: str, nodes) -> None:
    with open(path, "w") as f:
        for n in np.asarray(nodes, dtype=np.int64):
            f.write(f"{n + 1}\n")


def write_faces(path: str, faces) -> None:
    with open(path, "w") as f:
        for face in faces:
            f.write("    ".join(str(int(n) + 1) for n in face) + "\n")


# --------------------------------------------------------------------------- generators

def box_hex8(L, W, H, nx, ny, nz, origin=(0.0, 0.0, 0.0)) -> Mesh:
    """Structured C3D8 grid of the box [0,L]x[0,W]x[0,H]; node id = i + (nx+1)(j + (ny+1)k)."""
    xs = origin[0] + np.linspace(0.0, L, nx + 1)
    ys = origin[1] + np.linspace(0.0, W, ny + 1)
    zs = origin[2] + np.linspace(0.0, H, nz + 1)
    Z, Y, Xg = np.meshgrid(zs, ys, xs, indexing="ij")
    X = np.stack([Xg.ravel(), Y.ravel(), Z.ravel()], axis=1)
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    b = (i * sx + j * sy + k * sz).ravel()
    conn = np.stack([b, b + sx, b + sx + sy, b + sy,
                     b + sz, b + sz + sx, b + sz + sx + sy, b + sz + sy], axis=1)
    return Mesh(X, conn.astype(np.int64))


def hex8_to_tet4(m: Mesh) -> Mesh:
    """Kuhn split: 6 tets per hex sharing the 0-6 diagonal (conforming on a structured grid)."""
    tets = np.concatenate([m.conn[:, list(t)] for t in KUHN], axis=0)
    # interleave so the 6 tets of one hex are adjacent
    ne = m.conn.shape[0]
    order = np.arange(6 * ne).reshape(6, ne).T.ravel()
    tets = tets[order]
    return Mesh(m.X.copy(), _orient_tets(m.X, tets))


def _orient_tets(X, tets):
    a, b, c, d = (X[tets[:, i]] for i in range(4))
    vol = np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a))
    t = tets.copy()
    neg = vol < 0
    t[neg, 1], t[neg, 2] = tets[neg, 2], tets[neg, 1]
    return t


def _add_midside(X, conn, edges):
    """Append one mid-edge node per unique edge; returns (X_new, conn_quadratic)."""
    ne = conn.shape[0]
    a = np.concatenate([conn[:, e[0]] for e in edges])
    b = np.concatenate([conn[:, e[1]] for e in edges])
    lo, hi = np.minimum(a, b), np.maximum(a, b)
    key = lo.astype(np.int64) * (X.shape[0] + 1) + hi
    uniq, inv = np.unique(key, return_inverse=True)
    ulo, uhi = uniq // (X.shape[0] + 1), uniq % (X.shape[0] + 1)
    mids = 0.5 * (X[ulo] + X[uhi])
    new_ids = X.shape[0] + inv.reshape(len(edges), ne).T
    return np.concatenate([X, mids], axis=0), np.concatenate([conn, new_ids], axis=1)


def tet4_to_tet10(m: Mesh) -> Mesh:
    X, c = _add_midside(m.X, m.conn, TET10_EDGES)
    return Mesh(X, c, m.mat)


def hex8_to_hex20(m: Mesh) -> Mesh:
    X, c = _add_midside(m.X, m.conn, HEX_EDGES)
    return Mesh(X, c, m.mat)


def boundary_faces(m: Mesh, predicate) -> list:
    """Faces on the boundary (owned by exactly one element) whose nodes all satisfy
    ``predicate(X[nodes]) -> bool``.  Each face lists its corners in cyclic order,
    then its mid-edge nodes for quadratic elements (the reference builds A0 from
    the first 3/4 listed nodes, src/fe/ExternalConstraint.cpp:296,344,417,568)."""
    n_en = m.n_en
    if n_en in (4, 10):
        corner_faces, nc = TET_FACES, 4
    else:
        corner_faces, nc = HEX_FACES, 8
    seen = {}
    for e in range(m.conn.shape[0]):
        row = m.conn[e]
        for f in corner_faces:
            key = tuple(sorted(int(row[i]) for i in f))
            seen.setdefault(key, []).append((e, f))
    out = []
    for key, owners in seen.items():
        if len(owners) != 1:
            continue
        e, f = owners[0]
        row = m.conn[e]
        corners = [int(row[i]) for i in f]
        if not predicate(m.X[corners]):
            continue
        face = list(corners)
        if n_en == 10:
            local = {}
            for k, (p, q) in enumerate(TET10_EDGES):
                local[frozenset((p, q))] = 4 + k
            for t in range(3):
                face.append(int(row[local[frozenset((f[t], f[(t + 1) % 3]))]]))
        elif n_en == 20:
            local = {frozenset(ed): 8 + k for k, ed in enumerate(HEX_EDGES)}
            for t in range(4):
                face.append(int(row[local[frozenset((f[t], f[(t + 1) % 4]))]]))
        out.append(tuple(face))
    out.sort()
    return out


def nodes_where(m: Mesh, predicate) -> np.ndarray:
    return np.nonzero(predicate(m.X))[0]


# --------------------------------------------------------------------------- named workloads

def mat_nh(C10=114000.0, D1=1e-6, density=1050.0, mid=None):
    d = {"type": "neo_hookean", "density": density, "C10": C10, "D1": D1}
    if mid is not None:
        d["id"] = mid
    return d


def mat_mr(C10=80000.0, C01=20000.0, D1=1e-6, density=1050.0, mid=None):
    d = {"type": "mo_riv", "density": density, "C10": C10, "C01": C01, "D1": D1}
    if mid is not None:
        d["id"] = mid
    return d


def mat_yeoh(C10=110000.0, C20=20000.0, C30=-300.0, D1=1e-6, density=1050.0, mid=None):
    d = {"type": "yeoh", "density": density, "C10": C10, "C20": C20, "C30": C30, "D1": D1}
    if mid is not None:
        d["id"] = mid
    return d


def cantilever_c3d4_pressure(L=0.1, W=0.02, H=0.02, nx=10, ny=4, nz=4, p=1.0e4) -> Case:
    """C3D4 cantilever, 10x4x4 hexes split into 6 tets each (275 nodes, 960
    elements), Neo-Hookean C10=114 kPa, D1=1e-6; x=0 fixed; 10 kPa follower
    pressure on the x=L end face (32 triangles)."""
    m = hex8_to_tet4(box_hex8(L, W, H, nx, ny, nz))
    tol = 1e-9 * L
    fix = nodes_where(m, lambda X: np.abs(X[:, 0]) < tol)
    faces = boundary_faces(m, lambda P: bool(np.all(np.abs(P[:, 0] - L) < tol)))
    return Case(m, [mat_nh()], fix, pressure=[(p, faces)])


def cantilever_c3d8_force(L=0.2, W=0.04, H=0.04, nx=80, ny=16, nz=16, f=(0.0, 0.0, -0.5)) -> Case:
    """C3D8 beam, 80x16x16 hexes (23 409 nodes, 20 480 elements), Mooney-Rivlin
    C10=80 kPa, C01=20 kPa, D1=1e-6; x=0 fixed (289 nodes); nodal force
    [0,0,-0.5] N on each of the 289 x=L nodes."""
    m = box_hex8(L, W, H, nx, ny, nz)
    tol = 1e-9 * L
    fix = nodes_where(m, lambda X: np.abs(X[:, 0]) < tol)
    tip = nodes_where(m, lambda X: np.abs(X[:, 0] - L) < tol)
    return Case(m, [mat_mr()], fix, force=[(list(f), tip)])


def batch_beams(n=256, seed=20261203, el_min=500, el_max=40000) -> list:
    """Uneven batch of C3D4 cantilevers: length L ~ U[0.05, 0.20] m, square
    section side a ~ U[0.010, 0.030] m, element size h ~ U[0.002, 0.005] m
    adjusted so that the element count (6 tets per grid hex) stays within
    [el_min, el_max]; Neo-Hookean or Mooney-Rivlin with probability 1/2,
    C10 log-uniform in [5e4, 5e5] Pa, C01 = U[0, 0.3] C10 (Mooney-Rivlin
    only), D1 = 1e-6; x = 0 fixed; end-face follower pressure ~ U[1, 20] kPa,
    capped at half the beam's Euler buckling load (clamped-free,
    P_cr = pi^2 E I / (4 L^2) with E = 6 (C10 + C01)): the follower pressure
    on the end face compresses the beam, and a slender soft beam above P_cr
    has no stable straight equilibrium for any solver to converge to.
    Returns a list of Cases."""
    rng = np.random.default_rng(seed)
    cases = []
    for _ in range(n):
        L = rng.uniform(0.05, 0.20)
        a = rng.uniform(0.010, 0.030)
        h = rng.uniform(0.002, 0.005)
        mr = rng.uniform() < 0.5
        c10 = float(np.exp(rng.uniform(np.log(5e4), np.log(5e5))))
        c01 = float(rng.uniform(0.0, 0.3) * c10)
        p = float(rng.uniform(1e3, 2e4))
        E = 6.0 * (c10 + (c01 if mr else 0.0))
        p_cr = np.pi ** 2 * E * (a ** 4 / 12.0) / (4.0 * L * L) / (a * a)
        p = min(p, 0.5 * p_cr)

        def counts(hh):
            nx, na = max(1, int(round(L / hh))), max(1, int(round(a / hh)))
            return nx, na, 6 * nx * na * na

        nx, na, ne = counts(h)
        while ne > el_max:
            h *= 1.05
            nx, na, ne = counts(h)
        while ne < el_min:
            h /= 1.05
            nx, na, ne = counts(h)
        m = hex8_to_tet4(box_hex8(L, a, a, nx, na, na))
        tol = 1e-9 * L
        fix = nodes_where(m, lambda X: np.abs(X[:, 0]) < tol)
        faces = boundary_faces(m, lambda P: bool(np.all(np.abs(P[:, 0] - L) < tol)))
        mat = mat_mr(C10=c10, C01=c01) if mr else mat_nh(C10=c10)
        cases.append(Case(m, [mat], fix, pressure=[(p, faces)]))
    return cases


def small_case(etype: str, material: str, load: str, n=(3, 2, 2), size=(0.03, 0.01, 0.01),
               integration="full", seed=0) -> Case:
    """Small parity case: a cantilever block of any element type x material x load."""
    L, W, H = size
    base = box_hex8(L, W, H, *n)
    # perturb interior corner positions a little so elements are not all
    # identical (mid-edge nodes are added afterwards, so edges stay straight)
    rng = np.random.default_rng(seed)
    h = min(L / n[0], W / n[1], H / n[2])
    inner = np.all((base.X > 1e-12) & (base.X < np.array([L, W, H]) - 1e-12), axis=1)
    base.X[inner] += rng.uniform(-0.08 * h, 0.08 * h, size=(int(inner.sum()), 3))
    if etype == "C3D4":
        m = hex8_to_tet4(base)
    elif etype == "C3D10":
        m = tet4_to_tet10(hex8_to_tet4(base))
    elif etype == "C3D8":
        m = base
    elif etype == "C3D20":
        m = hex8_to_hex20(base)
    else:
        raise ValueError(etype)
    mats = {"nh": mat_nh(C10=114000.0), "mr": mat_mr(C10=57000.0, C01=57000.0),
            "yeoh": mat_yeoh(C10=114000.0, C20=16000.0, C30=16000.0)}[material]
    tol = 1e-9 * L
    fix = nodes_where(m, lambda X: np.abs(X[:, 0]) < tol)
    end = lambda P: bool(np.all(np.abs(P[:, 0] - L) < tol))
    case = Case(m, [mats], fix, integration=integration)
    if load == "pressure":
        case.pressure.append((2.0e4, boundary_faces(m, end)))
    elif load == "dpressure":
        case.pressure.append(([0.0, 3000.0, 0.0], boundary_faces(m, end)))
    elif load == "force":
        case.force.append(([0.0, 0.0, -0.05], nodes_where(m, lambda X: np.abs(X[:, 0] - L) < tol)))
    elif load == "top_pressure":
        case.pressure.append((1.5e4, boundary_faces(m, lambda P: bool(np.all(np.abs(P[:, 2] - H) < tol)))))
    else:
        raise ValueError(load)
    return case


def cylinder_cap_c3d20(ri=0.020, ro=0.025, h=0.030, plate=0.005, n_theta=64, n_r=4, n_z=24, n_ring=19,
                       n_plate=2, p=1.0e4, reduced=True) -> Case:
    """Hollow cylinder closed by a top plate, C3D20 (reduced integration by default).

    Shell: n_theta x n_r x n_z hexahedra between radii ri and ro, height h.
    Plate (thickness `plate`, n_plate layers): a butterfly mesh -- a square core
    of (n_theta/4)^2 hexahedra and an O-grid of n_ring layers from the core's
    boundary out to ro.  The O-grid's outer n_r layers share the shell's top
    nodes, and the angular index starts at the core's corner (-45 degrees).
    Neo-Hookean C10 = 114 kPa, D1 = 1e-6; z = 0 fixed; follower pressure p on
    the inner wall and on the plate's underside inside the cavity (a closed
    cavity)."""
    assert n_theta % 4 == 0 and n_ring > n_r
    nc = n_theta // 4
    nodes, index = [], {}

    def node(key, xyz):
        if key not in index:
            index[key] = len(nodes)
            nodes.append(xyz)
        return index[key]

    th = -np.pi / 4 + 2 * np.pi * np.arange(n_theta) / n_theta
    shell_r = np.linspace(ri, ro, n_r + 1)
    hw = 0.45 * ri / np.sqrt(2.0)  # half-width of the square core
    n_blend = n_ring - n_r         # O-grid layers from the square to radius ri

    def square_pt(j):
        side, t = divmod(j % n_theta, nc)
        u = -hw + 2 * hw * t / nc
        return [(hw, u), (-u, hw), (-hw, -u), (u, -hw)][side]

    def ring_xy(sidx, j):
        if sidx >= n_blend:
            r = shell_r[sidx - n_blend]
            return r * np.cos(th[j]), r * np.sin(th[j])
        t = sidx / n_blend
        sq = square_pt(j)
        return ((1 - t) * sq[0] + t * ri * np.cos(th[j]), (1 - t) * sq[1] + t * ri * np.sin(th[j]))

    def core_to_ring(a, b):
        """Square-grid boundary point (a, b) -> ring angular index, or None inside."""
        if a == nc:
            return b % n_theta
        if b == nc:
            return nc + (nc - a)
        if a == 0:
            return 2 * nc + (nc - b)
        if b == 0:
            return (3 * nc + a) % n_theta
        return None

    z_shell = np.linspace(0.0, h, n_z + 1)
    z_plate = h + np.linspace(0.0, plate, n_plate + 1)
    # plate level c = 0 is the shell's top, so shell nodes at iz = n_z use plate keys
    def shell_node(a, j, iz):
        if iz == n_z:
            return plate_node(n_blend + a, j, 0)
        r = shell_r[a]
        return node(("s", a, j, iz), (r * np.cos(th[j]), r * np.sin(th[j]), z_shell[iz]))

    def plate_node(sidx, j, c):
        x, y = ring_xy(sidx, j)
        return node(("r", sidx, j % n_theta, c), (x, y, z_plate[c]))

    def core_node(a, b, c):
        j = core_to_ring(a, b)
        if j is not None:
            return plate_node(0, j, c)
        return node(("c", a, b, c), (-hw + 2 * hw * a / nc, -hw + 2 * hw * b / nc, z_plate[c]))

    hexes = []
    for iz in range(n_z):
        for a in range(n_r):
            for j in range(n_theta):
                jn = (j + 1) % n_theta
                hexes.append([shell_node(a, j, iz), shell_node(a + 1, j, iz), shell_node(a + 1, jn, iz),
                              shell_node(a, jn, iz), shell_node(a, j, iz + 1), shell_node(a + 1, j, iz + 1),
                              shell_node(a + 1, jn, iz + 1), shell_node(a, jn, iz + 1)])
    for c in range(n_plate):
        for sidx in range(n_ring):
            for j in range(n_theta):
                jn = (j + 1) % n_theta
                hexes.append([plate_node(sidx, j, c), plate_node(sidx + 1, j, c), plate_node(sidx + 1, jn, c),
                              plate_node(sidx, jn, c), plate_node(sidx, j, c + 1), plate_node(sidx + 1, j, c + 1),
                              plate_node(sidx + 1, jn, c + 1), plate_node(sidx, jn, c + 1)])
        for a in range(nc):
            for b in range(nc):
                hexes.append([core_node(a, b, c), core_node(a + 1, b, c), core_node(a + 1, b + 1, c),
                              core_node(a, b + 1, c), core_node(a, b, c + 1), core_node(a + 1, b, c + 1),
                              core_node(a + 1, b + 1, c + 1), core_node(a, b + 1, c + 1)])
    X = np.array(nodes, dtype=np.float64)
    conn = np.array(hexes, dtype=np.int64)
    # orient every hexahedron so that its bottom loop 0-1-2-3 runs counter-clockwise seen from its top
    a_, b_, d_, e_ = (X[conn[:, k]] for k in (0, 1, 3, 4))
    neg = np.einsum("ij,ij->i", b_ - a_, np.cross(d_ - a_, e_ - a_)) < 0
    conn[neg] = conn[neg][:, [0, 3, 2, 1, 4, 7, 6, 5]]
    m = hex8_to_hex20(Mesh(X, conn))
    tol = 1e-9
    fix = nodes_where(m, lambda P: np.abs(P[:, 2]) < tol)
    r_xy = lambda P: np.sqrt(P[:, 0] ** 2 + P[:, 1] ** 2)
    inner_wall = lambda P: bool(np.all(np.abs(r_xy(P) - ri) < 1e-7) and np.all(P[:, 2] <= h + 1e-9))
    underside = lambda P: bool(np.all(np.abs(P[:, 2] - h) < 1e-9) and np.all(r_xy(P) <= ri + 1e-7))
    faces = boundary_faces(m, lambda P: inner_wall(P) or underside(P))
    return Case(m, [mat_nh()], fix, pressure=[(p, faces)], integration="reduced" if reduced else "full")


def finger_c3d10(L=0.080, W=0.015, H=0.015, nx=80, nyz=12, n_ch=8, ch_len=0.006, ch_w=0.010, pitch=0.009,
                 p=3.0e4) -> tuple:
    """Pneumatic finger: a block with n_ch internal rectangular chambers, voxel hex
    grid -> 6 tets per voxel -> C3D10.  Yeoh C10 = 110 kPa, C20 = 20 kPa,
    C30 = -300 Pa, D1 = 1e-6; x = 0 face fixed; follower pressure p on the
    chamber walls.  Returns (case, tip node index) with the tip node at the
    centre of the x = L face's bottom edge line (y = W/2, z = 0)."""
    hx, hyz = L / nx, W / nyz
    base = box_hex8(L, W, H, nx, nyz, nyz)
    # voxel centres; remove the chambers
    ci = np.arange(nx)
    cj = np.arange(nyz)
    K, J, I = np.meshgrid(cj, cj, ci, indexing="ij")
    xc, yc, zc = (I.ravel() + 0.5) * hx, (J.ravel() + 0.5) * hyz, (K.ravel() + 0.5) * hyz
    x0 = round(((L - ((n_ch - 1) * pitch + ch_len)) / 2) / hx) * hx
    inside = np.zeros(xc.shape, dtype=bool)
    for k in range(n_ch):
        xa = x0 + k * pitch
        inside |= (xc > xa) & (xc < xa + ch_len) & (np.abs(yc - W / 2) < ch_w / 2) & (np.abs(zc - H / 2) < ch_w / 2)
    conn = base.conn[~inside]
    used = np.unique(conn)
    remap = -np.ones(base.X.shape[0], dtype=np.int64)
    remap[used] = np.arange(used.shape[0])
    m = hex8_to_tet4(Mesh(base.X[used], remap[conn]))
    m = tet4_to_tet10(m)
    tol = 1e-9
    fix = nodes_where(m, lambda P: np.abs(P[:, 0]) < tol)
    outer = lambda P: bool(np.all(np.abs(P[:, 0]) < tol) or np.all(np.abs(P[:, 0] - L) < tol)
                           or np.all(np.abs(P[:, 1]) < tol) or np.all(np.abs(P[:, 1] - W) < tol)
                           or np.all(np.abs(P[:, 2]) < tol) or np.all(np.abs(P[:, 2] - H) < tol))
    faces = boundary_faces(m, lambda P: not outer(P))
    tip = int(np.argmin(np.sum((m.X - np.array([L, W / 2, 0.0])) ** 2, axis=1)))
    case = Case(m, [mat_yeoh()], fix, pressure=[(p, faces)])
    return case, tip
