"""Boundary meshes, boundary conditions and internal points in QUADESTH's data layout.

The arrays mirror the reference's module globals (``data_mod.f90:37-52``) so that a
``Mesh`` can be handed to the C ABI without reshaping:

* ``x, y, z``        node coordinates, float64 (n)
* ``nconec``         nodes per element, int32 (ne), 9 = quad9, 6 = tri6
* ``kconec``         connectivity (9, ne), int32, Fortran order, 1-based node numbers
* ``kode``           (3*ne) int32: 0 = displacement prescribed, 1 = traction prescribed
* ``bc``             (27, ne) float64, Fortran order: value of component ld at local node k
                     is ``bc[3*k + ld, e]``
* ``cx, cy, cz``     internal points (l)
* ``pins``           extra pinned displacement DOFs (0-based 3*node+comp) whose value is 0;
                     this has no counterpart in the reference (its supports are per element)

Reader: ``read_quadesth`` follows ``io_mod.f90:36-146`` (``input_data``) and
``io_mod.f90:8-34`` (``read_bc_line``), including the legacy 8-value header and the
complex ``(re,im)`` boundary-condition lines.

Generators build the structured workloads the benchmarks and tests use: the unit
cube under uniaxial stress, the clamped plate and the hollow cubed-sphere shell.
Local node order follows the quad9 convention of ``stress_mod.f90:47-50``:
1:(-1,-1) 2:(0,-1) 3:(1,-1) 4:(1,0) 5:(1,1) 6:(0,1) 7:(-1,1) 8:(-1,0) 9:(0,0), with
the parametric cross product dx/dxi1 x dx/dxi2 pointing out of the solid.
"""
from __future__ import annotations

import dataclasses
import re
from typing import Iterable, List, Optional, Sequence, Tuple

import numpy as np

# parent coordinates of the quad9 local nodes (stress_mod.f90:47-50)
QUAD9_XI = np.array(
    [[-1, -1], [0, -1], [1, -1], [1, 0], [1, 1], [0, 1], [-1, 1], [-1, 0], [0, 0]], dtype=np.int64
)


@dataclasses.dataclass
class Mesh:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    nconec: np.ndarray
    kconec: np.ndarray
    kode: np.ndarray
    bc: np.ndarray
    mu: float
    nu: float
    cx: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    cy: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    cz: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0))
    pins: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, dtype=np.int32))
    title: str = ""
    ntrack: int = 1

    def __post_init__(self):
        self.x = np.ascontiguousarray(self.x, dtype=np.float64)
        self.y = np.ascontiguousarray(self.y, dtype=np.float64)
        self.z = np.ascontiguousarray(self.z, dtype=np.float64)
        self.nconec = np.ascontiguousarray(self.nconec, dtype=np.int32)
        self.kconec = np.asfortranarray(self.kconec, dtype=np.int32)
        self.kode = np.ascontiguousarray(self.kode, dtype=np.int32)
        self.bc = np.asfortranarray(self.bc, dtype=np.float64)
        self.cx = np.ascontiguousarray(self.cx, dtype=np.float64)
        self.cy = np.ascontiguousarray(self.cy, dtype=np.float64)
        self.cz = np.ascontiguousarray(self.cz, dtype=np.float64)
        self.pins = np.ascontiguousarray(self.pins, dtype=np.int32)

    @property
    def n(self) -> int:
        return int(self.x.shape[0])

    @property
    def ne(self) -> int:
        return int(self.nconec.shape[0])

    @property
    def l(self) -> int:  # noqa: E743 - reference name
        return int(self.cx.shape[0])

    @property
    def ndof(self) -> int:
        return 3 * self.n

    @property
    def young(self) -> float:
        # data_mod.f90:101-102
        return 2.0 * self.mu * (1.0 + self.nu)

    def with_points(self, cx, cy, cz) -> "Mesh":
        return dataclasses.replace(self, cx=np.asarray(cx), cy=np.asarray(cy), cz=np.asarray(cz))

    def node_coords(self) -> np.ndarray:
        return np.stack([self.x, self.y, self.z], axis=1)

    def max_elements_per_node(self) -> int:
        cnt = np.zeros(self.n, dtype=np.int64)
        for e in range(self.ne):
            np.add.at(cnt, self.kconec[: self.nconec[e], e] - 1, 1)
        return int(cnt.max()) if self.n else 0

    def validate(self) -> None:
        if self.kconec.shape != (9, self.ne):
            raise ValueError("kconec must have shape (9, ne)")
        if self.bc.shape != (27, self.ne):
            raise ValueError("bc must have shape (27, ne)")
        if self.kode.shape != (3 * self.ne,):
            raise ValueError("kode must have shape (3*ne,)")
        if not np.all((self.nconec == 9) | (self.nconec == 6)):
            raise ValueError("nconec entries must be 6 or 9")
        for e in range(self.ne):
            k = self.kconec[: self.nconec[e], e]
            if k.min() < 1 or k.max() > self.n:
                raise ValueError(f"element {e + 1} references a node outside 1..{self.n}")
        if self.mu <= 0.0:
            raise ValueError("shear modulus must be positive")


# ----------------------------------------------------------------------------------
# cube8.dat reader (io_mod.f90:36-146)
# ----------------------------------------------------------------------------------

_SPLIT = re.compile(r"[\s,]+")


def _tokens(line: str) -> List[str]:
    return [t for t in _SPLIT.split(line.strip()) if t]


def _num(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


class _ListDirected:
    """Fortran list-directed READ over a line iterator: a read statement consumes
    whole records until its items are satisfied and discards the rest of the last
    record."""

    def __init__(self, lines: Sequence[str]):
        self.lines = list(lines)
        self.pos = 0

    def line(self) -> str:
        if self.pos >= len(self.lines):
            raise EOFError
        s = self.lines[self.pos]
        self.pos += 1
        return s

    def items(self, count: int) -> List[str]:
        out: List[str] = []
        while len(out) < count:
            out.extend(_tokens(self.line()))
        return out[:count]


def _read_bc_line(rd: _ListDirected, nconec: np.ndarray) -> Tuple[int, int, np.ndarray]:
    # io_mod.f90:8-34: legacy "(re,im)" pairs keep only the real part
    line = rd.line()
    vals = np.zeros(9)
    if "(" in line:
        line = line.replace("(", " ").replace(")", " ")
        tok = _tokens(line)
        ie, kd = int(tok[0]), int(tok[1])
        npt = int(nconec[ie - 1])
        pairs = [_num(t) for t in tok[2 : 2 + 2 * npt]]
        vals[:npt] = pairs[0::2]
    else:
        tok = _tokens(line)
        ie, kd = int(tok[0]), int(tok[1])
        npt = int(nconec[ie - 1])
        vals[:npt] = [_num(t) for t in tok[2 : 2 + npt]]
    return ie, kd, vals


def read_quadesth(path_or_text: str, is_text: bool = False) -> Mesh:
    """Parse a QUADESTH input file (the ``cube8.dat`` format)."""
    text = path_or_text if is_text else open(path_or_text).read()
    rd = _ListDirected(text.splitlines())
    title = rd.line().rstrip()
    hdr = _tokens(rd.line())
    if len(hdr) >= 8:  # legacy: nodes, elems, pts, nfr, mu, dam, ro, nu + frequency line
        n, ne, l = int(hdr[0]), int(hdr[1]), int(hdr[2])
        mu, nu = _num(hdr[4]), _num(hdr[7])
        rd.line()
    else:
        n, ne, l = int(hdr[0]), int(hdr[1]), int(hdr[2])
        mu, nu = _num(hdr[3]), _num(hdr[4])
    x = np.zeros(n)
    y = np.zeros(n)
    z = np.zeros(n)
    for _ in range(n):
        t = rd.items(4)
        i = int(t[0]) - 1
        x[i], y[i], z[i] = _num(t[1]), _num(t[2]), _num(t[3])
    nconec = np.zeros(ne, dtype=np.int32)
    kconec = np.zeros((9, ne), dtype=np.int32, order="F")
    for _ in range(ne):
        first = _tokens(rd.line())
        ie, nc = int(first[0]), int(first[1])
        rest = first[2:]
        while len(rest) < nc:
            rest.extend(_tokens(rd.line()))
        nconec[ie - 1] = nc
        kconec[:nc, ie - 1] = [int(v) for v in rest[:nc]]
    kode = np.zeros(3 * ne, dtype=np.int32)
    bc = np.zeros((27, ne), order="F")
    for _ in range(ne):
        for k in range(3):
            ie, kd, vals = _read_bc_line(rd, nconec)
            kode[3 * (ie - 1) + k] = kd
            for j in range(nconec[ie - 1]):
                bc[3 * j + k, ie - 1] = vals[j]
    cx = np.zeros(l)
    cy = np.zeros(l)
    cz = np.zeros(l)
    if l > 0:
        t = rd.items(3 * l)
        v = np.array([_num(s) for s in t]).reshape(l, 3)
        cx, cy, cz = v[:, 0].copy(), v[:, 1].copy(), v[:, 2].copy()
    ntrack = 1
    try:
        ntrack = int(rd.items(1)[0])
    except (EOFError, ValueError):
        ntrack = 1
    return Mesh(x, y, z, nconec, kconec, kode, bc, mu, nu, cx, cy, cz, title=title, ntrack=ntrack)


def write_quadesth(mesh: Mesh, path: str) -> None:
    """Write a mesh in the modern 5-value ``cube8.dat`` format (readable by the
    reference's ``input_data``)."""
    out = [mesh.title or "BEM3D-B200 GENERATED MESH"]
    out.append(f" {mesh.n},{mesh.ne},{mesh.l},{mesh.mu!r},{mesh.nu!r}")
    for i in range(mesh.n):
        out.append(f" {i + 1} {mesh.x[i]!r} {mesh.y[i]!r} {mesh.z[i]!r}")
    for e in range(mesh.ne):
        nc = int(mesh.nconec[e])
        out.append(f" {e + 1} {nc} " + " ".join(str(int(v)) for v in mesh.kconec[:nc, e]))
    for e in range(mesh.ne):
        nc = int(mesh.nconec[e])
        for k in range(3):
            vals = " ".join(repr(float(mesh.bc[3 * j + k, e])) for j in range(nc))
            out.append(f" {e + 1} {int(mesh.kode[3 * e + k])} {vals}")
    for i in range(mesh.l):
        out.append(f" {mesh.cx[i]!r} {mesh.cy[i]!r} {mesh.cz[i]!r}")
    out.append(f" {mesh.ntrack}")
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


# ----------------------------------------------------------------------------------
# structured generators
# ----------------------------------------------------------------------------------


class _NodeTable:
    """Deduplicates nodes by an exact integer lattice key."""

    def __init__(self):
        self.index = {}
        self.coords: List[Tuple[float, float, float]] = []

    def get(self, key, xyz) -> int:
        i = self.index.get(key)
        if i is None:
            i = len(self.coords)
            self.index[key] = i
            self.coords.append(xyz)
        return i


def _face_elements(nodes: _NodeTable, origin_key, du_key, dv_key, mu_el, mv_el, to_xyz):
    """Quad9 elements of one planar lattice face.

    origin_key, du_key, dv_key are integer lattice vectors (half-element steps);
    the face normal du x dv must point out of the solid.  Returns a list of 9-node
    element tuples (0-based)."""
    elems = []
    o = np.array(origin_key)
    du = np.array(du_key)
    dv = np.array(dv_key)
    for p in range(mu_el):
        for q in range(mv_el):
            conn = []
            for a, b in QUAD9_XI:
                key = tuple(int(v) for v in (o + (2 * p + 1 + a) * du + (2 * q + 1 + b) * dv))
                conn.append(nodes.get(key, to_xyz(key)))
            elems.append(tuple(conn))
    return elems


def _box_faces(nx, ny, nz):
    """Six faces of the lattice box [0,2nx]x[0,2ny]x[0,2nz] (half-element units),
    each as (name, origin, du, dv, mu, mv) with du x dv outward."""
    X, Y, Z = 2 * nx, 2 * ny, 2 * nz
    return [
        # z = 0, outward -z: du=+y, dv=+x  (y x x = -z)
        ("z0", (0, 0, 0), (0, 1, 0), (1, 0, 0), ny, nx),
        # z = top, outward +z: du=+x, dv=+y
        ("z1", (0, 0, Z), (1, 0, 0), (0, 1, 0), nx, ny),
        # x = 0, outward -x: du=+z, dv=+y  (z x y = -x)
        ("x0", (0, 0, 0), (0, 0, 1), (0, 1, 0), nz, ny),
        # x = right, outward +x: du=+y, dv=+z
        ("x1", (X, 0, 0), (0, 1, 0), (0, 0, 1), ny, nz),
        # y = 0, outward -y: du=+x, dv=+z  (x x z = -y)
        ("y0", (0, 0, 0), (1, 0, 0), (0, 0, 1), nx, nz),
        # y = right, outward +y: du=+z, dv=+x
        ("y1", (0, Y, 0), (0, 0, 1), (1, 0, 0), nz, nx),
    ]


def box_mesh(lx: float, ly: float, lz: float, nx: int, ny: int, nz: int):
    """Quad9 surface mesh of the box [0,lx]x[0,ly]x[0,lz] with nx, ny, nz elements
    along the edges.  Returns (coords (n,3), kconec (9,ne) 1-based, face name per
    element)."""
    nodes = _NodeTable()
    scale = np.array([lx / (2 * nx), ly / (2 * ny), lz / (2 * nz)])

    def to_xyz(key):
        return tuple(float(v) for v in np.array(key) * scale)

    kcon = []
    faces = []
    for name, o, du, dv, mu_, mv_ in _box_faces(nx, ny, nz):
        els = _face_elements(nodes, o, du, dv, mu_, mv_, to_xyz)
        kcon.extend(els)
        faces.extend([name] * len(els))
    coords = np.array(nodes.coords)
    # exact lattice coordinates for the max faces (avoid 0.1*10 != 1.0 style drift)
    kconec = np.asfortranarray(np.array(kcon, dtype=np.int32).T + 1)
    return coords, kconec, np.array(faces)


def _find_node(coords: np.ndarray, p, tol=1e-12) -> int:
    d = np.abs(coords - np.asarray(p)[None, :]).max(axis=1)
    i = int(np.argmin(d))
    if d[i] > tol:
        raise ValueError(f"no node at {p}")
    return i


def uniaxial_cube(m: int, young: float = 1.0, nu: float = 0.3, side: float = 1.0,
                  traction: float = 1.0, points: Optional[np.ndarray] = None) -> Mesh:
    """Cube [0,side]^3, m x m quad9 elements per face, under uniaxial stress.

    Supports: u_z = 0 on z = 0 (per element, as the reference models supports),
    plus three pinned displacement DOFs that remove the rigid modes left by a
    roller base: u_x = u_y = 0 at the origin and u_y = 0 at (side, 0, 0).
    Loading: t_z = traction on z = side; every other traction is zero.
    Exact solution: sigma_zz = traction, u_z = traction*z/E, u_x = -nu*traction*x/E,
    u_y = -nu*traction*y/E.
    """
    coords, kconec, faces = box_mesh(side, side, side, m, m, m)
    ne = kconec.shape[1]
    kode = np.ones(3 * ne, dtype=np.int32)
    bc = np.zeros((27, ne), order="F")
    for e, f in enumerate(faces):
        if f == "z0":
            kode[3 * e + 2] = 0
        if f == "z1":
            bc[2::3, e] = traction
    i0 = _find_node(coords, (0.0, 0.0, 0.0))
    i1 = _find_node(coords, (side, 0.0, 0.0))
    pins = np.array([3 * i0 + 0, 3 * i0 + 1, 3 * i1 + 1], dtype=np.int32)
    mu = young / (2.0 * (1.0 + nu))
    pts = np.zeros((0, 3)) if points is None else np.asarray(points, dtype=np.float64)
    return Mesh(coords[:, 0], coords[:, 1], coords[:, 2], np.full(ne, 9, np.int32), kconec,
                kode, bc, mu, nu, pts[:, 0], pts[:, 1], pts[:, 2], pins=pins,
                title=f"UNIT CUBE {m}x{m} QUAD9 PER FACE, UNIAXIAL STRESS")


def loaded_box(lx: float, ly: float, lz: float, k: int, nu: float, young: float = 1.0,
               top_tractions: Optional[np.ndarray] = None):
    """Box [0,lx]x[0,ly]x[0,lz], k quad9 elements along every edge, supported like the
    uniaxial cube (u_z = 0 on z = 0 and three pins), one load case per row of
    top_tractions ((nrhs, 3): a uniform traction vector on z = lz; default one case,
    t = (0, 0, 1)).  Returns (mesh, [bc per load case])."""
    coords, kconec, faces = box_mesh(lx, ly, lz, k, k, k)
    ne = kconec.shape[1]
    kode = np.ones(3 * ne, dtype=np.int32)
    top = [e for e, f in enumerate(faces) if f == "z1"]
    for e, f in enumerate(faces):
        if f == "z0":
            kode[3 * e + 2] = 0
    tt = np.array([[0.0, 0.0, 1.0]]) if top_tractions is None else np.asarray(top_tractions, dtype=np.float64)
    bcs = []
    for t in tt:
        bc = np.zeros((27, ne), order="F")
        for e in top:
            for ld in range(3):
                bc[ld::3, e] = t[ld]
        bcs.append(bc)
    i0 = _find_node(coords, (0.0, 0.0, 0.0))
    i1 = _find_node(coords, (lx, 0.0, 0.0))
    pins = np.array([3 * i0 + 0, 3 * i0 + 1, 3 * i1 + 1], dtype=np.int32)
    mu = young / (2.0 * (1.0 + nu))
    mesh = Mesh(coords[:, 0], coords[:, 1], coords[:, 2], np.full(ne, 9, np.int32), kconec, kode,
                bcs[0], mu, nu, pins=pins, title=f"BOX {lx:g}x{ly:g}x{lz:g}, {k} QUAD9 PER EDGE")
    return mesh, bcs


def box_batch(count: int = 512, seed: int = 20261203, loads: int = 8):
    """The batching workload: boxes with sides uniform in [0.5, 2], k in {1..6} quad9
    elements per edge, nu uniform in [0.05, 0.45], E = 1, `loads` random top-face
    traction vectors ~ N(0, 1) each, supports as the uniaxial cube."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        lx, ly, lz = rng.uniform(0.5, 2.0, size=3)
        k = int(rng.integers(1, 7))
        nu = float(rng.uniform(0.05, 0.45))
        tt = rng.standard_normal((loads, 3))
        out.append(loaded_box(lx, ly, lz, k, nu, 1.0, tt))
    return out


def cube_grid_points(vals: Iterable[float]) -> np.ndarray:
    v = np.asarray(list(vals), dtype=np.float64)
    g = np.stack(np.meshgrid(v, v, v, indexing="ij"), axis=-1).reshape(-1, 3)
    return g


def uniform_points(count: int, lo: float, hi: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, size=(count, 3))


def clamped_plate(nxy: int = 40, nz: int = 4, lx: float = 10.0, ly: float = 10.0,
                  lz: float = 1.0, young: float = 210e3, nu: float = 0.3,
                  traction: float = -1.0, points: Optional[np.ndarray] = None) -> Mesh:
    """Plate [0,lx]x[0,ly]x[0,lz], nxy x nxy quad9 elements on the large faces and
    nxy x nz on the side faces; face x = 0 clamped (u = 0), t_z = traction on the
    top face, all other faces traction-free."""
    coords, kconec, faces = box_mesh(lx, ly, lz, nxy, nxy, nz)
    ne = kconec.shape[1]
    kode = np.ones(3 * ne, dtype=np.int32)
    bc = np.zeros((27, ne), order="F")
    for e, f in enumerate(faces):
        if f == "x0":
            kode[3 * e : 3 * e + 3] = 0
        if f == "z1":
            bc[2::3, e] = traction
    mu = young / (2.0 * (1.0 + nu))
    pts = np.zeros((0, 3)) if points is None else np.asarray(points, dtype=np.float64)
    return Mesh(coords[:, 0], coords[:, 1], coords[:, 2], np.full(ne, 9, np.int32), kconec,
                kode, bc, mu, nu, pts[:, 0], pts[:, 1], pts[:, 2],
                title=f"CLAMPED PLATE {lx}x{ly}x{lz}, {nxy}x{nxy}/{nxy}x{nz} QUAD9")


def plate_grid_points(nx=200, ny=200, nz=5, lx=10.0, ly=10.0, lz=1.0) -> np.ndarray:
    xs = (np.arange(nx) + 0.5) * lx / nx
    ys = (np.arange(ny) + 0.5) * ly / ny
    zs = (np.arange(nz) + 0.5) * lz / nz
    return np.stack(np.meshgrid(xs, ys, zs, indexing="ij"), axis=-1).reshape(-1, 3)


def _cubed_sphere_surface(m: int, radius: float, inward: bool, nodes: _NodeTable, tag: int):
    """Quad9 cubed-sphere surface: the 6 faces of the lattice cube [-m, m]^3
    (half-element units, 2m per edge... here m elements per face edge) projected
    radially onto the sphere.  inward=True reverses the orientation so the normal
    points into the cavity (out of the solid shell)."""
    def to_xyz(key):
        v = np.array(key[1:], dtype=np.float64)
        return tuple(float(c) for c in radius * v / np.linalg.norm(v))

    els = []
    M2 = 2 * m  # lattice cube [-m, m] in half-element steps is [-2m/2 ...]; use [0, 2m] shifted
    for name, o, du, dv, mu_, mv_ in _box_faces(m, m, m):
        if inward:
            o2 = o
            du, dv = dv, du
            mu_, mv_ = mv_, mu_
        else:
            o2 = o
        ob = np.array(o2) - m  # centre the lattice cube at the origin
        fac = []
        for p in range(mu_):
            for q in range(mv_):
                conn = []
                for a, b in QUAD9_XI:
                    key3 = ob + (2 * p + 1 + a) * np.array(du) + (2 * q + 1 + b) * np.array(dv)
                    key = (tag,) + tuple(int(v) for v in key3)
                    conn.append(nodes.get(key, to_xyz(key)))
                fac.append(tuple(conn))
        els.extend(fac)
    return els


def hollow_sphere(m: int = 16, a: float = 1.0, b: float = 2.0, young: float = 1.0,
                  nu: float = 0.3, pressure: float = 1.0) -> Mesh:
    """Thick hollow sphere a <= r <= b: cubed-sphere quad9 surfaces with m x m
    elements per cube face on each surface.  Internal pressure p on r = a
    (traction t = p * r_hat on the cavity wall, whose outward normal is -r_hat),
    r = b traction-free.  Six pinned displacement DOFs on the outer surface remove
    the rigid modes."""
    nodes = _NodeTable()
    outer = _cubed_sphere_surface(m, b, inward=False, nodes=nodes, tag=1)
    inner = _cubed_sphere_surface(m, a, inward=True, nodes=nodes, tag=0)
    kcon = outer + inner
    coords = np.array(nodes.coords)
    ne = len(kcon)
    kconec = np.asfortranarray(np.array(kcon, dtype=np.int32).T + 1)
    kode = np.ones(3 * ne, dtype=np.int32)
    bc = np.zeros((27, ne), order="F")
    for e in range(len(outer), ne):
        for k in range(9):
            p = coords[kconec[k, e] - 1]
            rhat = p / np.linalg.norm(p)
            bc[3 * k : 3 * k + 3, e] = pressure * rhat
    # pins: nodes on the outer sphere at +x, +y, +z poles remove 6 rigid modes
    px = _find_node(coords, (b, 0.0, 0.0), tol=1e-9)
    py = _find_node(coords, (0.0, b, 0.0), tol=1e-9)
    pz = _find_node(coords, (0.0, 0.0, b), tol=1e-9)
    pins = np.array([3 * px + 1, 3 * px + 2, 3 * py + 0, 3 * py + 2, 3 * pz + 0, 3 * pz + 1],
                    dtype=np.int32)
    mu = young / (2.0 * (1.0 + nu))
    return Mesh(coords[:, 0], coords[:, 1], coords[:, 2], np.full(ne, 9, np.int32), kconec,
                kode, bc, mu, nu, pins=pins, title=f"HOLLOW SPHERE a={a} b={b} m={m}")


def lame_sphere_displacement(r, a, b, p, young, nu):
    """Radial displacement of a thick sphere under internal pressure (Lame)."""
    r = np.asarray(r, dtype=np.float64)
    k = p * a**3 / (young * (b**3 - a**3))
    return k * ((1.0 - 2.0 * nu) * r + (1.0 + nu) * b**3 / (2.0 * r * r))


def config_mesh(name: str, nu: float = 0.3, with_points: bool = True) -> Mesh:
    """Named workloads: 'cube2' (2x2 per face, 294 DOF, 27 grid points), 'plate40'
    (46,086 DOF, 200x200x5 points), 'cube32' (73,734 DOF, 1M uniform points)."""
    if name == "cube2":
        pts = cube_grid_points([0.25, 0.5, 0.75]) if with_points else None
        return uniaxial_cube(2, young=1.0, nu=nu, points=pts)
    if name == "plate40":
        pts = plate_grid_points() if with_points else None
        return clamped_plate(points=pts, nu=nu)
    if name == "cube32":
        pts = uniform_points(1_000_000, 0.05, 0.95, 20261203) if with_points else None
        return uniaxial_cube(32, young=1.0, nu=nu, points=pts)
    m = re.fullmatch(r"cube(\d+)", name)
    if m:
        k = int(m.group(1))
        pts = cube_grid_points([0.25, 0.5, 0.75]) if with_points else None
        return uniaxial_cube(k, young=1.0, nu=nu, points=pts)
    raise KeyError(name)
