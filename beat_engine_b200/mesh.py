"""Boundary meshes and observation sets for the exterior Burton-Miller path.

Host-side mirror of the reference's mesh handling (paths relative to
``src/beat_engine/julia_local/``):

* :class:`BoundaryMesh` -- ``BoundaryMesh`` and its constructor
  (``src/BeatEngineCore.jl:224-232,344-364``): centroids, unit normals
  ``(v2-v1) x (v3-v1)`` normalised, areas.  Faces are stored 0-based here; the
  reference is 1-based.
* :func:`load_gmsh22_with_tags` -- ``src/BeatEngineCore.jl:301-342``.
* :func:`reference_sphere` -- the icosphere of
  ``tests/analytical_exterior_tests.jl:4-66`` (outward winding enforced).
* :func:`oscillating_sphere` -- the octahedron sphere of
  ``tests/axial_source_tests.jl:71-88``.
* :func:`fibonacci_sphere` -- ``src/BeatEngineCore.jl:828-840``.

All arrays are numpy; nothing here touches the GPU.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class BoundaryMesh:
    """Triangle surface mesh with P1 (vertex) and DP0 (face) dofs.

    ``vertices`` is ``V x 3`` float64, ``faces`` ``F x 3`` int32 (0-based),
    ``physical_tags`` ``F`` int32.  The P1 space has ``V`` dofs numbered like
    the vertices; the DP0 space has ``F`` dofs numbered like the faces
    (``build_p1_space`` / ``build_dp0_space``, ``src/BeatEngineCore.jl:445-446``).
    """

    vertices: np.ndarray
    faces: np.ndarray
    physical_tags: np.ndarray

    def __post_init__(self):
        self.vertices = np.ascontiguousarray(self.vertices, dtype=np.float64).reshape(-1, 3)
        self.faces = np.ascontiguousarray(self.faces, dtype=np.int32).reshape(-1, 3)
        if self.physical_tags is None:
            self.physical_tags = np.ones(len(self.faces), dtype=np.int32)
        self.physical_tags = np.ascontiguousarray(self.physical_tags, dtype=np.int32).reshape(-1)
        if len(self.physical_tags) != len(self.faces):
            raise ValueError("one physical tag per face is required")
        if len(self.faces) and (self.faces.min() < 0 or self.faces.max() >= len(self.vertices)):
            raise ValueError("face vertex index out of range")
        v1 = self.vertices[self.faces[:, 0]]
        v2 = self.vertices[self.faces[:, 1]]
        v3 = self.vertices[self.faces[:, 2]]
        cross = np.cross(v2 - v1, v3 - v1)
        norm = np.linalg.norm(cross, axis=1)
        if np.any(norm == 0):
            raise ValueError("degenerate triangle in mesh")
        self.centroids = (v1 + v2 + v3) / 3.0
        self.areas = norm / 2.0
        self.normals = cross / norm[:, None]

    @property
    def num_vertices(self) -> int:
        return int(self.vertices.shape[0])

    @property
    def num_faces(self) -> int:
        return int(self.faces.shape[0])

    # P1 / DP0 dof counts, as P1Space.global_dof_count / DP0Space.global_dof_count
    @property
    def p1_dofs(self) -> int:
        return self.num_vertices

    @property
    def dp0_dofs(self) -> int:
        return self.num_faces


def load_gmsh22_with_tags(path: str, scale: float = 1.0) -> BoundaryMesh:
    """Read a Gmsh 2.2 ASCII mesh: nodes and triangle (type 2) elements with
    their physical tag (``src/BeatEngineCore.jl:301-342``)."""
    with open(path, "r", encoding="utf-8") as fh:
        lines = [ln.rstrip("\n") for ln in fh]
    try:
        ns, ne = lines.index("$Nodes"), lines.index("$EndNodes")
        es, ee = lines.index("$Elements"), lines.index("$EndElements")
    except ValueError as exc:
        raise ValueError("Only Gmsh 2.2 ASCII meshes with Nodes and Elements sections are supported.") from exc
    index = {}
    verts = []
    for ln in lines[ns + 2:ne]:
        parts = ln.split()
        if len(parts) < 4:
            continue
        index[int(parts[0])] = len(verts)
        verts.append([float(parts[1]) * scale, float(parts[2]) * scale, float(parts[3]) * scale])
    faces, tags = [], []
    for ln in lines[es + 2:ee]:
        parts = ln.split()
        if len(parts) < 8 or int(parts[1]) != 2:
            continue
        tri = [index.get(int(parts[-3]), -1), index.get(int(parts[-2]), -1), index.get(int(parts[-1]), -1)]
        if min(tri) < 0:
            continue
        faces.append(tri)
        tags.append(int(parts[3]))
    return BoundaryMesh(np.array(verts), np.array(faces), np.array(tags))


def write_gmsh22(path: str, mesh: BoundaryMesh) -> None:
    """Write a Gmsh 2.2 ASCII file that :func:`load_gmsh22_with_tags` (and the
    reference's loader) reads back, so generated meshes feed either path."""
    with open(path, "w", encoding="utf-8") as fh:
        fh.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n")
        fh.write(f"{mesh.num_vertices}\n")
        for i, v in enumerate(mesh.vertices):
            fh.write(f"{i + 1} {v[0]:.17e} {v[1]:.17e} {v[2]:.17e}\n")
        fh.write("$EndNodes\n$Elements\n")
        fh.write(f"{mesh.num_faces}\n")
        for i, (f, t) in enumerate(zip(mesh.faces, mesh.physical_tags)):
            fh.write(f"{i + 1} 2 2 {int(t)} {int(t)} {f[0] + 1} {f[1] + 1} {f[2] + 1}\n")
        fh.write("$EndElements\n")


_ICO_FACES = np.array([
    (1, 12, 6), (1, 6, 2), (1, 2, 8), (1, 8, 11), (1, 11, 12),
    (2, 6, 10), (6, 12, 5), (12, 11, 3), (11, 8, 7), (8, 2, 9),
    (4, 10, 5), (4, 5, 3), (4, 3, 7), (4, 7, 9), (4, 9, 10),
    (5, 10, 6), (3, 5, 12), (7, 3, 11), (9, 7, 8), (10, 9, 2),
], dtype=np.int64) - 1


def reference_sphere(radius: float, subdivisions: int, centre=(0.0, 0.0, 0.0), tag: int = 1) -> BoundaryMesh:
    """Icosphere: unit icosahedron, midpoint subdivision ``subdivisions``
    times, vertices projected to ``radius`` about ``centre``, every winding
    oriented outward (``tests/analytical_exterior_tests.jl:4-66``).

    ``subdivisions=3`` gives 1,280 faces / 642 vertices; ``5`` gives
    20,480 faces / 10,242 vertices.
    """
    if subdivisions < 0:
        raise ValueError("Icosphere subdivision level must be >= 0.")
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    verts = [np.array(v, dtype=np.float64) for v in (
        (-1, phi, 0), (1, phi, 0), (-1, -phi, 0), (1, -phi, 0),
        (0, -1, phi), (0, 1, phi), (0, -1, -phi), (0, 1, -phi),
        (phi, 0, -1), (phi, 0, 1), (-phi, 0, -1), (-phi, 0, 1))]
    faces = [tuple(int(x) for x in f) for f in _ICO_FACES]
    for _ in range(subdivisions):
        mids: dict = {}

        def midpoint(a: int, b: int) -> int:
            key = (a, b) if a < b else (b, a)
            idx = mids.get(key)
            if idx is not None:
                return idx
            verts.append((verts[a] + verts[b]) / 2.0)
            mids[key] = len(verts) - 1
            return len(verts) - 1

        nxt = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            nxt.extend([(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)])
        faces = nxt
    centre = np.asarray(centre, dtype=np.float64)
    V = np.array(verts)
    V = centre + radius * (V / np.linalg.norm(V, axis=1)[:, None])
    Fa = np.array(faces, dtype=np.int64)
    v1, v2, v3 = V[Fa[:, 0]], V[Fa[:, 1]], V[Fa[:, 2]]
    outward = (v1 + v2 + v3) / 3.0 - centre
    flip = np.einsum("ij,ij->i", np.cross(v2 - v1, v3 - v1), outward) < 0
    Fa[flip] = Fa[flip][:, [0, 2, 1]]
    mesh = BoundaryMesh(V, Fa, np.full(len(Fa), tag))
    if np.any(np.einsum("ij,ij->i", mesh.normals, mesh.centroids - centre) <= 0):
        raise RuntimeError("icosphere has an inward normal")
    return mesh


def oscillating_sphere(refinements: int, radius: float, tag: int = 2) -> BoundaryMesh:
    """Octahedron refined by normalised midpoints ``refinements`` times
    (``tests/axial_source_tests.jl:71-88``): 128 faces at 2, 512 at 3."""
    verts = [np.array(v, dtype=np.float64) for v in
             ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1))]
    faces = [(0, 2, 4), (2, 1, 4), (1, 3, 4), (3, 0, 4), (2, 0, 5), (1, 2, 5), (3, 1, 5), (0, 3, 5)]
    for _ in range(refinements):
        mids: dict = {}

        def midpoint(a: int, b: int) -> int:
            key = (min(a, b), max(a, b))
            if key not in mids:
                v = verts[a] + verts[b]
                verts.append(v / np.linalg.norm(v))
                mids[key] = len(verts) - 1
            return mids[key]

        ref = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            ref.extend([(a, ab, ca), (ab, b, bc), (ca, bc, c), (ab, bc, ca)])
        faces = ref
    return BoundaryMesh(radius * np.array(verts), np.array(faces), np.full(len(faces), tag))


def rounded_box_enclosure(n_faces_target: int, size=(0.2, 0.3, 0.25), fillet: float = 0.02,
                          piston_radius: float = 0.05, jitter: float = 0.05, seed: int = 0,
                          body_tag: int = 1, piston_tag: int = 2) -> BoundaryMesh:
    """Loudspeaker-like enclosure: a box of ``size`` (x width, y height,
    z depth) with edges and corners rounded to ``fillet``, and a circular
    piston of ``piston_radius`` centred on the front face (z = +depth / 2)
    whose faces carry ``piston_tag``.

    Triangulated at one target edge length so that there are about
    ``n_faces_target`` triangles: each face of a cube is cut into a grid whose
    cell counts follow the box's extents, every cell into two triangles, and
    each lattice point b (in box coordinates) is mapped onto the rounded box by
    p = c + fillet (b - c) / |b - c|, c = b clamped to the box shrunk by the
    fillet.  That gives flat faces, cylindrical edges and spherical corners.
    Vertices are jittered by up to ``jitter`` x the edge length along the
    grid directions free on their cube face (seeded), which keeps them on the
    surface; windings are outward."""
    half = np.asarray(size, dtype=np.float64) / 2.0
    area = 2.0 * (size[0] * size[1] + size[1] * size[2] + size[0] * size[2])
    h = math.sqrt(2.0 * area / n_faces_target)
    n = [max(2, int(round(s / h))) for s in size]
    index: dict = {}
    lattice: list = []

    def vid(i, j, k):
        key = (i, j, k)
        if key not in index:
            index[key] = len(lattice)
            lattice.append(key)
        return index[key]

    faces = []
    for axis in range(3):
        u, v = [a for a in range(3) if a != axis]
        for side in (0, n[axis]):
            outward = 1.0 if side else -1.0
            for a in range(n[u]):
                for b in range(n[v]):
                    corner = []
                    for du, dv in ((0, 0), (1, 0), (1, 1), (0, 1)):
                        ijk = [0, 0, 0]
                        ijk[axis], ijk[u], ijk[v] = side, a + du, b + dv
                        corner.append(vid(*ijk))
                    # (u, v, axis) is right-handed for axis = 0, 2 and left-handed for 1
                    right = (axis != 1) == (outward > 0)
                    t1, t2 = (corner[0], corner[1], corner[2]), (corner[0], corner[2], corner[3])
                    if not right:
                        t1, t2 = (corner[0], corner[2], corner[1]), (corner[0], corner[3], corner[2])
                    faces.extend([t1, t2])
    L = np.asarray(lattice, dtype=np.float64)
    rng = np.random.default_rng(seed)
    step = np.array([2.0 / n[a] for a in range(3)])  # lattice spacing in cube coordinates
    cube = L * step - 1.0
    free = (L > 0) & (L < np.asarray(n))  # coordinates not pinned to a cube face
    cube += free * rng.uniform(-jitter, jitter, size=cube.shape) * step
    box = cube * half
    inner = np.clip(box, -(half - fillet), half - fillet)
    d = box - inner
    dl = np.linalg.norm(d, axis=1)
    verts = inner + fillet * d / dl[:, None]
    F = np.asarray(faces, dtype=np.int64)
    c = verts[F].mean(axis=1)
    tags = np.full(len(F), body_tag)
    front = (c[:, 2] > half[2] - 1e-9) & (np.hypot(c[:, 0], c[:, 1]) <= piston_radius)
    tags[front] = piston_tag
    mesh = BoundaryMesh(verts, F, tags)
    # outward: the normals point away from the box's centre and the volume is positive
    vol = np.einsum("ij,ij->i", verts[F[:, 0]], np.cross(verts[F[:, 1]], verts[F[:, 2]])).sum() / 6.0
    if vol <= 0 or np.any(np.einsum("ij,ij->i", mesh.normals, mesh.centroids) <= 0):
        raise RuntimeError("rounded box has an inward normal")
    return mesh


def fibonacci_sphere(n_points: int, radius: float) -> np.ndarray:
    """``fibonacci_sphere`` of ``src/BeatEngineCore.jl:828-840`` (``n x 3``)."""
    golden = math.pi * (3.0 - math.sqrt(5.0))
    i = np.arange(n_points, dtype=np.float64)
    z = 1.0 - (2.0 * i + 1.0) / n_points
    r = np.sqrt(1.0 - z * z)
    phi = i * golden
    return np.stack([r * np.cos(phi) * radius, r * np.sin(phi) * radius, z * radius], axis=1)


def arc_points(n: int, radius: float) -> np.ndarray:
    """``n`` points on a meridian arc of ``radius``, theta from 0 to 180 deg
    (x-z plane)."""
    th = np.linspace(0.0, math.pi, n)
    return np.stack([radius * np.sin(th), np.zeros(n), radius * np.cos(th)], axis=1)


def equator_meridian_directions(n_equator: int = 360, n_meridian: int = 181) -> np.ndarray:
    """Unit far-field directions: ``n_equator`` on the equator (1 deg steps for
    360) followed by ``n_meridian`` on the x-z meridian, theta 0..180 deg."""
    ph = np.arange(n_equator) * (2.0 * math.pi / n_equator)
    eq = np.stack([np.cos(ph), np.sin(ph), np.zeros(n_equator)], axis=1)
    th = np.linspace(0.0, math.pi, n_meridian)
    me = np.stack([np.sin(th), np.zeros(n_meridian), np.cos(th)], axis=1)
    return np.concatenate([eq, me], axis=0)


def uv_sphere_patch(radius: float, n_theta: int, n_phi: int, phi0: float, phi1: float,
                    centre=(0.0, 0.0, 0.0), tag: int = 1) -> BoundaryMesh:
    """Latitude-longitude patch of a sphere: polar angle 0..pi in n_theta
    bands, azimuth phi0..phi1 in n_phi bands (both poles included, outward
    normals).  With phi in [-pi/2, pi/2] it is the x >= 0 half; in [0, pi/2]
    the x, y >= 0 quarter; the boundary meridians lie exactly on the planes."""
    c = np.asarray(centre, dtype=float)
    verts = [c + (0.0, 0.0, radius)]
    full = abs((phi1 - phi0) - 2 * np.pi) < 1e-12
    ncol = n_phi if full else n_phi + 1
    for i in range(1, n_theta):
        th = np.pi * i / n_theta
        for j in range(ncol):
            ph = phi0 + (phi1 - phi0) * j / n_phi
            x, y = np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph)
            # exact zeros on the planes x = 0 / y = 0 of the patch boundary
            if abs(np.cos(ph)) < 1e-12:
                x = 0.0
            if abs(np.sin(ph)) < 1e-12:
                y = 0.0
            verts.append(c + radius * np.array([x, y, np.cos(th)]))
    verts.append(c + (0.0, 0.0, -radius))
    V = len(verts)

    def ring(i, j):
        return 1 + (i - 1) * ncol + (j % ncol if full else j)

    faces = []
    for j in range(n_phi):
        faces.append((0, ring(1, j), ring(1, j + 1)))
        faces.append((V - 1, ring(n_theta - 1, j + 1), ring(n_theta - 1, j)))
    for i in range(1, n_theta - 1):
        for j in range(n_phi):
            a, b, d, e = ring(i, j), ring(i, j + 1), ring(i + 1, j), ring(i + 1, j + 1)
            faces.append((a, d, e))
            faces.append((a, e, b))
    verts = np.array(verts)
    faces = np.array(faces, dtype=np.int64)
    # orient outward
    for f in range(len(faces)):
        p0, p1, p2 = verts[faces[f]]
        n = np.cross(p1 - p0, p2 - p0)
        if np.dot(n, (p0 + p1 + p2) / 3 - c) < 0:
            faces[f] = faces[f][[0, 2, 1]]
    return BoundaryMesh(verts, faces, np.full(len(faces), tag, dtype=np.int64))


def mirror(mesh: BoundaryMesh, axis: int, tol: float = 1e-12) -> BoundaryMesh:
    """The mesh together with its mirror image across the plane x[axis] = 0:
    vertices on the plane are shared, mirrored faces are reversed so that the
    normals stay outward.  Mirrored copies keep the order of the originals
    (vertex v at V + v unless it lies on the plane; face f at F + f)."""
    v = np.asarray(mesh.vertices, dtype=float)
    V = v.shape[0]
    on = np.abs(v[:, axis]) <= tol
    idx = np.empty(V, dtype=np.int64)
    extra = []
    for i in range(V):
        if on[i]:
            idx[i] = i
        else:
            idx[i] = V + len(extra)
            w = v[i].copy()
            w[axis] = -w[axis]
            extra.append(w)
    verts = np.vstack([v, np.array(extra)]) if extra else v.copy()
    f = np.asarray(mesh.faces)
    mf = idx[f][:, [0, 2, 1]]
    return BoundaryMesh(verts, np.vstack([f, mf]), np.concatenate([mesh.physical_tags, mesh.physical_tags]))
