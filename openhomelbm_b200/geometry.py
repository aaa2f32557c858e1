"""Host-side geometry preparation for the solids, without MuJoCo or trimesh installed.

3D (replaces envs/lbm3d/mjcf_parser.py): `parse_mjcf` reads an MJCF file's body tree, joints
and geoms (15-300) and meshes every geom (box, sphere, ellipsoid, cylinder, capsule, mesh file)
in its body's frame; `get_body_world_positions` (341-372), `parse_mjcf_to_meshes` (375-393)
and `parse_mjcf_as_urdf_format` (396-460) keep their output layouts. Meshes are `TriMesh`
objects (vertices (V, 3), faces (F, 3)), which `LBM_Solver3D.create_solid_from_mesh` takes
directly. The primitives are this module's own tessellations of the same shapes (an
icosphere of 3 subdivisions, 32-section cylinders, 16 x 8 capsules), not trimesh's vertex
lists.

2D (replaces envs/lbm/mujoco_to_lbm.py): `get_geom_vertices_2d` (152-282),
`get_body_vertices_2d` (285-316), `extract_mesh_projection_2d` (6-42), `resample_polygon`
(45-98), `compute_convex_hull_2d` (319-341) and `extract_lbm_polygon_from_mujoco` (344-398)
project a body's geoms onto the xy plane for `HomeFlow.configure_solid`. They read a MuJoCo
model and data through the attributes the reference uses (`model.geom(name).id`,
`geom_type`, `geom_size`, `geom_rbound`, `geom_dataid`, `geom_bodyid`, `mesh_vertadr`,
`mesh_vertnum`, `mesh_vert`, `data.geom_xpos`, `data.geom_xmat`, `model.body(name).id`,
`data.xipos`, `data.xquat`), so a real mujoco.MjModel / MjData works and so does any object
with those fields.
"""
from __future__ import annotations

import math
import os
import struct
import xml.etree.ElementTree as ET
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence

import numpy as np

# MuJoCo's geom type codes (mjtGeom)
GEOM_PLANE, GEOM_HFIELD, GEOM_SPHERE, GEOM_CAPSULE, GEOM_ELLIPSOID, GEOM_CYLINDER, GEOM_BOX, GEOM_MESH = range(8)


# ----------------------------------------------------------------------------- meshes
@dataclass
class TriMesh:
    """A triangle mesh: vertices (V, 3) float64, faces (F, 3) int64 (counter-clockwise seen
    from outside for the primitives)."""

    vertices: np.ndarray
    faces: np.ndarray

    def copy(self) -> "TriMesh":
        return TriMesh(self.vertices.copy(), self.faces.copy())

    @staticmethod
    def concatenate(meshes: Sequence["TriMesh"]) -> "TriMesh":
        verts, faces, base = [], [], 0
        for m in meshes:
            verts.append(m.vertices)
            faces.append(m.faces + base)
            base += len(m.vertices)
        return TriMesh(np.concatenate(verts), np.concatenate(faces))


def box_mesh(half_size) -> TriMesh:
    """Box with the given half extents, centred at the origin (8 vertices, 12 triangles)."""
    hx, hy, hz = (float(v) for v in half_size)
    v = np.array([[x, y, z] for x in (-hx, hx) for y in (-hy, hy) for z in (-hz, hz)], np.float64)
    # faces of the cube in the vertex numbering 4x + 2y + z (each coordinate 0 low, 1 high)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    f = []
    for a, b, c, d in quads:
        f += [(a, b, c), (a, c, d)]
    return TriMesh(v, np.array(f, np.int64))


def icosphere(subdivisions: int = 3, radius: float = 1.0) -> TriMesh:
    """Sphere from a regular icosahedron whose triangles are split in four `subdivisions` times,
    the new vertices pushed onto the sphere (10 4^s + 2 vertices, 20 4^s triangles)."""
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    verts = [np.array(p, np.float64) / math.sqrt(1 + t * t) for p in v]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11),
             (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    for _ in range(int(subdivisions)):
        mid: Dict = {}

        def midpoint(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = verts[a] + verts[b]
                verts.append(p / np.linalg.norm(p))
                mid[key] = len(verts) - 1
            return mid[key]

        new = []
        for a, b, c in faces:
            ab, bc, ca = midpoint(a, b), midpoint(b, c), midpoint(c, a)
            new += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        faces = new
    return TriMesh(np.array(verts) * float(radius), np.array(faces, np.int64))


def cylinder_mesh(radius: float, height: float, sections: int = 32) -> TriMesh:
    """Closed cylinder along z, centred at the origin."""
    a = 2 * np.pi * np.arange(sections) / sections
    ring = np.stack([radius * np.cos(a), radius * np.sin(a)], 1)
    h = height / 2
    v = np.concatenate([np.c_[ring, np.full(sections, -h)], np.c_[ring, np.full(sections, h)], [[0, 0, -h], [0, 0, h]]])
    f = []
    lo_c, hi_c = 2 * sections, 2 * sections + 1
    for i in range(sections):
        j = (i + 1) % sections
        f += [(i, j, sections + j), (i, sections + j, sections + i), (lo_c, j, i), (hi_c, sections + i, sections + j)]
    return TriMesh(v.astype(np.float64), np.array(f, np.int64))


def capsule_mesh(height: float, radius: float, count=(16, 8)) -> TriMesh:
    """Capsule along z: two hemispheres of `radius` whose centres are `height` apart, joined by
    a cylinder; count = (meridians, rings per hemisphere)."""
    n_lon, n_lat = int(count[0]), int(count[1])
    a = 2 * np.pi * np.arange(n_lon) / n_lon
    h = height / 2
    rings = []  # (ring radius, z): the upper hemisphere from the pole to its equator, then the lower
    for k in range(1, n_lat + 1):
        th = (np.pi / 2) * k / n_lat
        rings.append((radius * math.sin(th), h + radius * math.cos(th)))
    for k in range(n_lat):
        ph = (np.pi / 2) * k / n_lat
        rings.append((radius * math.cos(ph), -h - radius * math.sin(ph)))
    verts = [[0.0, 0.0, h + radius]]
    for r, z in rings:
        verts += [[r * math.cos(x), r * math.sin(x), z] for x in a]
    verts.append([0.0, 0.0, -h - radius])
    start = [1 + n_lon * k for k in range(len(rings))]
    f = [(0, start[0] + i, start[0] + (i + 1) % n_lon) for i in range(n_lon)]
    for r0, r1 in zip(start[:-1], start[1:]):
        for i in range(n_lon):
            j = (i + 1) % n_lon
            f += [(r0 + i, r1 + i, r1 + j), (r0 + i, r1 + j, r0 + j)]
    bottom, last = len(verts) - 1, start[-1]
    f += [(bottom, last + (i + 1) % n_lon, last + i) for i in range(n_lon)]
    return TriMesh(np.array(verts, np.float64), np.array(f, np.int64))


def load_mesh_file(path: str) -> TriMesh:
    """A triangle mesh from an OBJ (polygons fanned into triangles) or STL (ASCII or binary) file."""
    ext = os.path.splitext(path)[1].lower()
    if ext == ".obj":
        v, f = [], []
        with open(path) as fh:
            for line in fh:
                p = line.split()
                if not p:
                    continue
                if p[0] == "v":
                    v.append([float(x) for x in p[1:4]])
                elif p[0] == "f":
                    idx = [int(q.split("/")[0]) for q in p[1:]]
                    idx = [i - 1 if i > 0 else len(v) + i for i in idx]
                    f += [(idx[0], idx[k], idx[k + 1]) for k in range(1, len(idx) - 1)]
        return TriMesh(np.array(v, np.float64), np.array(f, np.int64))
    if ext == ".stl":
        with open(path, "rb") as fh:
            data = fh.read()
        if len(data) >= 84 and len(data) == 84 + 50 * struct.unpack("<I", data[80:84])[0]:
            n = struct.unpack("<I", data[80:84])[0]
            rec = np.frombuffer(data, dtype=np.dtype([("n", "<f4", 3), ("v", "<f4", (3, 3)), ("a", "<u2")]), count=n,
                                offset=84)
            tri = rec["v"].astype(np.float64)
        else:
            tri = np.array([[float(x) for x in line.split()[1:4]] for line in data.decode().splitlines()
                            if line.strip().startswith("vertex")]).reshape(-1, 3, 3)
        return TriMesh(tri.reshape(-1, 3), np.arange(len(tri) * 3, dtype=np.int64).reshape(-1, 3))
    raise ValueError(f"unsupported mesh file {path} (OBJ or STL)")


# ----------------------------------------------------------------------------- rotations
def quat_mul(a, b):
    """Hamilton product of quaternions (w, x, y, z)."""
    aw, ax, ay, az = a
    bw, bx, by, bz = b
    return np.array([aw * bw - ax * bx - ay * by - az * bz, aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx, aw * bz + ax * by - ay * bx + az * bw])


def euler_to_quat(euler_deg) -> np.ndarray:
    """(w, x, y, z) of rotations about the fixed x, then y, then z axes by the given degrees
    (the convention the reference's parser applies to MJCF `euler`)."""
    q = np.array([1.0, 0.0, 0.0, 0.0])
    for axis, ang in enumerate(np.radians(np.asarray(euler_deg, np.float64))):
        r = np.zeros(4)
        r[0] = math.cos(ang / 2)
        r[1 + axis] = math.sin(ang / 2)
        q = quat_mul(r, q)
    return q


def quat_to_matrix(q) -> np.ndarray:
    w, x, y, z = np.asarray(q, np.float64) / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                     [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                     [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])


def _rotation_onto(direction) -> np.ndarray:
    """A rotation taking +z onto the unit vector `direction`."""
    z = np.array([0.0, 0.0, 1.0])
    d = np.asarray(direction, np.float64)
    c = float(np.dot(z, d))
    if c > 1 - 1e-12:
        return np.eye(3)
    if c < -1 + 1e-12:
        return np.diag([1.0, -1.0, -1.0])
    axis = np.cross(z, d)
    axis /= np.linalg.norm(axis)
    ang = math.acos(max(-1.0, min(1.0, c)))
    k = np.array([[0, -axis[2], axis[1]], [axis[2], 0, -axis[0]], [-axis[1], axis[0], 0]])
    return np.eye(3) + math.sin(ang) * k + (1 - math.cos(ang)) * (k @ k)


def rpy_from_quat(q) -> np.ndarray:
    """Angles (radians) of rotations about the fixed x, y, z axes giving the quaternion q."""
    m = quat_to_matrix(q)
    return np.array([math.atan2(m[2, 1], m[2, 2]), math.asin(max(-1.0, min(1.0, -m[2, 0]))),
                     math.atan2(m[1, 0], m[0, 0])])


# ----------------------------------------------------------------------------- MJCF
def _vec(elem, name, default):
    return np.array([float(x) for x in elem.get(name, default).split()], np.float64)


def _pose(elem):
    pos = _vec(elem, "pos", "0 0 0")
    quat = _vec(elem, "quat", "1 0 0 0")
    if elem.get("euler") is not None:
        quat = euler_to_quat(_vec(elem, "euler", "0 0 0"))
    return pos, quat


def _resolve(uri: Optional[str], search: List[str]) -> Optional[str]:
    if uri is None:
        return None
    if os.path.isabs(uri):
        return uri if os.path.exists(uri) else None
    for p in search:
        full = os.path.join(p, uri)
        if os.path.exists(full):
            return full
    return None


def geom_mesh(geom: ET.Element, assets: Dict, search: List[str]) -> Optional[TriMesh]:
    """The mesh of one MJCF geom in its body's frame (mjcf_parser.py:155-299), or None."""
    kind = geom.get("type", "sphere")
    pos, quat = _pose(geom)
    size = [float(x) for x in geom.get("size", "0.5 0.5 0.5").split()]
    fromto = geom.get("fromto")
    if kind in ("cylinder", "capsule") and fromto is not None:
        ft = np.array([float(x) for x in fromto.split()])
        p1, p2 = ft[:3], ft[3:]
        length = float(np.linalg.norm(p2 - p1))
        m = cylinder_mesh(size[0], length) if kind == "cylinder" else capsule_mesh(length, size[0])
        d = (p2 - p1) / length if length > 1e-6 else np.array([0.0, 0.0, 1.0])
        m.vertices = m.vertices @ _rotation_onto(d).T + (p1 + p2) / 2
        return m
    if kind == "box":
        m = box_mesh(size[:3] if len(size) >= 3 else [size[0]] * 3)
    elif kind == "sphere":
        m = icosphere(3, size[0])
    elif kind == "ellipsoid":
        m = icosphere(3, 1.0)
        m.vertices = m.vertices * np.array((size + size * 3)[:3])
    elif kind == "cylinder":
        m = cylinder_mesh(size[0], 2 * (size[1] if len(size) > 1 else size[0]))
    elif kind == "capsule":
        m = capsule_mesh(2 * (size[1] if len(size) > 1 else size[0]), size[0])
    elif kind == "mesh":
        asset = assets.get(geom.get("mesh"))
        path = _resolve(asset["file"], search) if asset else None
        if path is None:
            return None
        m = load_mesh_file(path)
        m.vertices = m.vertices * asset["scale"]
    else:
        return None
    m.vertices = m.vertices @ quat_to_matrix(quat).T + pos
    return m


def parse_mjcf(mjcf_path: str, mesh_search_paths: Optional[List[str]] = None) -> Dict:
    """{'model_name', 'bodies': [{'name', 'meshes', 'combined_mesh', 'parent', 'pos', 'quat'}],
    'joints': [{'name', 'type', 'body', 'axis', 'range'}]} (mjcf_parser.py:15-95); bodies
    without a meshable geom are left out, as in the reference."""
    if not os.path.exists(mjcf_path):
        raise FileNotFoundError(f"MJCF file not found: {mjcf_path}")
    search = list(mesh_search_paths or [])
    base = os.path.dirname(os.path.abspath(mjcf_path))
    if base not in search:
        search.insert(0, base)
    root = ET.parse(mjcf_path).getroot()
    comp = root.find("compiler")
    if comp is not None and comp.get("meshdir") is not None:
        md = os.path.normpath(os.path.join(base, comp.get("meshdir")))
        if md not in search:
            search.insert(0, md)
    assets = {}
    if root.find("asset") is not None:
        for m in root.find("asset").findall("mesh"):
            assets[m.get("name")] = {"file": m.get("file"), "scale": _vec(m, "scale", "1 1 1")}
    bodies: List[Dict] = []
    joints: List[Dict] = []

    def walk(elem, parent):
        for b in elem.findall("body"):
            name = b.get("name", f"body_{len(bodies)}")
            pos, quat = _pose(b)
            meshes = [m for m in (geom_mesh(g, assets, search) for g in b.findall("geom")) if m is not None]
            if meshes:
                bodies.append({"name": name, "meshes": meshes,
                               "combined_mesh": meshes[0] if len(meshes) == 1 else TriMesh.concatenate(meshes),
                               "parent": parent, "pos": pos, "quat": quat})
            for j in b.findall("joint"):
                rng = [float(x) for x in j.get("range", "-180 180").split()]
                joints.append({"name": j.get("name", f"joint_{name}"), "type": j.get("type", "hinge"), "body": name,
                               "axis": _vec(j, "axis", "0 0 1"),
                               "range": (rng[0], rng[1]) if len(rng) >= 2 else (-180.0, 180.0)})
            walk(b, name)

    if root.find("worldbody") is not None:
        walk(root.find("worldbody"), None)
    return {"model_name": root.get("model", "unnamed_model"), "bodies": bodies, "joints": joints}


def get_body_world_positions(mjcf_data: Dict) -> Dict[str, np.ndarray]:
    """Each body's origin in the world frame, composing its ancestors' poses (341-372)."""
    by_name = {b["name"]: b for b in mjcf_data["bodies"]}
    out = {}
    for b in mjcf_data["bodies"]:
        p, parent = b["pos"].copy(), b["parent"]
        while parent is not None and parent in by_name:
            pb = by_name[parent]
            p = quat_to_matrix(pb["quat"]) @ p + pb["pos"]
            parent = pb["parent"]
        out[b["name"]] = p
    return out


def parse_mjcf_to_meshes(mjcf_path: str, mesh_search_paths: Optional[List[str]] = None) -> Dict[str, TriMesh]:
    """{body name: combined mesh} (375-393)."""
    return {b["name"]: b["combined_mesh"] for b in parse_mjcf(mjcf_path, mesh_search_paths)["bodies"]}


def parse_mjcf_as_urdf_format(mjcf_path: str) -> Dict:
    """The parse_urdf layout (396-460): links with their meshes (unit mass and 0.01 I inertia,
    the reference's defaults) and a revolute joint about z per parent-child pair."""
    data = parse_mjcf(mjcf_path)
    links = [{"name": b["name"], "mesh": b["combined_mesh"], "origin_xyz": np.zeros(3), "origin_rpy": np.zeros(3),
              "mass": 1.0, "inertia": np.eye(3) * 0.01} for b in data["bodies"]]
    joints = [{"name": f"joint_{b['parent']}_{b['name']}", "type": "revolute", "parent": b["parent"],
               "child": b["name"], "origin_xyz": b["pos"], "origin_rpy": rpy_from_quat(b["quat"]),
               "axis": np.array([0, 0, 1])} for b in data["bodies"] if b["parent"] is not None]
    return {"robot_name": data["model_name"], "links": links, "joints": joints}


# ----------------------------------------------------------------------------- 2D polygons
def compute_convex_hull_2d(vertices: np.ndarray) -> np.ndarray:
    """Convex hull of 2D points, counter-clockwise (Andrew's monotone chain); fewer than 3
    points are returned as they are."""
    v = np.asarray(vertices, np.float64)
    if len(v) < 3:
        return v
    pts = sorted(map(tuple, v))

    def cross(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])

    lower, upper = [], []
    for p in pts:
        while len(lower) >= 2 and cross(lower[-2], lower[-1], p) <= 0:
            lower.pop()
        lower.append(p)
    for p in reversed(pts):
        while len(upper) >= 2 and cross(upper[-2], upper[-1], p) <= 0:
            upper.pop()
        upper.append(p)
    return np.array(lower[:-1] + upper[:-1])


def resample_polygon(vertices: np.ndarray, n_samples: int) -> np.ndarray:
    """n_samples points equally spaced along the boundary of the points' convex hull (45-98);
    a degenerate outline becomes a circle of radius 0.1."""
    v = np.asarray(vertices, np.float64)
    if len(v) < 2:
        return v
    if len(v) >= 3:
        v = compute_convex_hull_2d(v)
    seg = np.diff(np.vstack([v, v[:1]]), axis=0)
    length = np.linalg.norm(seg, axis=1)
    cum = np.concatenate([[0.0], np.cumsum(length)])
    if cum[-1] < 1e-10:
        a = np.linspace(0, 2 * np.pi, n_samples, endpoint=False)
        return np.stack([0.1 * np.cos(a), 0.1 * np.sin(a)], 1)
    s = np.linspace(0, cum[-1], n_samples, endpoint=False)
    k = np.minimum(np.searchsorted(cum[1:], s), len(v) - 1)
    t = np.clip((s - cum[k]) / (length[k] + 1e-10), 0, 1)
    return v[k] + t[:, None] * seg[k]


def extract_mesh_projection_2d(model, geom_id: int, n_samples: Optional[int] = None) -> np.ndarray:
    """xy of a mesh geom's vertices, resampled to n_samples if given (6-42)."""
    dataid = int(model.geom_dataid[geom_id])
    if dataid < 0:
        a = np.linspace(0, 2 * np.pi, n_samples or 20, endpoint=False)
        return np.stack([0.1 * np.cos(a), 0.1 * np.sin(a)], 1)
    adr, num = int(model.mesh_vertadr[dataid]), int(model.mesh_vertnum[dataid])
    v2 = np.asarray(model.mesh_vert[adr:adr + num]).reshape(-1, 3)[:, :2]
    if n_samples is not None and len(v2) != n_samples:
        v2 = resample_polygon(v2, n_samples)
    return v2


def _circle(r, n):
    a = np.linspace(0, 2 * np.pi, n, endpoint=False)
    return np.stack([r * np.cos(a), r * np.sin(a)], 1)


def get_geom_vertices_2d(model, data, geom_name: str, n_samples: int = 20) -> np.ndarray:
    """A geom's outline in the xy plane at its current pose (152-282): box corners, circles for
    spheres and cylinders, an ellipse for ellipsoids, a stadium for capsules (turned towards
    the xy projection of their axis), the mesh's xy vertices for meshes."""
    gid = model.geom(geom_name).id
    kind = int(model.geom_type[gid])
    size = np.asarray(model.geom_size[gid], np.float64)
    pos = np.asarray(data.geom_xpos[gid], np.float64)[:2]
    mat = np.asarray(data.geom_xmat[gid], np.float64).reshape(3, 3)
    angle = math.atan2(mat[1, 0], mat[0, 0])
    if kind == GEOM_BOX:
        hx, hy = size[0], size[1]
        local = np.array([[-hx, -hy], [hx, -hy], [hx, hy], [-hx, hy]])
    elif kind in (GEOM_SPHERE, GEOM_CYLINDER):
        local = _circle(size[0], n_samples)
    elif kind == GEOM_CAPSULE:
        r, half = size[0], size[1]
        if half < 1e-6:
            half = max(float(model.geom_rbound[gid]) - r, 0.0)
        axis2 = mat[:2, 2]
        n = np.linalg.norm(axis2)
        turn = math.atan2(axis2[0] / n, axis2[1] / n) if n > 1e-6 else 0.0  # from +y
        h = n_samples // 2
        top = np.linspace(0, np.pi, h, endpoint=False)
        bot = np.linspace(np.pi, 2 * np.pi, h, endpoint=False)
        caps = np.vstack([np.stack([r * np.cos(top), half + r * np.sin(top)], 1),
                          np.stack([r * np.cos(bot), -half + r * np.sin(bot)], 1)])
        c, s = math.cos(turn), math.sin(turn)
        local = caps @ np.array([[c, -s], [s, c]]).T
    elif kind == GEOM_ELLIPSOID:
        a = np.linspace(0, 2 * np.pi, n_samples, endpoint=False)
        local = np.stack([size[0] * np.cos(a), size[1] * np.sin(a)], 1)
    elif kind == GEOM_MESH:
        local = extract_mesh_projection_2d(model, gid, n_samples)
    else:
        local = _circle(0.1, n_samples)
    c, s = math.cos(angle), math.sin(angle)
    return local @ np.array([[c, -s], [s, c]]).T + pos


def get_body_vertices_2d(model, data, body_name: str, n_samples: int = 20) -> np.ndarray:
    """The outlines of all the body's geoms, stacked (285-316)."""
    bid = model.body(body_name).id
    out = [get_geom_vertices_2d(model, data, model.geom(g).name, n_samples)
           for g in range(int(model.ngeom)) if int(model.geom_bodyid[g]) == bid]
    if not out:
        raise ValueError(f"body '{body_name}' has no geoms")
    return np.vstack(out)


def extract_lbm_polygon_from_mujoco(model, data, body_or_geom_name: str, n_samples: int = 20,
                                    use_convex_hull: bool = True, normalize: bool = True,
                                    is_body: bool = True) -> Dict:
    """{'vertices', 'position', 'angle'} for HomeFlow.configure_solid (344-398): the body's (or
    geom's) outline, its convex hull, centred on the vertices' mean; the pose's xy and yaw."""
    if is_body:
        v = get_body_vertices_2d(model, data, body_or_geom_name, n_samples)
        bid = model.body(body_or_geom_name).id
        position = np.asarray(data.xipos[bid], np.float64)[:2]
        w, x, y, z = np.asarray(data.xquat[bid], np.float64)
        angle = math.atan2(2 * (w * z + x * y), 1 - 2 * (y * y + z * z))
    else:
        v = get_geom_vertices_2d(model, data, body_or_geom_name, n_samples)
        gid = model.geom(body_or_geom_name).id
        position = np.asarray(data.geom_xpos[gid], np.float64)[:2]
        mat = np.asarray(data.geom_xmat[gid], np.float64).reshape(3, 3)
        angle = math.atan2(mat[1, 0], mat[0, 0])
    if use_convex_hull and len(v) > 3:
        v = compute_convex_hull_2d(v)
    if normalize:
        v = v - v.mean(axis=0)
    return {"vertices": v, "position": position, "angle": angle}
