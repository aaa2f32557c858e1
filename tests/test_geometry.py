"""Host-side geometry preparation (openhomelbm_b200.geometry): primitive meshes, MJCF parsing
and the xy projections of MuJoCo geoms (through a stand-in model / data with MuJoCo's field
names; MuJoCo itself is not installed). No GPU."""
import math
import struct
from types import SimpleNamespace

import numpy as np
import pytest

from openhomelbm_b200 import geometry as g


def _volume(m):
    v = m.vertices[m.faces]
    return float(np.einsum("ij,ij->i", v[:, 0], np.cross(v[:, 1], v[:, 2])).sum() / 6)


def _closed(m):
    edges = {}
    for a, b, c in m.faces:
        for e in ((a, b), (b, c), (c, a)):
            edges[e] = edges.get(e, 0) + 1
    return all(edges.get((b, a), 0) == n for (a, b), n in edges.items())


@pytest.mark.parametrize("mesh,exact,rtol", [
    (g.box_mesh([1, 2, 3]), 48.0, 1e-12),
    (g.icosphere(3, 2.0), 4 / 3 * math.pi * 8, 0.01),
    (g.cylinder_mesh(1.0, 4.0), math.pi * 4, 0.01),
    (g.capsule_mesh(4.0, 1.0), math.pi * 4 + 4 / 3 * math.pi, 0.03),
])
def test_primitives_are_closed_outward_and_of_the_right_volume(mesh, exact, rtol):
    assert _closed(mesh)
    assert _volume(mesh) > 0
    assert abs(_volume(mesh) - exact) <= rtol * exact


def test_euler_is_about_fixed_x_then_y_then_z():
    a, b, c = 30.0, -50.0, 110.0
    rx = g.quat_to_matrix(g.euler_to_quat([a, 0, 0]))
    ry = g.quat_to_matrix(g.euler_to_quat([0, b, 0]))
    rz = g.quat_to_matrix(g.euler_to_quat([0, 0, c]))
    np.testing.assert_allclose(g.quat_to_matrix(g.euler_to_quat([a, b, c])), rz @ ry @ rx, atol=1e-12)
    np.testing.assert_allclose(rx @ [0, 1, 0], [0, math.cos(math.radians(a)), math.sin(math.radians(a))], atol=1e-12)
    np.testing.assert_allclose(np.degrees(g.rpy_from_quat(g.euler_to_quat([a, b, c]))), [a, b, c], atol=1e-9)


MJCF = """<mujoco model="swimmer">
  <compiler meshdir="assets"/>
  <asset>
    <mesh name="fin" file="fin.obj" scale="2 2 2"/>
    <mesh name="tail" file="tail.stl"/>
  </asset>
  <worldbody>
    <body name="head" pos="1 0 0" euler="0 0 90">
      <joint name="yaw0" type="hinge" axis="0 0 1" range="-30 30"/>
      <geom type="ellipsoid" size="0.3 0.2 0.1"/>
      <geom type="box" size="0.1 0.1 0.1" pos="0.3 0 0"/>
      <body name="mid" pos="0.5 0 0">
        <joint name="yaw1" axis="0 0 1"/>
        <geom type="capsule" fromto="0 0 0 0.4 0 0" size="0.05"/>
        <body name="fin" pos="0.4 0 0">
          <geom type="mesh" mesh="fin"/>
        </body>
        <body name="tail" pos="0.6 0 0" quat="0.7071068 0 0 0.7071068">
          <geom type="mesh" mesh="tail"/>
          <geom type="cylinder" size="0.02 0.1"/>
        </body>
      </body>
      <body name="nogeom" pos="0 1 0"/>
    </body>
  </worldbody>
</mujoco>
"""


def _write_assets(tmp_path):
    (tmp_path / "assets").mkdir()
    (tmp_path / "assets" / "fin.obj").write_text("v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nf 1 2 3 4\n")
    tri = np.array([[[0, 0, 0], [1, 0, 0], [0, 1, 0]], [[0, 0, 0], [0, 1, 0], [0, 0, 1]]], np.float32)
    data = b"\0" * 80 + struct.pack("<I", len(tri))
    for t in tri:
        data += struct.pack("<3f", 0, 0, 0) + t.tobytes() + struct.pack("<H", 0)
    (tmp_path / "assets" / "tail.stl").write_bytes(data)
    p = tmp_path / "model.xml"
    p.write_text(MJCF)
    return str(p)


def test_parse_mjcf_tree_geoms_and_joints(tmp_path):
    d = g.parse_mjcf(_write_assets(tmp_path))
    assert d["model_name"] == "swimmer"
    names = [b["name"] for b in d["bodies"]]
    assert names == ["head", "mid", "fin", "tail"]  # a body without geoms is left out
    by = {b["name"]: b for b in d["bodies"]}
    assert by["mid"]["parent"] == "head" and by["tail"]["parent"] == "mid" and by["head"]["parent"] is None
    np.testing.assert_allclose(by["head"]["quat"], [math.cos(math.pi / 4), 0, 0, math.sin(math.pi / 4)], atol=1e-12)
    assert len(by["head"]["meshes"]) == 2
    assert len(by["head"]["combined_mesh"].vertices) == 642 + 8
    cap = by["mid"]["combined_mesh"].vertices  # capsule from (0,0,0) to (0.4,0,0), radius 0.05
    np.testing.assert_allclose([cap[:, 0].min(), cap[:, 0].max()], [-0.05, 0.45], atol=1e-9)
    fin = by["fin"]["combined_mesh"]
    assert fin.faces.shape == (2, 3) and fin.vertices.max() == 2.0  # quad fanned, asset scale
    assert by["tail"]["combined_mesh"].faces.shape == (2 + 128, 3)
    assert [(j["name"], j["body"], j["range"]) for j in d["joints"]] == [("yaw0", "head", (-30.0, 30.0)),
                                                                          ("yaw1", "mid", (-180.0, 180.0))]


def test_world_positions_and_urdf_layout(tmp_path):
    path = _write_assets(tmp_path)
    pos = g.get_body_world_positions(g.parse_mjcf(path))
    # head turned 90 degrees about z: its child's +x offset points along +y
    np.testing.assert_allclose(pos["mid"], [1.0, 0.5, 0.0], atol=1e-12)
    np.testing.assert_allclose(pos["tail"], [1.0, 1.1, 0.0], atol=1e-12)
    meshes = g.parse_mjcf_to_meshes(path)
    assert set(meshes) == {"head", "mid", "fin", "tail"}
    u = g.parse_mjcf_as_urdf_format(path)
    assert u["robot_name"] == "swimmer" and len(u["links"]) == 4
    j = {x["child"]: x for x in u["joints"]}
    assert j["tail"]["parent"] == "mid"
    np.testing.assert_allclose(j["tail"]["origin_rpy"], [0, 0, math.pi / 2], atol=1e-6)


def _fake_model():
    """Stand-in for mujoco.MjModel / MjData with the fields the projections read."""
    th = math.radians(30)
    rz = np.array([[math.cos(th), -math.sin(th), 0], [math.sin(th), math.cos(th), 0], [0, 0, 1]])
    capsule_axis = np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], float).T  # geom z axis along world x
    names = ["box", "ball", "cap", "egg", "mesh"]
    model = SimpleNamespace(
        ngeom=5, geom_type=[g.GEOM_BOX, g.GEOM_SPHERE, g.GEOM_CAPSULE, g.GEOM_ELLIPSOID, g.GEOM_MESH],
        geom_size=[[0.2, 0.1, 0.1], [0.3, 0, 0], [0.1, 0.5, 0], [0.4, 0.2, 0.1], [1, 1, 1]],
        geom_rbound=[0, 0, 0.6, 0, 0], geom_dataid=[-1, -1, -1, -1, 0], geom_bodyid=[1, 1, 2, 2, 2],
        mesh_vertadr=[0], mesh_vertnum=[4], mesh_vert=np.array([[0, 0, 0], [1, 0, 5], [1, 1, 0], [0, 1, 9]], float))
    model.geom = lambda key: SimpleNamespace(id=names.index(key) if isinstance(key, str) else key,
                                             name=key if isinstance(key, str) else names[key])
    model.body = lambda name: SimpleNamespace(id={"a": 1, "b": 2}[name])
    data = SimpleNamespace(
        geom_xpos=np.array([[1.0, 2.0, 0], [0, 0, 0], [3, 3, 0], [0, 0, 0], [0, 0, 0]]),
        geom_xmat=np.array([rz.ravel(), np.eye(3).ravel(), capsule_axis.ravel(), np.eye(3).ravel(),
                            np.eye(3).ravel()]),
        xipos=np.array([[0, 0, 0], [1.0, 2.0, 0.5], [3, 3, 0]]),
        xquat=np.array([[1, 0, 0, 0], [math.cos(th / 2), 0, 0, math.sin(th / 2)], [1, 0, 0, 0]]))
    return model, data, rz


def test_geom_outlines_in_the_xy_plane():
    model, data, rz = _fake_model()
    box = g.get_geom_vertices_2d(model, data, "box")
    ref = np.array([[-0.2, -0.1], [0.2, -0.1], [0.2, 0.1], [-0.2, 0.1]]) @ rz[:2, :2].T + [1, 2]
    np.testing.assert_allclose(box, ref, atol=1e-12)
    ball = g.get_geom_vertices_2d(model, data, "ball", n_samples=12)
    np.testing.assert_allclose(np.linalg.norm(ball, axis=1), 0.3, atol=1e-12)
    cap = g.get_geom_vertices_2d(model, data, "cap", n_samples=20) - [3, 3]
    # the geom's z axis lies along world x: a stadium 2 (0.5 + 0.1) long
    assert cap.shape == (20, 2) and abs(np.abs(cap).max() - 0.6) < 1e-9
    mesh = g.get_geom_vertices_2d(model, data, "mesh", n_samples=8)
    assert mesh.shape == (8, 2) and mesh.min() >= -1e-12 and mesh.max() <= 1 + 1e-12
    body = g.get_body_vertices_2d(model, data, "b", n_samples=20)
    assert body.shape == (3 * 20, 2)  # capsule, ellipse, mesh resampled to n_samples


def test_hull_resampling_and_lbm_polygon():
    sq = np.array([[0, 0], [2, 0], [2, 2], [0, 2], [1, 1], [0.5, 1.5]], float)
    hull = g.compute_convex_hull_2d(sq)
    assert len(hull) == 4 and set(map(tuple, hull)) == {(0, 0), (2, 0), (2, 2), (0, 2)}
    x, y = hull[:, 0], hull[:, 1]
    assert 0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y) > 0  # counter-clockwise
    rs = g.resample_polygon(sq, 16)
    step = np.linalg.norm(np.diff(np.vstack([rs, rs[:1]]), axis=0), axis=1)
    np.testing.assert_allclose(step[step > 0.4], 0.5, atol=1e-9)  # 8 / 16 along the boundary
    model, data, _ = _fake_model()
    poly = g.extract_lbm_polygon_from_mujoco(model, data, "a")
    np.testing.assert_allclose(poly["vertices"].mean(axis=0), 0, atol=1e-12)
    np.testing.assert_allclose(poly["position"], [1.0, 2.0])
    assert abs(poly["angle"] - math.radians(30)) < 1e-12
    geom = g.extract_lbm_polygon_from_mujoco(model, data, "box", is_body=False, use_convex_hull=False,
                                             normalize=False)
    assert abs(geom["angle"] - math.radians(30)) < 1e-12 and geom["vertices"].shape == (4, 2)
