"""The triangle screens of the D3Q27 cut-link kernel (csrc/d3q27_solids.cu, cut_cell), restated
in binary32 numpy and checked against the exact ray test on the CPU.

Before its exact Moller-Trumbore tests, cut_cell drops (1) the candidate triangles whose
bounding box misses the box every link of the cell stays in, the body-frame point +- (largest
|component| of the 27 link directions + 2e-3), and (2) for each direction, the triangles whose
bounding box misses that link's own segment box widened by 1e-3. The kernel's hits are the
reference's (a ray cast against every triangle, envs/lbm3d/lbm_func_3d.py:254-316) only if no
screen drops a triangle that the exact test, in binary32 as the kernel computes it, reports hit
with 0 <= t <= 1. Random rotations, meshes and cells; the screens must keep every such pair.
"""
import numpy as np
import pytest

F = np.float32
DIRS = np.array([(x, y, z) for x in (-1, 0, 1) for y in (-1, 0, 1) for z in (-1, 0, 1)], np.float32)


def _quat(rng):
    q = rng.normal(size=4)
    return (q / np.linalg.norm(q)).astype(np.float32)


def _qrot(q, v):
    """qrot of mesh_geom.cuh in binary32: v (2 w^2 - 1) + 2 w (q_v x v) + 2 (q_v . v) q_v."""
    qx, qy, qz, qw = (F(c) for c in q)
    c = F(2) * qw * qw - F(1)
    d = F(2) * (qx * v[..., 0] + qy * v[..., 1] + qz * v[..., 2])
    e = F(2) * qw
    cx = qy * v[..., 2] - qz * v[..., 1]
    cy = qz * v[..., 0] - qx * v[..., 2]
    cz = qx * v[..., 1] - qy * v[..., 0]
    return np.stack([v[..., 0] * c + cx * e + qx * d, v[..., 1] * c + cy * e + qy * d, v[..., 2] * c + cz * e + qz * d],
                    axis=-1).astype(np.float32)


def _mt_hits(tris, o, d):
    """mt_hit of d3q27_solids.cu for every triangle, binary32, no contraction: hit and t."""
    v0 = tris[:, 0]
    e1, e2 = tris[:, 1] - v0, tris[:, 2] - v0
    px = d[1] * e2[:, 2] - d[2] * e2[:, 1]
    py = d[2] * e2[:, 0] - d[0] * e2[:, 2]
    pz = d[0] * e2[:, 1] - d[1] * e2[:, 0]
    det = e1[:, 0] * px + e1[:, 1] * py + e1[:, 2] * pz
    ok = det != F(0)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = F(1) / det
        s = o - v0
        u = (s[:, 0] * px + s[:, 1] * py + s[:, 2] * pz) * inv
        qx = s[:, 1] * e1[:, 2] - s[:, 2] * e1[:, 1]
        qy = s[:, 2] * e1[:, 0] - s[:, 0] * e1[:, 2]
        qz = s[:, 0] * e1[:, 1] - s[:, 1] * e1[:, 0]
        w = (d[0] * qx + d[1] * qy + d[2] * qz) * inv
        t = (e2[:, 0] * qx + e2[:, 1] * qy + e2[:, 2] * qz) * inv
    hit = ok & (u >= 0) & (u <= 1) & (w >= 0) & (u + w <= 1) & (t >= 0) & (t <= 1)
    return hit


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_screens_keep_every_hit(seed):
    rng = np.random.default_rng(seed)
    hits_seen = 0
    for _ in range(40):  # solids
        q = _quat(rng)
        inv_q = np.array([-q[0], -q[1], -q[2], q[3]], np.float32)
        # a body of small triangles around the origin, in the body frame
        centres = rng.uniform(-4, 4, (400, 1, 3))
        tris = (centres + rng.normal(0, 0.35, (400, 3, 3))).astype(np.float32)
        tmn, tmx = tris.min(axis=1), tris.max(axis=1)
        lds_all = _qrot(inv_q, -DIRS)  # body-frame link directions
        r = np.abs(lds_all).max(axis=0) + F(2e-3)  # the cell box half-widths (screen 1)
        for _ in range(60):  # cells (their body-frame points)
            los = rng.uniform(-5, 5, 3).astype(np.float32)
            keep1 = np.all((tmx >= los - r) & (tmn <= los + r), axis=1)
            for di in range(1, 27):
                ld = lds_all[di]
                hit = _mt_hits(tris, los, ld)
                if not hit.any():
                    continue
                hits_seen += int(hit.sum())
                seg_lo = np.minimum(los, los + ld) - F(1e-3)
                seg_hi = np.maximum(los, los + ld) + F(1e-3)
                keep2 = np.all((tmx >= seg_lo) & (tmn <= seg_hi), axis=1)
                assert np.all(keep1[hit]), (seed, di)
                assert np.all(keep2[hit]), (seed, di)
    assert hits_seen > 200
