"""Triangle bins of the D3Q27 cut links (lbm3d/lbm_solver_3d.py triangle_bins), checked on the CPU.

The cut-link kernels look up the bin of a cell's body-frame point and ray-cast only the
triangles that bin lists. The result is the reference's (a ray cast against every triangle,
envs/lbm3d/lbm_func_3d.py:254-316) only if a bin lists every triangle that a link from any point
in it can reach: links are at most sqrt(3) long, the bins list every triangle whose bounding box
widened by 1.75 meets them, and the grid spans the mesh's box widened the same way. These tests
check that by brute force on random meshes: box distances, and the 26 lattice links themselves
(Moller-Trumbore, as the kernels test them).
"""
import numpy as np
import pytest

from openhomelbm_b200.lbm3d.lbm_solver_3d import triangle_bins

REACH = float(np.sqrt(3.0))
DIRS = np.array([(x, y, z) for x in (-1, 0, 1) for y in (-1, 0, 1) for z in (-1, 0, 1) if (x, y, z) != (0, 0, 0)],
                np.float64)


def _mesh(rng, n_small=300, n_large=6):
    """Small triangles scattered in a 12^3 box and a few large ones spanning many bins."""
    centres = rng.uniform(0.0, 12.0, (n_small, 1, 3))
    small = centres + rng.normal(0.0, 0.4, (n_small, 3, 3))
    large = rng.uniform(-2.0, 14.0, (n_large, 3, 3))
    return np.concatenate([small, large]).astype(np.float32)


def _bin_list(box, dims, start, lst, p):
    """The triangles listed for point p (None: p lies outside the grid), as the kernels look it up."""
    f = (p - np.array(box[:3])) / box[3]
    if not (np.all(f >= 0) and np.all(f < np.array(dims))):
        return None
    i = f.astype(np.int64)
    b = (i[0] * dims[1] + i[1]) * dims[2] + i[2]
    return set(lst[start[b]:start[b + 1]].tolist())


def _box_distance(tris, p):
    lo, hi = tris.min(axis=1), tris.max(axis=1)
    d = np.maximum(np.maximum(lo - p, p - hi), 0.0)
    return np.linalg.norm(d, axis=1)


def _segment_hits(tris, o, d):
    """Triangles the segment o -> o + d crosses (double-sided Moller-Trumbore, 0 <= t <= 1)."""
    v0, e1, e2 = tris[:, 0], tris[:, 1] - tris[:, 0], tris[:, 2] - tris[:, 0]
    pv = np.cross(d, e2)
    det = np.einsum("ij,ij->i", e1, pv)
    ok = np.abs(det) > 1e-12
    inv = np.where(ok, 1.0 / np.where(ok, det, 1.0), 0.0)
    s = o - v0
    u = np.einsum("ij,ij->i", s, pv) * inv
    q = np.cross(s, e1)
    w = (q @ d) * inv
    t = np.einsum("ij,ij->i", e2, q) * inv
    return np.nonzero(ok & (u >= 0) & (u <= 1) & (w >= 0) & (u + w <= 1) & (t >= 0) & (t <= 1))[0]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_bins_list_every_triangle_within_reach(seed):
    rng = np.random.default_rng(seed)
    tris = _mesh(rng)
    box, dims, start, lst = triangle_bins(tris)
    t64 = tris.astype(np.float64)
    lo = t64.reshape(-1, 3).min(axis=0) - 3.0
    hi = t64.reshape(-1, 3).max(axis=0) + 3.0
    pts = rng.uniform(lo, hi, (3000, 3))
    # points a hair either side of bin faces, where the lookup's rounding decides the bin
    faces = np.array(box[:3]) + box[3] * rng.integers(0, np.array(dims) + 1, (300, 3))
    pts = np.concatenate([pts, faces + rng.choice([-1e-6, 1e-6], (300, 3))])
    checked = 0
    for p in pts:
        listed = _bin_list(box, dims, start, lst, p)
        near = np.nonzero(_box_distance(t64, p) <= REACH)[0]
        if listed is None:
            assert len(near) == 0, (p, near[:5])
            continue
        missing = set(near.tolist()) - listed
        assert not missing, (p, sorted(missing)[:5])
        checked += len(near)
    assert checked > 0


@pytest.mark.parametrize("seed", [3, 4])
def test_bins_list_every_triangle_a_link_crosses(seed):
    rng = np.random.default_rng(seed)
    tris = _mesh(rng)
    box, dims, start, lst = triangle_bins(tris)
    t64 = tris.astype(np.float64)
    lo = t64.reshape(-1, 3).min(axis=0) - 2.0
    hi = t64.reshape(-1, 3).max(axis=0) + 2.0
    hits = 0
    for p in rng.uniform(lo, hi, (1500, 3)):
        listed = _bin_list(box, dims, start, lst, p)
        for d in DIRS:
            crossed = _segment_hits(t64, p, d)
            if len(crossed) == 0:
                continue
            hits += len(crossed)
            assert listed is not None, (p, d)
            assert set(crossed.tolist()) <= listed, (p, d, sorted(set(crossed.tolist()) - listed)[:5])
    assert hits > 100
