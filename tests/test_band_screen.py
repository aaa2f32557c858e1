"""The candidate screen of the D2Q9 cut-link kernel (csrc/d2q9.cu, band_kernel), restated in
binary32 numpy and checked against get_cutcell's crossing test on the CPU.

band_kernel keeps, as a cell's candidate segments, only those whose bounding box meets the
square [x - 1.001, x + 1.001] x [y - 1.001, y + 1.001] that every link of the cell lies in, and
runs get_cutcell (envs/lbm/lbm_func.py:545-607) over them alone. That is the reference's result
only if the screen keeps every segment that get_cutcell, in binary32 as the kernel computes it,
finds crossing a link. Random outlines near random cells at coordinates up to 512 (where binary32
rounding is largest), all 8 links.
"""
import numpy as np
import pytest

F = np.float32
LINKS = [(dx, dy) for dx in (-1, 0, 1) for dy in (-1, 0, 1) if (dx, dy) != (0, 0)]


def _crossing(x, y, dx, dy, cx, cy, ex, ey):
    """get_cutcell's test for link (x - dx, y - dy) -> (x, y) against segments c -> e (binary32,
    the kernel's expression order, cdb from the identity the kernel uses)."""
    ax, ay, bx, by = F(x) - F(dx), F(y) - F(dy), F(x), F(y)
    abc = (ax - cx) * (by - cy) - (ay - cy) * (bx - cx)
    abd = (ax - ex) * (by - ey) - (ay - ey) * (bx - ex)
    cda = (cx - ax) * (ey - ay) - (cy - ay) * (ex - ax)
    cdb = cda + abc - abd
    return ((abc * abd) < F(0)) & ~((cda * cdb) > F(0))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_band_screen_keeps_every_crossing_segment(seed):
    rng = np.random.default_rng(seed)
    crossings = 0
    for _ in range(400):  # cells
        x, y = int(rng.integers(2, 510)), int(rng.integers(2, 510))
        # segments around the cell: short edges of an outline passing nearby, some far
        n = 200
        c = np.stack([x + rng.uniform(-3, 3, n), y + rng.uniform(-3, 3, n)], axis=1)
        ang = rng.uniform(0, 2 * np.pi, n)
        ln = rng.uniform(0.05, 2.5, n)
        e = c + np.stack([np.cos(ang), np.sin(ang)], axis=1) * ln[:, None]
        c, e = c.astype(np.float32), e.astype(np.float32)
        keep = ~((np.maximum(c[:, 0], e[:, 0]) < F(x) - F(1.001)) | (np.minimum(c[:, 0], e[:, 0]) > F(x) + F(1.001)) |
                 (np.maximum(c[:, 1], e[:, 1]) < F(y) - F(1.001)) | (np.minimum(c[:, 1], e[:, 1]) > F(y) + F(1.001)))
        for dx, dy in LINKS:
            hit = _crossing(x, y, dx, dy, c[:, 0], c[:, 1], e[:, 0], e[:, 1])
            crossings += int(hit.sum())
            assert np.all(keep[hit]), (seed, x, y, dx, dy)
    assert crossings > 1000
