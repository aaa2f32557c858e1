"""Test infrastructure only: numpy restatement of the reference's display kernels (the field
diagnostics), the checker for openhomelbm_b200.diagnostics / hl_d2q9_image / hl_d3q27_image.

Every function works in binary32 in the reference's operation order:
  2D, envs/lbm/lbm_func.py: get_u_img 163-166, get_velocity_rgb 169-193, get_vorticity_img
      196-233, get_vorticity_with_solid_img 236-319, point_segment_dist 792-801,
      get_solid_boundary_img 804-866;
  3D, envs/lbm3d/lbm_func_3d.py: slices 753-840, solid overlays 843-987, projections 990-1313,
      any_mesh_hit_along_ray_3d 320-362.
  live view, tools/lbm3d_realtime_control.py: _extract_live_vorticity_slices 68-148,
      _live_vorticity_to_rgba 157-182.
The reference's mesh queries live in NVIDIA Warp (wp.mesh_query_ray,
wp.mesh_query_point_sign_normal), not in the reference tree; they are restated as a
Moller-Trumbore any-hit test and as the closest point (Ericson, Real-Time Collision Detection,
5.1.5) plus the parity of ray crossings for inside/outside, the same restatement the CUDA code
uses. Parity of those two queries with Warp is unpinned.
"""
from __future__ import annotations

import numpy as np

F = np.float32
SOLID_MARK = F(1000.0)
ML_SOLID, ML_WALL = 1, 2


def _f(a):
    return np.asarray(a, F)


# ----------------------------------------------------------------------------------- 2D
def u_img(u):
    """u: (2, nx, ny) binary32."""
    ux, uy = _f(u[0]), _f(u[1])
    return np.sqrt(ux * ux + uy * uy)


def velocity_rgb(u, max_velocity):
    m = F(max_velocity)
    ux, uy = _f(u[0]), _f(u[1])
    mag = np.sqrt(ux * ux + uy * uy)
    r = np.clip(mag / m, F(0), F(1))
    g = np.clip((ux + m) / (F(2) * m), F(0), F(1))
    b = np.clip((uy + m) / (F(2) * m), F(0), F(1))
    return np.stack([r, g, b], axis=-1)


def _deriv(f, axis, h):
    """d f / d axis: central inside, one-sided on the two border layers (binary32)."""
    f = _f(f)
    h = F(h)
    out = np.empty_like(f)
    n = f.shape[axis]
    sl = lambda a, b: tuple(slice(a, b) if k == axis else slice(None) for k in range(f.ndim))
    out[sl(1, n - 1)] = (f[sl(2, n)] - f[sl(0, n - 2)]) / (F(2) * h)
    out[sl(0, 1)] = (f[sl(1, 2)] - f[sl(0, 1)]) / h
    out[sl(n - 1, n)] = (f[sl(n - 1, n)] - f[sl(n - 2, n - 1)]) / h
    return out


def vorticity_2d(u, h):
    return _deriv(u[1], 0, h) - _deriv(u[0], 1, h)


def point_segment_dist(px, py, ax, ay, bx, by):
    abx, aby, apx, apy = bx - ax, by - ay, px - ax, py - ay
    len_sq = abx * abx + aby * aby
    if len_sq == F(0):
        return np.sqrt(apx * apx + apy * apy)
    t = min(max((apx * abx + apy * aby) / len_sq, F(0)), F(1))
    cx, cy = ax + abx * t, ay + aby * t
    return np.sqrt((px - cx) * (px - cx) + (py - cy) * (py - cy))


def solid_mask_2d(nx, ny, tf, line_num, position, scale, max_radius, thickness):
    """Inside a polygon (even-odd, +x ray) or within `thickness` of its outline."""
    tf, position, scale, max_radius = _f(tf), _f(position), _f(scale), _f(max_radius)
    th = F(thickness)
    out = np.zeros((nx, ny), bool)
    for x in range(nx):
        for y in range(ny):
            px, py = F(x), F(y)
            min_d, inside = F(1.0e6), False
            for o in range(len(line_num)):
                sc = scale[o] * F(nx)
                cx, cy = position[o]
                if (px - cx) * (px - cx) + (py - cy) * (py - cy) > max_radius[o] * sc * sc + th:
                    continue
                n, cross = int(line_num[o]), 0
                for k in range(n):
                    x1, y1 = tf[o, k]
                    x2, y2 = tf[o, (k + 1) % n]
                    d = point_segment_dist(px, py, x1, y1, x2, y2)
                    min_d = min(min_d, d)
                    if (y1 > py) != (y2 > py):
                        ix = x1 + (py - y1) * (x2 - x1) / (y2 - y1)
                        if px < ix:
                            cross += 1
                if cross % 2 == 1:
                    inside = True
            out[x, y] = inside or min_d < th
    return out


# ----------------------------------------------------------------------------------- 3D
def vorticity_3d(u, axis, h):
    """Component along `axis`: z dv/dx - du/dy, x dw/dy - dv/dz, y du/dz - dw/dx. u: (3, nx, ny, nz)."""
    if axis == 2:
        return _deriv(u[1], 0, h) - _deriv(u[0], 1, h)
    if axis == 0:
        return _deriv(u[2], 1, h) - _deriv(u[1], 2, h)
    return _deriv(u[0], 2, h) - _deriv(u[2], 0, h)


def plane(field, axis, index):
    """The plane normal to `axis` at `index`, the other axes in increasing order."""
    return np.take(field, index, axis=axis)


def wall_mask(shape, flag=None):
    if flag is not None:
        return np.asarray(flag) == ML_WALL
    m = np.zeros(shape, bool)
    m[0], m[-1], m[:, 0], m[:, -1], m[:, :, 0], m[:, :, -1] = True, True, True, True, True, True
    return m


def projection(u, axis, kind, h, flag=None):
    """kind 0: max |u| along axis (walls skipped); 1: |u| of the first cell above 1e-8 from the
    high end; 2: vorticity component along axis of largest magnitude over the interior layers."""
    mag = np.sqrt(_f(u[0]) ** 2 + _f(u[1]) ** 2 + _f(u[2]) ** 2)
    walls = wall_mask(mag.shape, flag)
    n = mag.shape[axis]
    if kind == 0:
        return np.where(walls, F(0), mag).max(axis=axis).astype(F)
    if kind == 1:
        m = np.moveaxis(np.where(walls, F(0), mag), axis, -1)[..., ::-1]
        hit = m > F(1e-8)
        first = np.argmax(hit, axis=-1)
        val = np.take_along_axis(m, first[..., None], axis=-1)[..., 0]
        return np.where(hit.any(axis=-1), val, F(0)).astype(F)
    v = np.moveaxis(vorticity_3d(u, axis, h), axis, -1)
    w = np.moveaxis(walls, axis, -1)
    best = np.zeros(v.shape[:-1], F)
    for l in range(1, n - 1):
        cand = v[..., l]
        take = (~w[..., l]) & (np.abs(cand) > np.abs(best))
        best = np.where(take, cand, best)
    return best


def _qrot(q, v):
    """Rotation by the unit quaternion q = (x, y, z, w) (binary32, the CUDA expression order)."""
    qx, qy, qz, qw = (F(c) for c in q)
    v = _f(v)
    c = F(2) * qw * qw - F(1)
    d = F(2) * (qx * v[..., 0] + qy * v[..., 1] + qz * v[..., 2])
    e = F(2) * qw
    cx = qy * v[..., 2] - qz * v[..., 1]
    cy = qz * v[..., 0] - qx * v[..., 2]
    cz = qx * v[..., 1] - qy * v[..., 0]
    return np.stack([v[..., 0] * c + cx * e + qx * d, v[..., 1] * c + cy * e + qy * d,
                     v[..., 2] * c + cz * e + qz * d], axis=-1)


def _to_body(t, p):
    """Point p (..., 3) into the body frame of transform t = (px, py, pz, qx, qy, qz, qw)."""
    t = _f(t)
    q_inv = (-t[3], -t[4], -t[5], t[6])
    pi = -_qrot(q_inv, t[:3])
    return _qrot(q_inv, p) + pi


def ray_any_hit(tris, o, d, max_t):
    """Any double-sided hit 0 <= t <= max_t (tris (T, 3, 3), o and d (3,))."""
    tris = _f(tris)
    v0, v1, v2 = tris[:, 0], tris[:, 1], tris[:, 2]
    e1, e2 = v1 - v0, v2 - v0
    p = np.cross(np.broadcast_to(d, e2.shape), e2).astype(F)
    det = (e1 * p).sum(-1)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = F(1) / det
        s = o - v0
        u = (s * p).sum(-1) * inv
        q = np.cross(s, e1).astype(F)
        w = (np.broadcast_to(d, q.shape) * q).sum(-1) * inv
        t = (e2 * q).sum(-1) * inv
    ok = (det != 0) & (u >= 0) & (u <= 1) & (w >= 0) & (u + w <= 1) & (t >= 0) & (t <= F(max_t))
    return bool(ok.any())


def silhouette(shape, axis, tri_offset, tris, transforms, scale_sizes):
    """Columns whose ray from beyond the high end of `axis` hits a mesh (any_mesh_hit_along_ray_3d)."""
    na, nb = [shape[k] for k in range(3) if k != axis]
    nl = shape[axis]
    out = np.zeros((na, nb), bool)
    for i in range(na):
        for j in range(nb):
            c = [0, 0, 0]
            others = [k for k in range(3) if k != axis]
            c[others[0]], c[others[1]] = i, j
            origin = _f(c)
            origin[axis] = F(nl) + F(1)
            d = np.zeros(3, F)
            d[axis] = F(-1)
            for o in range(len(tri_offset) - 1):
                t0, t1 = int(tri_offset[o]), int(tri_offset[o + 1])
                if t1 == t0:
                    continue
                sc = _f(scale_sizes[o])
                lo = _to_body(transforms[o], origin) / sc
                t = _f(transforms[o])
                ld = _qrot((-t[3], -t[4], -t[5], t[6]), d) / sc
                if ray_any_hit(tris[t0:t1], lo, ld, F(nl) + F(2)):
                    out[i, j] = True
                    break
    return out


def _tri_dist2(tris, p):
    """Squared distance from p (3,) to each triangle (T, 3, 3): closest point by Voronoi region
    (Ericson 5.1.5), binary32 in the CUDA order."""
    tris = _f(tris)
    a, b, c = tris[:, 0], tris[:, 1], tris[:, 2]
    ab, ac = b - a, c - a
    ap, bp, cp = p - a, p - b, p - c
    dot = lambda x, y: (x * y).sum(-1, dtype=F)
    d1, d2, d3, d4, d5, d6 = dot(ab, ap), dot(ac, ap), dot(ab, bp), dot(ac, bp), dot(ab, cp), dot(ac, cp)
    vc, vb, va = d1 * d4 - d3 * d2, d5 * d2 - d1 * d6, d3 * d6 - d5 * d4
    out = np.empty(len(tris), F)
    for k in range(len(tris)):
        if d1[k] <= 0 and d2[k] <= 0:
            q = a[k]
        elif d3[k] >= 0 and d4[k] <= d3[k]:
            q = b[k]
        elif vc[k] <= 0 and d1[k] >= 0 and d3[k] <= 0:
            q = a[k] + (d1[k] / (d1[k] - d3[k])) * ab[k]
        elif d6[k] >= 0 and d5[k] <= d6[k]:
            q = c[k]
        elif vb[k] <= 0 and d2[k] >= 0 and d6[k] <= 0:
            q = a[k] + (d2[k] / (d2[k] - d6[k])) * ac[k]
        elif va[k] <= 0 and (d4[k] - d3[k]) >= 0 and (d5[k] - d6[k]) >= 0:
            q = b[k] + ((d4[k] - d3[k]) / ((d4[k] - d3[k]) + (d5[k] - d6[k]))) * (c[k] - b[k])
        else:
            den = F(1) / (va[k] + vb[k] + vc[k])
            q = a[k] + ab[k] * (vb[k] * den) + ac[k] * (vc[k] * den)
        r = p - q
        out[k] = dot(r, r)
    return out


def _crossings(tris, o):
    """Crossings with t > 0 of the ray from o along the fixed direction of the CUDA code."""
    tris = _f(tris)
    d = _f([0.5773503, 0.5773491, 0.5773515])
    v0 = tris[:, 0]
    e1, e2 = tris[:, 1] - v0, tris[:, 2] - v0
    p = np.cross(np.broadcast_to(d, e2.shape), e2).astype(F)
    det = (e1 * p).sum(-1)
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = F(1) / det
        s = o - v0
        u = (s * p).sum(-1) * inv
        q = np.cross(s, e1).astype(F)
        w = (np.broadcast_to(d, q.shape) * q).sum(-1) * inv
        t = (e2 * q).sum(-1) * inv
    return int(((det != 0) & (u >= 0) & (u <= 1) & (w >= 0) & (u + w <= 1) & (t > 0)).sum())


def solid_plane_mask(shape, axis, index, tri_offset, tris, transforms, scale_sizes, thickness, flag=None):
    """The *_with_solid_3d overlay on a slice: flagged ML_SOLID, or inside a mesh, or within
    `thickness` of it (query radius 100)."""
    others = [k for k in range(3) if k != axis]
    out = np.zeros((shape[others[0]], shape[others[1]]), bool)
    for i in range(out.shape[0]):
        for j in range(out.shape[1]):
            c = [0, 0, 0]
            c[axis], c[others[0]], c[others[1]] = index, i, j
            if flag is not None and flag[tuple(c)] == ML_SOLID:
                out[i, j] = True
                continue
            for o in range(len(tri_offset) - 1):
                t0, t1 = int(tri_offset[o]), int(tri_offset[o + 1])
                if t1 == t0:
                    continue
                lo = _to_body(transforms[o], _f(c)) / _f(scale_sizes[o])
                best = _tri_dist2(tris[t0:t1], lo).min()
                if best > F(100) * F(100):
                    continue
                if _crossings(tris[t0:t1], lo) % 2 == 1 or np.sqrt(best) < F(thickness):
                    out[i, j] = True
                    break
    return out


# ------------------------------------------------------------------------------ live view
LIVE_BINS = 256
LIVE_LOG_MIN = F(-18.420680743952367)  # log(1e-8)
LIVE_LOG_MAX = F(0.0)


def live_slices(u, positions, width, height, stride, slice_axis, color_axis, margin):
    """_extract_live_vorticity_slices (tools/lbm3d_realtime_control.py:68-142): the vorticity
    component `color_axis` on planes normal to `slice_axis` at `positions`, in-plane samples
    p * stride (p < width) and q * stride (q < height) clamped to the grid, flattened as
    (slice, q, p). A position outside the grid gives zeros (the CUDA kernel's rule; the
    reference would index out of bounds). u: (3, nx, ny, nz) binary32."""
    u = _f(u)
    n = u.shape[1:]
    out = np.zeros((len(positions), height, width), F)
    P, Q = np.meshgrid(np.arange(width), np.arange(height))
    for k, pos in enumerate(positions):
        if not 0 <= pos < n[slice_axis]:
            continue
        full = np.full(P.shape, pos)
        if slice_axis == 0:
            x, y, z = full, np.minimum(P * stride, n[1] - 1), np.minimum(Q * stride, n[2] - 1)
        elif slice_axis == 1:
            x, y, z = np.minimum(P * stride, n[0] - 1), full, np.minimum(Q * stride, n[2] - 1)
        else:
            x, y, z = np.minimum(P * stride, n[0] - 1), np.minimum(Q * stride, n[1] - 1), full
        xm, xp = np.maximum(x - 1, 0), np.minimum(x + 1, n[0] - 1)
        ym, yp = np.maximum(y - 1, 0), np.minimum(y + 1, n[1] - 1)
        zm, zp = np.maximum(z - 1, 0), np.minimum(z + 1, n[2] - 1)
        inv_dx = F(1) / np.maximum(xp - xm, 1).astype(F)
        inv_dy = F(1) / np.maximum(yp - ym, 1).astype(F)
        inv_dz = F(1) / np.maximum(zp - zm, 1).astype(F)
        if color_axis == 0:
            v = (u[2][x, yp, z] - u[2][x, ym, z]) * inv_dy - (u[1][x, y, zp] - u[1][x, y, zm]) * inv_dz
        elif color_axis == 1:
            v = (u[0][x, y, zp] - u[0][x, y, zm]) * inv_dz - (u[2][xp, y, z] - u[2][xm, y, z]) * inv_dx
        else:
            v = (u[1][xp, y, z] - u[1][xm, y, z]) * inv_dx - (u[0][x, yp, z] - u[0][x, ym, z]) * inv_dy
        edge = ((x < margin) | (x >= n[0] - margin) | (y < margin) | (y >= n[1] - margin) | (z < margin) |
                (z >= n[2] - margin))
        out[k] = np.where(edge, F(0), v)
    return out.reshape(-1)


def live_histogram(values):
    """The 256-bin histogram of log|value| over [log 1e-8, log 1] for |value| > 1e-8
    (tools/lbm3d_realtime_control.py:143-148), with the logarithm in binary64; and how many
    values lie within 1e-4 of a bin edge (in bins), whose bin a binary32 logarithm may move."""
    mag = np.abs(_f(values))
    m = mag[mag > F(1e-8)].astype(np.float64)
    c = np.clip((np.log(m) - float(LIVE_LOG_MIN)) / (float(LIVE_LOG_MAX) - float(LIVE_LOG_MIN)), 0.0, 0.999999)
    pos = c * LIVE_BINS
    hist = np.bincount(pos.astype(np.int64), minlength=LIVE_BINS)
    frac = pos - np.floor(pos)
    return hist, int(((frac < 1e-4) | (frac > 1 - 1e-4)).sum())


def live_rgba(values, vmax, alpha):
    """_live_vorticity_to_rgba (tools/lbm3d_realtime_control.py:157-182) in binary32: uint8
    (n, 4)."""
    v = _f(values)
    t0 = np.clip(F(0.5) + F(0.5) * v / np.maximum(F(vmax), F(1e-8)), F(0), F(1))
    low = t0 < F(0.5)
    t_lo = t0 * F(2)
    t_hi = (t0 - F(0.5)) * F(2)
    r = np.where(low, F(255) * t_lo, F(255))
    g = np.where(low, F(255) * t_lo, F(255) * (F(1) - t_hi))
    b = np.where(low, F(255), F(255) * (F(1) - t_hi))
    a = np.full_like(v, F(255) * np.clip(F(alpha), F(0), F(1)))
    return np.stack([r, g, b, a], axis=1).astype(np.uint8)


# ---------------------------------------------------------------------- 2D realtime view
def uimg_rgba(img, mode, vmax):
    """lbm_uimg_to_rgba_kernel (tools/lbm2d_realtime_control.py:417-464) in binary32: uint8
    (ny, nx, 4) from an (nx, ny) image."""
    v = _f(img)
    if mode == 2:
        c = (F(1) - np.clip(v, F(0), F(1))) * F(255)
        r = g = b = c
    elif mode == 1:
        n = np.clip(F(0.5) + F(0.5) * v / np.maximum(F(vmax), F(1e-6)), F(0), F(1))
        lo = n < F(0.5)
        t_lo, t_hi = n * F(2), (n - F(0.5)) * F(2)
        r = np.where(lo, F(255) * t_lo, F(255))
        g = np.where(lo, F(255) * t_lo, F(255) * (F(1) - t_hi))
        b = np.where(lo, F(255), F(255) * (F(1) - t_hi))
        solid = v >= F(999)
        r, g, b = (np.where(solid, F(200), c) for c in (r, g, b))
    else:
        n = np.clip(v / np.maximum(F(vmax), F(1e-6)), F(0), F(1))
        r, g, b = F(255) * n, F(180) * n * n, F(60) * (F(1) - n)
    out = np.stack([r, g, b, np.full_like(v, F(255))], axis=-1).astype(np.uint8)
    return np.ascontiguousarray(out.transpose(1, 0, 2))


def local_force(nx, ny, cx, cy, rx, ry, fx, fy):
    """set_local_force_kernel (tools/lbm2d_realtime_control.py:144-157) in binary32:
    (forcex, forcey), each (nx, ny)."""
    x = np.arange(nx, dtype=F)[:, None]
    y = np.arange(ny, dtype=F)[None, :]
    dx = (x - F(cx)) / np.maximum(F(rx), F(1e-6))
    dy = (y - F(cy)) / np.maximum(F(ry), F(1e-6))
    w = np.maximum(F(0), F(1) - (dx * dx + dy * dy))
    return F(fx) * w, F(fy) * w
