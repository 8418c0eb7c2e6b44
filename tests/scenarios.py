"""Seeded test scenes following the reference's renderer tests.

tests/single_tet_test.py (one random tet, 32x32, 90 deg focal convention of
utils/compare_quad.py:35-57, density 10, camera inside / outside / on a face)
and tests/multi_tet_test.py (10-20 points in a radius-10/100 ball, 16x16
image, 8x8 tiles, camera at the cloud centre or outside looking in), re-seeded
with numpy so they are deterministic on the CPU.
"""
import math

import numpy as np

from radiance_meshes_b200.camera import make_tcam
from radiance_meshes_b200.scenes import delaunay


def _rot(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def compare_quad_tcam(c2w_R, origin, height, width, tile_size, tmin=0.01, fov=90.0):
    """Camera of utils/compare_quad.py:35-57: f = H / tan(fov/2)."""
    f = height / math.tan(fov * math.pi / 180 / 2.0)
    K = np.array([[f, 0, width / 2], [0, f, height / 2], [0, 0, 1]], np.float32)
    c2w = np.eye(4)
    c2w[:3, :3] = c2w_R
    c2w[:3, 3] = origin
    w2c = np.linalg.inv(c2w).astype(np.float32)
    return make_tcam(w2c, K, np.asarray(origin, np.float32), height, width, tile_size, tmin)


def look_from(pos, target, height, width, tile_size, tmin=0.01):
    z = np.asarray(target, np.float64) - np.asarray(pos, np.float64)
    z /= np.linalg.norm(z)
    x = np.cross(z, [0.0, 1.0, 0.0])
    if np.linalg.norm(x) < 1e-6:
        x = np.cross(z, [1.0, 0.0, 0.0])
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return compare_quad_tcam(np.stack([x, y, z], 1), pos, height, width, tile_size, tmin)


def single_tet(seed, view="center", radius=0.4, offset=1.0):
    rng = np.random.default_rng(seed)
    verts = ((rng.uniform(size=(4, 3)) * 2 - 1) * radius).astype(np.float32)
    idx = np.array([[0, 1, 2, 3]], np.int32)
    t = verts[idx[0]].astype(np.float64)
    if np.linalg.det(np.stack([t[1] - t[0], t[2] - t[0], t[3] - t[0]])) < 0:
        idx = idx[:, [1, 0, 2, 3]]
    cv = np.array([[10.0, 0.25, 0.5, 0.1, -0.15, 0.25, 0.1]], np.float32)
    if view == "center":
        b = rng.uniform(size=4)
        b /= b.sum()
        origin = verts.T.astype(np.float64) @ b
        tcam = compare_quad_tcam(_rot(rng), origin, 32, 32, 16)
    elif view == "face":
        fi = [[1, 2, 3], [0, 2, 3], [0, 1, 3], [0, 1, 2]][int(rng.integers(0, 4))]
        fv = verts[fi].astype(np.float64)
        b = rng.uniform(size=3)
        b /= b.sum()
        p = fv.T @ b
        n = np.cross(fv[1] - fv[0], fv[2] - fv[0])
        n /= np.linalg.norm(n)
        pos = p + n * (rng.uniform() * 2 - 1) * offset
        tcam = look_from(pos, verts.mean(0), 32, 32, 16)
    else:  # outside, looking at the tet
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        tcam = look_from(d * (radius * 4 + offset), verts.mean(0), 32, 32, 16)
    return verts, idx, cv, tcam


def multi_tet(seed, n_points=20, radius=10.0, view="center", offset_mag=10.0, tile=8):
    rng = np.random.default_rng(seed)
    pts = (rng.uniform(size=(n_points * 2, 3)) * 2 - 1) * radius
    pts = pts[np.linalg.norm(pts, axis=1) <= radius][:n_points].astype(np.float32)
    idx = delaunay(pts)
    N = len(idx)
    cols = rng.uniform(size=(N, 3))
    grd = (2 * rng.uniform(size=(N, 3)) - 1) / math.sqrt(3) / radius
    cv = np.concatenate([np.ones((N, 1)), cols, grd], 1).astype(np.float32)
    if view in ("center", "random_point"):
        # "center": the cloud point nearest the centroid; "random_point": any
        # cloud point (tests/multi_tet_test.py:92-94 picks a random one)
        k = int(np.argmin(np.linalg.norm(pts - pts.mean(0), axis=1))) if view == "center" else \
            int(rng.integers(0, len(pts)))
        tcam = compare_quad_tcam(_rot(rng), pts[k].astype(np.float64), 16, 16, tile)
    else:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        tcam = look_from(d * (radius + offset_mag), pts.mean(0), 16, 16, tile)
    return pts, idx, cv, tcam
