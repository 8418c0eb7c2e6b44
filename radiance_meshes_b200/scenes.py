"""Seeded synthetic meshes and cameras for the benchmark and test workloads.

No public dataset is available offline, so every workload is generated from a
fixed numpy seed and tetrahedralised with ``scipy.spatial.Delaunay`` (the
reference's ``high_precision`` path, ``models/ingp_color.py:523-528``).
Negative-volume tets are flipped by swapping their first two indices, as in
``models/ingp_color.py:537-541``.  Per-tet features use the reference's
``[T,7]`` layout (density, r, g, b, gx, gy, gz): the colour gradient is one
3-vector whose dot product with (x - v0) is added to all three channels
(``interp_version.slang:53-58``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .camera import look_at_world_view, intrinsics, make_tcam

__all__ = [
    "Mesh",
    "View",
    "delaunay",
    "mixture_points",
    "make_features",
    "workload_plain_forward",
    "workload_gradient_check",
    "workload_training_step",
    "workload_multiview",
    "ring_views",
    "sphere_view",
    "serving_meshes",
    "serving_trace",
]


@dataclass
class Mesh:
    vertices: np.ndarray  # [V,3] float32
    indices: np.ndarray  # [T,4] int32, positive volume
    cell_values: np.ndarray  # [T,7] float32
    name: str = ""


@dataclass
class View:
    world_view: np.ndarray  # [4,4] row-major world->camera
    K: np.ndarray  # [3,3]
    cam_pos: np.ndarray  # [3]
    height: int
    width: int
    fovx: float
    fovy: float
    tile_size: int = 16
    min_t: float = 0.1
    extra: dict = field(default_factory=dict)

    def tcam(self, device=None, tile_size=None):
        return make_tcam(self.world_view, self.K, self.cam_pos, self.height, self.width,
                         tile_size or self.tile_size, self.min_t, self.fovx, self.fovy, device)


def delaunay(points: np.ndarray) -> np.ndarray:
    from scipy.spatial import Delaunay

    pts = np.asarray(points, np.float64)
    idx = Delaunay(pts).simplices.astype(np.int32)
    t = pts[idx]
    vol = np.einsum("ij,ij->i", np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), t[:, 3] - t[:, 0])
    neg = vol < 0
    idx[neg] = idx[neg][:, [1, 0, 2, 3]]
    return np.ascontiguousarray(idx)


def _random_rotations(rng, n):
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.stack([
        1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w),
        2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w),
        2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y),
    ], 1).reshape(n, 3, 3)
    return R


def _uniform_ball(rng, n, radius):
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.uniform(0.0, 1.0, size=(n, 1)) ** (1.0 / 3.0)
    return d * r


def mixture_points(n_points: int, seed: int, n_gauss: int = 64, centre_radius: float = 8.0,
                   background_radius: float = 10.0, background_frac: float = 0.1) -> np.ndarray:
    """Mixture of anisotropic Gaussians (per-axis scales log-uniform in
    [0.02, 0.5], random rotations, centres uniform in a radius-8 ball) plus a
    uniform background in a radius-10 ball."""
    rng = np.random.default_rng(seed)
    n_bg = int(round(n_points * background_frac))
    n_fg = n_points - n_bg
    centres = _uniform_ball(rng, n_gauss, centre_radius)
    scales = np.exp(rng.uniform(math.log(0.02), math.log(0.5), size=(n_gauss, 3)))
    rots = _random_rotations(rng, n_gauss)
    comp = rng.integers(0, n_gauss, size=n_fg)
    z = rng.normal(size=(n_fg, 3)) * scales[comp]
    fg = np.einsum("nij,nj->ni", rots[comp], z) + centres[comp]
    bg = _uniform_ball(rng, n_bg, background_radius)
    pts = np.concatenate([fg, bg], 0).astype(np.float32)
    return pts


def make_features(n_tets: int, seed: int, mu: float = -1.0, sigma: float = 1.5,
                  grad_sigma: float = 0.1, low_density_frac: float = 0.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    density = np.exp(rng.normal(mu, sigma, size=n_tets))
    if low_density_frac > 0:
        m = rng.uniform(size=n_tets) < low_density_frac
        density[m] = 1e-4
    rgb = rng.uniform(0.0, 1.0, size=(n_tets, 3))
    grd = rng.normal(0.0, grad_sigma, size=(n_tets, 3))
    return np.concatenate([density[:, None], rgb, grd], 1).astype(np.float32)


def _view(pos, target, height, width, fovy_deg=60.0, tile_size=16, min_t=0.1, up=(0.0, 1.0, 0.0)):
    M = look_at_world_view(pos, target, up)
    K, fovx, fovy = intrinsics(height, width, fovy_deg)
    return View(M, K, np.asarray(pos, np.float32), height, width, fovx, fovy, tile_size, min_t)


def workload_plain_forward(tile_size: int = 16):
    """4,096 points uniform in [-1,1]^3 (seed 0), Delaunay; density
    log-normal(-1, 1.5); rgb U[0,1]; gradient N(0, 0.1); one 256x256 camera,
    60 deg fov, at (0,0,-3) looking at the origin with OpenCV axes."""
    rng = np.random.default_rng(0)
    pts = rng.uniform(-1.0, 1.0, size=(4096, 3)).astype(np.float32)
    idx = delaunay(pts)
    cv = make_features(len(idx), seed=100)
    M = np.eye(4, dtype=np.float32)
    M[2, 3] = 3.0
    K, fovx, fovy = intrinsics(256, 256, 60.0)
    view = View(M, K, np.array([0.0, 0.0, -3.0], np.float32), 256, 256, fovx, fovy, tile_size, 0.1)
    return Mesh(pts, idx, cv, "uniform4096"), view


def workload_gradient_check(tile_size: int = 16):
    """2,000 points uniform in the unit ball (seed 1); densities
    log-normal(0, 2); 128x128 camera at distance 3 looking at the origin."""
    rng = np.random.default_rng(1)
    pts = _uniform_ball(rng, 2000, 1.0).astype(np.float32)
    idx = delaunay(pts)
    cv = make_features(len(idx), seed=101, mu=0.0, sigma=2.0)
    view = _view((0.3, 0.4, -2.9), (0.0, 0.0, 0.0), 128, 128, 60.0, tile_size)
    return Mesh(pts, idx, cv, "ball2000"), view


def workload_training_step(n_points: int = 200_000, seed: int = 2, tile_size: int = 16,
                           height: int = 840, width: int = 1297):
    """Mixture-of-Gaussians cloud (default 200k points, ~1.3M tets) with 30% of
    densities set to 1e-4; one 1297x840 camera at (4, 0.5, 0) looking at the
    origin, world up +y, 60 deg vertical fov."""
    pts = mixture_points(n_points, seed)
    idx = delaunay(pts)
    cv = make_features(len(idx), seed=seed + 1000, low_density_frac=0.3)
    view = _view((4.0, 0.5, 0.0), (0.0, 0.0, 0.0), height, width, 60.0, tile_size)
    return Mesh(pts, idx, cv, f"mixture{n_points}"), view


def ring_views(n_views: int, resolutions, radius: float = 4.0, height_offset: float = 0.5,
               tile_size: int = 16):
    views = []
    for k in range(n_views):
        th = 2.0 * math.pi * k / n_views
        pos = (radius * math.cos(th), height_offset, radius * math.sin(th))
        h, w = resolutions[k]
        views.append(_view(pos, (0.0, 0.0, 0.0), h, w, 60.0, tile_size))
    return views


def multiview_cameras(tile_size: int = 16):
    """16 cameras evenly spaced on the radius-4 ring: 8 x 1297x840,
    4 x 1920x1080, 4 x 640x480 (interleaved)."""
    res = [(840, 1297)] * 8 + [(1080, 1920)] * 4 + [(480, 640)] * 4
    order = [0, 8, 1, 12, 2, 9, 3, 13, 4, 10, 5, 14, 6, 11, 7, 15]
    return ring_views(16, [res[i] for i in order], tile_size=tile_size)


def mixture_mesh(n_points: int, seed: int) -> "Mesh":
    """A mixture cloud tetrahedralised, with the workloads' features (30% of
    densities at 1e-4, feature seed = seed + 1000)."""
    pts = mixture_points(n_points, seed)
    idx = delaunay(pts)
    cv = make_features(len(idx), seed=seed + 1000, low_density_frac=0.3)
    return Mesh(pts, idx, cv, f"mixture{n_points}")


def workload_multiview(n_points: int = 1_000_000, seed: int = 3, tile_size: int = 16):
    """1M mixture points; 16 ring cameras: 8 x 1297x840, 4 x 1920x1080, 4 x 640x480."""
    return mixture_mesh(n_points, seed), multiview_cameras(tile_size)


def sphere_view(rng, height: int, width: int, radius: float = 4.0, tile_size: int = 16) -> View:
    """Camera at a uniformly random point of the radius-`radius` sphere,
    looking at the origin (world up +y, or +x when looking along y)."""
    d = rng.normal(size=3)
    d /= np.linalg.norm(d)
    up = (0.0, 1.0, 0.0) if abs(d[1]) < 0.99 else (1.0, 0.0, 0.0)
    return _view(tuple(radius * d), (0.0, 0.0, 0.0), height, width, 60.0, tile_size, up=up)


SERVING_RESOLUTIONS = [(480, 640), (720, 1280), (1080, 1920)]


def serving_meshes(point_counts=(250_000, 1_000_000, 3_000_000), seeds=(4, 5, 6)):
    """The resident meshes of the serving workload: mixture clouds of the
    given sizes (30% of densities at 1e-4), one seed each."""
    out = []
    for n, s in zip(point_counts, seeds):
        pts = mixture_points(n, s)
        idx = delaunay(pts)
        cv = make_features(len(idx), seed=s + 1000, low_density_frac=0.3)
        out.append(Mesh(pts, idx, cv, f"mixture{n}"))
    return out


def serving_trace(n_requests: int, rate_hz: float, mesh_names, seed: int = 7, resolutions=None,
                  tile_size: int = 16, radius: float = 4.0):
    """Poisson request stream: exponential inter-arrival times at `rate_hz`,
    each request picking a mesh uniformly, a camera uniformly on the sphere
    and a resolution uniformly from `resolutions`.  Returns a list of
    (arrival_s, mesh_name, View)."""
    rng = np.random.default_rng(seed)
    resolutions = resolutions or SERVING_RESOLUTIONS
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=n_requests))
    out = []
    for k in range(n_requests):
        name = mesh_names[int(rng.integers(0, len(mesh_names)))]
        h, w = resolutions[int(rng.integers(0, len(resolutions)))]
        out.append((float(t[k]), name, sphere_view(rng, h, w, radius, tile_size)))
    return out
