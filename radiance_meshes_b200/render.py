"""``render()`` with the reference's signature and outputs (utils/train_util.py:15-77).

``camera`` is any object with ``image_height``, ``image_width``,
``gt_alpha_mask`` and ``to_dict(device)`` returning the reference's
camera keys (data/camera.py:72-91); ``model`` has ``vertices``, ``indices`` and,
when ``cell_values`` is not given, ``get_cell_values``/``feature_dim``/
``mask_values`` as in the reference.  ``rasterize()`` is the same pipeline for
callers that hold plain tensors and a ``tcam`` dict.
"""
from __future__ import annotations

import torch

from .camera import tcam_to_struct
from .delaunay_rasterization.internal.alphablend_tiled_slang_interp import AlphaBlendTiledRender
from .delaunay_rasterization.internal.render_grid import RenderGrid
from .delaunay_rasterization.internal.tile_shader_slang import vertex_and_tile_shader

__all__ = ["render", "rasterize", "distortion_loss", "weigh_degree"]


def weigh_degree(sh_coeffs: torch.Tensor, values) -> torch.Tensor:
    """Per-coefficient weight by SH degree, shape [1, C, 1]: coefficient i has
    degree floor(sqrt(i)) and gets values[degree] (utils/eval_sh_py.py:28-40)."""
    C = sh_coeffs.shape[1]
    degrees = torch.floor(torch.sqrt(torch.arange(C, device=sh_coeffs.device, dtype=torch.float32))).long()
    return torch.tensor(values, device=sh_coeffs.device, dtype=sh_coeffs.dtype)[degrees].view(1, C, 1)


def distortion_loss(distortion_img: torch.Tensor) -> torch.Tensor:
    """Per-pixel distortion loss of utils/train_util.py:66-67."""
    total_density = (distortion_img[:, :, 2] ** 2).clip(min=1e-6)
    return (((distortion_img[:, :, 0] - distortion_img[:, :, 1]) + distortion_img[:, :, 4])
            / total_density).clip(min=0)


def rasterize(vertices, indices, cell_values, tcam: dict, ray_jitter=None):
    """Stages (a)-(d) for one view; returns (image [H,W,4], distortion [H,W,5],
    extras dict with sorted ids, ranges, mask, vs, circumcenter)."""
    H, W = int(tcam["image_height"]), int(tcam["image_width"])
    grid = RenderGrid(H, W, tile_width=int(tcam["tile_width"]), tile_height=int(tcam["tile_height"]))
    if ray_jitter is None:
        ray_jitter = torch.full((H, W, 2), 0.5, device=vertices.device)
    sorted_ids, ranges, vs, cc, mask, rect = vertex_and_tile_shader(indices, vertices, tcam, grid)
    img, dist, _ = AlphaBlendTiledRender.apply(sorted_ids, ranges, indices, vertices, cell_values, grid, tcam,
                                               ray_jitter)
    return img, dist, dict(sorted_tetra_idx=sorted_ids, tile_ranges=ranges, mask=mask, vs_tetra=vs,
                           circumcenter=cc, rect_tile_space=rect)


def render(camera, model, cell_values=None, tile_size=16, min_t=0.1, scene_scaling=1, clip_multi=0,
           ray_jitter=None, **kwargs):
    device = model.device
    if ray_jitter is None:
        ray_jitter = 0.5 * torch.ones((camera.image_height, camera.image_width, 2), device=device)
    else:
        assert ray_jitter.shape[0] == camera.image_height
        assert ray_jitter.shape[1] == camera.image_width
        assert ray_jitter.shape[2] == 2
    vertices = model.vertices
    render_grid = RenderGrid(camera.image_height, camera.image_width, tile_height=tile_size,
                             tile_width=tile_size)
    tcam = dict(tile_height=tile_size, tile_width=tile_size, grid_height=render_grid.grid_height,
                grid_width=render_grid.grid_width, min_t=min_t, **camera.to_dict(device))
    sorted_tetra_idx, tile_ranges, vs_tetra, circumcenter, mask, _ = vertex_and_tile_shader(
        model.indices, vertices, tcam, render_grid)
    extras = {}
    sh_reg = 0
    if cell_values is None:
        cell_values = torch.zeros((mask.shape[0], model.feature_dim), device=circumcenter.device)
        if mask.sum() > 0 and model.mask_values:
            shs, values = model.get_cell_values(camera, mask, circumcenter[mask])
            cell_values[mask] = values
        else:
            shs, cell_values = model.get_cell_values(camera, all_circumcenters=circumcenter)
        weighting = weigh_degree(shs, [0, 0.1, 0.5, 1])  # utils/train_util.py:52-53
        sh_reg = ((weighting * shs) ** 2).mean()
    image_rgb, distortion_img, tet_alive = AlphaBlendTiledRender.apply(
        sorted_tetra_idx, tile_ranges, model.indices, vertices, cell_values, render_grid, tcam, ray_jitter)
    alpha = image_rgb.permute(2, 0, 1)[3, ...]
    rgb = image_rgb.permute(2, 0, 1)[:3, ...] * camera.gt_alpha_mask.to(device)
    return {
        "render": rgb,
        "alpha": alpha,
        "distortion_loss": distortion_loss(distortion_img).mean(),
        "mask": mask,
        "sh_reg": sh_reg,
        **extras,
    }
