"""Densification statistics: drop-in for
delaunay_rasterization/internal/render_err.py (``render_err``), running the
sm_100a kernels of librm_b200.so.

``render_err(gt_image, camera, model, tile_size, min_t)`` renders the view,
forms the per-pixel L1 and SSIM errors as the reference does
(render_err.py:118-131) and accumulates the per-tet statistics of
calc_tet_err (alphablend_shader_interp.slang:433-599) with
``rm_calc_tet_err``: returns ``(tet_err [T,16], extras)`` with ``extras``
holding ``tet_count``, ``pixel_err``, ``ssim_err``, ``render_img`` and
``cell_values``.  The walk uses the 8x8-pixel lists built beside the tile
lists when present, which visit the same hits in the same order.
"""
import torch

from ... import rasterizer as R
from ...camera import tcam_to_struct
from ...ssim import ssim_map
from .render_grid import RenderGrid
from .tile_shader_slang import vertex_and_tile_shader


def render_err(gt_image, camera, model, tile_size=16, min_t=0.1, **kwargs):
    device = model.device
    indices = model.indices
    vertices = model.vertices
    render_grid = RenderGrid(camera.image_height, camera.image_width, tile_height=tile_size, tile_width=tile_size)
    tcam = dict(tile_height=tile_size, tile_width=tile_size, grid_height=render_grid.grid_height,
                grid_width=render_grid.grid_width, min_t=min_t, **camera.to_dict(device))
    with torch.no_grad():
        sorted_ids, ranges, vs, cc, mask, _ = vertex_and_tile_shader(indices, vertices, tcam, render_grid)
        cell_values = torch.zeros((mask.shape[0], model.feature_dim), device=cc.device)
        _, cell_values[mask] = model.get_cell_values(camera, mask)
        camst = tcam_to_struct(tcam)
        ids, rg, bcam = sorted_ids, ranges, camst
        jitter = torch.full((camera.image_height, camera.image_width, 2), 0.5, device=device)
        fine = R.fine_lists_of(sorted_ids, camst, jitter)
        if fine is not None:
            ids, rg, bcam = fine.sorted_ids, fine.ranges, fine.cam
        img, _, _, _ = R.blend_fwd(ids, rg, indices, vertices, cell_values, jitter, bcam,
                                   tiles_touched=mask.to(torch.int32))
        render_img = img.permute(2, 0, 1)[:3].clip(min=0, max=1)
        pixel_err = (render_img - gt_image).mean(dim=0)
        ssim_err = (1 - ssim_map(render_img, gt_image).mean(dim=0)).clip(min=0, max=1)
        amask = camera.gt_alpha_mask.to(device)
        pixel_err = (pixel_err * amask[0]).contiguous()
        ssim_err = (ssim_err * amask[0]).contiguous()
        render_img = render_img * amask
        tet_err, tet_count = R.calc_tet_err(ids, rg, indices, vertices, cell_values, bcam, pixel_err, ssim_err,
                                            tiles_touched=mask.to(torch.int32))
    return tet_err, dict(tet_count=tet_count, pixel_err=pixel_err, ssim_err=ssim_err, render_img=render_img,
                         cell_values=cell_values)
